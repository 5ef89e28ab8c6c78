// lps_common.cuh -- device helpers shared by the kernel translation units.
#pragma once
#include <cuda_runtime.h>

#include "lps_device.cuh"

namespace lps {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return __shfl_sync(0xffffffffu, v, 0);
}

// Accumulator of the diagnostics of src/main.cpp:986-1062.  Equal maxima
// resolve to the lower node index, so the argmax is the first node whatever
// the order of combining, as the strict '>' scan of :1000-1001 finds it
// (node index order is cell index order on both paths).
struct DiagAcc {
  double E, Ek, Ep, Px, Py, max_u, max_v, max_a, th_min, th_max, uB, vB;
  int iu, iv, nact;

  __device__ __forceinline__ void init() {
    E = Ek = Ep = Px = Py = 0.0;
    max_u = max_v = max_a = 0.0;
    th_min = 1e30;
    th_max = -1e30;
    uB = vB = 0.0;
    iu = iv = -1;
    nact = 0;
  }
  __device__ __forceinline__ void add_maxima(double2 u, double2 v, double2 a, double th, int idx) {
    const double um = sqrt(u.x * u.x + u.y * u.y);
    const double vm = sqrt(v.x * v.x + v.y * v.y);
    const double am = sqrt(a.x * a.x + a.y * a.y);
    if (um > max_u || (um == max_u && iu >= 0 && idx < iu)) { max_u = um; iu = idx; }
    if (vm > max_v || (vm == max_v && iv >= 0 && idx < iv)) { max_v = vm; iv = idx; }
    max_a = (max_a < am) ? am : max_a;      // std::max(max_a, a_mag)
    th_min = (th < th_min) ? th : th_min;   // std::min(theta_min, theta)
    th_max = (th_max < th) ? th : th_max;   // std::max(theta_max, theta)
  }
  // this = this (+) r
  __device__ __forceinline__ void combine(const DiagAcc &r) {
    E += r.E; Ek += r.Ek; Ep += r.Ep; Px += r.Px; Py += r.Py;
    uB += r.uB; vB += r.vB; nact += r.nact;
    if (r.max_u > max_u || (r.max_u == max_u && r.iu >= 0 && (iu < 0 || r.iu < iu))) { max_u = r.max_u; iu = r.iu; }
    if (r.max_v > max_v || (r.max_v == max_v && r.iv >= 0 && (iv < 0 || r.iv < iv))) { max_v = r.max_v; iv = r.iv; }
    max_a = (max_a < r.max_a) ? r.max_a : max_a;
    th_min = (r.th_min < th_min) ? r.th_min : th_min;
    th_max = (th_max < r.th_max) ? r.th_max : th_max;
  }
  __device__ __forceinline__ void shfl_from(const DiagAcc &s, int off) {
    const unsigned m = 0xffffffffu;
    E = __shfl_down_sync(m, s.E, off); Ek = __shfl_down_sync(m, s.Ek, off);
    Ep = __shfl_down_sync(m, s.Ep, off); Px = __shfl_down_sync(m, s.Px, off);
    Py = __shfl_down_sync(m, s.Py, off); max_u = __shfl_down_sync(m, s.max_u, off);
    max_v = __shfl_down_sync(m, s.max_v, off); max_a = __shfl_down_sync(m, s.max_a, off);
    th_min = __shfl_down_sync(m, s.th_min, off); th_max = __shfl_down_sync(m, s.th_max, off);
    uB = __shfl_down_sync(m, s.uB, off); vB = __shfl_down_sync(m, s.vB, off);
    iu = __shfl_down_sync(m, s.iu, off); iv = __shfl_down_sync(m, s.iv, off);
    nact = __shfl_down_sync(m, s.nact, off);
  }
  __device__ __forceinline__ void warp_reduce() {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      DiagAcc r;
      r.shfl_from(*this, o);
      if ((lane & (2 * o - 1)) == 0) combine(r);  // lane l merges its right neighbour block
    }
  }
  __device__ __forceinline__ void to_partial(DiagPartial *p) const {
    p->E = E; p->Ek = Ek; p->Ep = Ep; p->Px = Px; p->Py = Py;
    p->max_u = max_u; p->max_v = max_v; p->max_a = max_a;
    p->th_min = th_min; p->th_max = th_max; p->uB_sq = uB; p->vB_sq = vB;
    p->iu = iu; p->iv = iv; p->nact = nact; p->pad = 0;
  }
  __device__ __forceinline__ void from_partial(const DiagPartial *p) {
    E = p->E; Ek = p->Ek; Ep = p->Ep; Px = p->Px; Py = p->Py;
    max_u = p->max_u; max_v = p->max_v; max_a = p->max_a;
    th_min = p->th_min; th_max = p->th_max; uB = p->uB_sq; vB = p->vB_sq;
    iu = p->iu; iv = p->iv; nact = p->nact;
  }
  // Block-wide ordered reduction; thread 0 stores the block's partial.
  __device__ void block_reduce_store(DiagPartial *out) {
    __shared__ DiagPartial sh[32];
    warp_reduce();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) to_partial(&sh[w]);
    __syncthreads();
    if (threadIdx.x == 0) {
      DiagAcc t;
      t.from_partial(&sh[0]);
      for (int k = 1; k < nw; k++) {
        DiagAcc r;
        r.from_partial(&sh[k]);
        t.combine(r);
      }
      t.to_partial(out);
    }
  }
};

// Second reduction level: one block per instance folds its node blocks and
// its ABC blocks (in order) into one record appended to the instance's log.
void launch_diag_finish(const InstParams *ip, int n_inst, const DiagPartial *partials, int n_node_blocks,
                        DiagRecord *log, int *log_count, int log_capacity, const int *d_step, cudaStream_t st);
// The same for the dense path's tile partials: instance k folds its tiles
// [tile_begin, tile_begin + tile_count) and then its ABC blocks, which follow
// the n_tiles tile partials.
void launch_diag_finish_tiles(const InstParams *ip, int n_inst, const DiagPartial *partials, int n_tiles,
                              DiagRecord *log, int *log_count, int log_capacity, const int *d_step,
                              cudaStream_t st);

}  // namespace lps
