// lps_diag.cu -- the second level of the diagnostics reduction
// (src/main.cpp:986-1062).
#include "lps_common.cuh"
#include "lps_kernels.cuh"

namespace lps {

// One 256-thread block per instance.  Each thread folds a contiguous run of
// block partials (node blocks, then ABC blocks), then the block folds the
// threads in order; the result is one DiagRecord appended to the log.
__global__ void __launch_bounds__(256)
    k_diag_finish(const InstParams *__restrict__ ip, const DiagPartial *__restrict__ partials, int n_node_blocks,
                  DiagRecord *log, int *log_count, int log_capacity, const int *d_step) {
  const int inst = blockIdx.x;
  const InstParams &P = ip[inst];
  const int nb0 = P.node_begin / kNodeBlock;
  const int nb1 = (P.node_begin + P.node_count + kNodeBlock - 1) / kNodeBlock;
  const int ab0 = n_node_blocks + P.abc_begin / kNodeBlock;
  const int ab1 = n_node_blocks + (P.abc_begin + P.abc_count + kNodeBlock - 1) / kNodeBlock;
  const int n_nb = nb1 - nb0, n_ab = ab1 - ab0, total = n_nb + n_ab;
  const int per = (total + blockDim.x - 1) / blockDim.x;
  DiagAcc acc;
  acc.init();
  for (int k = threadIdx.x * per; k < min(total, (int)(threadIdx.x + 1) * per); k++) {
    const int b = k < n_nb ? nb0 + k : ab0 + (k - n_nb);
    DiagAcc r;
    r.from_partial(partials + b);
    acc.combine(r);
  }
  __shared__ DiagPartial res;
  acc.block_reduce_store(&res);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int cnt = log_count[inst];
    if (cnt < log_capacity) {
      DiagRecord &d = log[(size_t)inst * log_capacity + cnt];
      const int s = *d_step;
      d.t = s * P.dt;
      d.E = res.E; d.Ek = res.Ek; d.Ep = res.Ep; d.Px = res.Px; d.Py = res.Py;
      d.max_u = res.max_u; d.max_v = res.max_v; d.max_a = res.max_a;
      d.th_min = res.th_min; d.th_max = res.th_max; d.uB_sq = res.uB_sq; d.vB_sq = res.vB_sq;
      d.step = s; d.iu = res.iu; d.iv = res.iv; d.nact = res.nact;
    }
    log_count[inst] = cnt + 1;
  }
}

// Dense path: the tile partials of instance k, then its ABC blocks.
__global__ void __launch_bounds__(256)
    k_diag_finish_tiles(const InstParams *__restrict__ ip, const DiagPartial *__restrict__ partials, int n_tiles,
                        DiagRecord *log, int *log_count, int log_capacity, const int *d_step) {
  const int inst = blockIdx.x;
  const InstParams &P = ip[inst];
  const int tb = P.tile_begin, n_tb = P.tile_count;
  const int ab0 = n_tiles + P.abc_begin / kNodeBlock;
  const int n_ab = (P.abc_count + kNodeBlock - 1) / kNodeBlock;
  const int total = n_tb + n_ab;
  const int per = (total + blockDim.x - 1) / blockDim.x;
  DiagAcc acc;
  acc.init();
  for (int k = threadIdx.x * per; k < min(total, (int)(threadIdx.x + 1) * per); k++) {
    DiagAcc r;
    r.from_partial(partials + (k < n_tb ? tb + k : ab0 + (k - n_tb)));
    acc.combine(r);
  }
  __shared__ DiagPartial res;
  acc.block_reduce_store(&res);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int cnt = log_count[inst];
    if (cnt < log_capacity) {
      DiagRecord &d = log[(size_t)inst * log_capacity + cnt];
      const int s = *d_step;
      d.t = s * P.dt;
      d.E = res.E; d.Ek = res.Ek; d.Ep = res.Ep; d.Px = res.Px; d.Py = res.Py;
      d.max_u = res.max_u; d.max_v = res.max_v; d.max_a = res.max_a;
      d.th_min = res.th_min; d.th_max = res.th_max; d.uB_sq = res.uB_sq; d.vB_sq = res.vB_sq;
      d.step = s; d.iu = res.iu; d.iv = res.iv; d.nact = res.nact;
    }
    log_count[inst] = cnt + 1;
  }
}

void launch_diag_finish_tiles(const InstParams *ip, int n_inst, const DiagPartial *partials, int n_tiles,
                              DiagRecord *log, int *log_count, int log_capacity, const int *d_step,
                              cudaStream_t st) {
  k_diag_finish_tiles<<<n_inst, 256, 0, st>>>(ip, partials, n_tiles, log, log_count, log_capacity, d_step);
}

void launch_diag_finish(const InstParams *ip, int n_inst, const DiagPartial *partials, int n_node_blocks,
                        DiagRecord *log, int *log_count, int log_capacity, const int *d_step, cudaStream_t st) {
  k_diag_finish<<<n_inst, 256, 0, st>>>(ip, partials, n_node_blocks, log, log_count, log_capacity, d_step);
}

}  // namespace lps
