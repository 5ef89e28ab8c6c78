// lps_kernels_dense32.cu -- FP32-mixed form of the dense tile kernels, sm_100a.
//
// Same two persistent passes as the FP64 form (lps_kernels_dense.cu), with
// the bond arithmetic in FP32:
//   k_theta32<M>   dilatation (src/main.cpp:736-761) from an FP32 copy of the
//                  predicted displacements
//   k_force32<M>   force (:821-874) in FP32; corrector (:922-925) and the next
//                  predictor (:725-728) in FP64, which also writes the FP32
//                  copy of the next predicted level
// Kept in FP64: the displacement / velocity / acceleration state and its
// Verlet update, theta storage, the absorbing-boundary operators (their own
// kernels are shared with the FP64 form) and the diagnostics.
//
// Per-offset constants are compile-time values in lattice units: on the dense
// path dx = dy and delta = m dx, so with xi = dx (a, b), r = |(a, b)|,
//   beta = 1 (r <= m - 1/2), m + 1/2 - r (r <= m + 1/2), 0    (:98-105)
//   theta_i = (2 dx^3 / m_i) sum beta (a, b) . eta
//   F_i     = alpha dx^2 sum beta xi_hat [ (A'+ - A'-) r + (B'_i + B'+) e+ - (B'_i + B'-) e- ]
// with B' = B / alpha = m_ref / m and A' = dx B' (lambda_PD / alpha) theta,
// alpha = 8 mu / m_ref: material constants stay out of the FP32 arithmetic.
// Each stencil column's partial sum is added to the cell's total with Kahan
// compensation.
#include <cmath>

#include "lps_common.cuh"
#include "lps_dense.cuh"
#include "lps_tile.cuh"

namespace lps {

// Square root by Newton's iteration, for compile-time tables only.
__host__ __device__ constexpr double ct_sqrt(double x) {
  double r = x > 1.0 ? x : 1.0;
  for (int i = 0; i < 100; i++) r = 0.5 * (r + x / r);
  return r;
}

// Per-offset constants in lattice units, evaluated by the compiler for each
// (a, b) of the unrolled stencil.
enum StenQ { kHx, kHy, kR, kGx, kGy, kWx, kWy };

__host__ __device__ constexpr float sten_q(int Q, int M, int a, int b) {
  const double r = ct_sqrt((double)(a * a + b * b));
  const double beta = r <= M - 0.5 ? 1.0 : (r <= M + 0.5 ? M + 0.5 - r : 0.0);
  switch (Q) {
    case kHx: return (float)(a / r);           // xi_hat
    case kHy: return (float)(b / r);
    case kR: return (float)r;                  // |xi| / dx
    case kGx: return (float)(beta * a / r);    // beta xi_hat
    case kGy: return (float)(beta * b / r);
    case kWx: return (float)(beta * a);        // beta (a, b)
    default: return (float)(beta * b);
  }
}

template <int M>
using Region32 = Region<M, 8, 8>;

// Two FP32 values in one 64-bit register pair, for Blackwell's paired FP32
// instructions (add/sub/fma .f32x2: one instruction for the x and y parts).
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 f2_unpack(f32x2 v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// s + x with Kahan's running compensation c (the estimate is s - c).
__device__ __forceinline__ void kahan_add(float &s, float &c, float x) {
  const float y = x - c;
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}

// The dilatation thread owns K (4 or 2) adjacent rows of one column, so a
// staged value it loads feeds the pairs of up to K cells; each cell's sums
// are the same whatever K.  The x and y parts of a bond pair's displacement
// difference and of the column's partial sums travel together in paired FP32
// instructions.  The force thread owns cells (r0, c) and (r0 + 1, c), as in
// the FP64 form.
constexpr int th32_threads(int K) { return kTileRows * kTileCols / K; }

template <int M, bool FULL, int K>
__device__ __forceinline__ void theta_tile32(const float2 *__restrict__ su, const uint8_t *__restrict__ sty, int r0,
                                             int c, float th[K]) {
  using R = Region32<M>;
  const f32x2 *__restrict__ sp = reinterpret_cast<const f32x2 *>(su);
  f32x2 ui[K], part[K];  // own displacement; (x, y) partial sums of the column
  float S[K], C[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    ui[k] = sp[QI<M>(r0 + k, c)];
    part[k] = 0ull;
    S[k] = C[k] = 0.f;
  }
  for_each_pair<M>(
      [&](auto ac, auto bc) {
        constexpr int a = decltype(ac)::value, b = decltype(bc)::value;
        const f32x2 w = f2_pack(sten_q(kWx, M, a, b), sten_q(kWy, M, a, b));
#pragma unroll
        for (int k = 0; k < K; k++) {
          const int r = r0 + k;
          f32x2 d = f2_sub(sp[QI<M>(r + a, c + b)], sp[QI<M>(r - a, c - b)]);
          if (!FULL) {
            // absent neighbours hold u = 0; restore the -u_i of the present side
            const float mp = (sty[(r + a + M) * R::RT + c + b + M] & kExists) ? 1.f : 0.f;
            const float mm = (sty[(r - a + M) * R::RT + c - b + M] & kExists) ? 1.f : 0.f;
            d = f2_fma(f2_pack(mm - mp, mm - mp), ui[k], d);
          }
          part[k] = f2_fma(w, d, part[k]);
        }
      },
      [&](auto) {
#pragma unroll
        for (int k = 0; k < K; k++) {
          const float2 pk = f2_unpack(part[k]);
          kahan_add(S[k], C[k], pk.x + pk.y);
          part[k] = 0ull;
        }
      });
#pragma unroll
  for (int k = 0; k < K; k++) th[k] = S[k] - C[k];
}

template <int M, bool FULL>
__device__ __forceinline__ void force_tile32(const float2 *__restrict__ su, const float2 *__restrict__ sab, int r0,
                                             int c, float F[2][2]) {
  const f32x2 *__restrict__ sp = reinterpret_cast<const f32x2 *>(su);
  f32x2 ui[2];
  float2 ab_i[2];
  float S0[2] = {0.f, 0.f}, C0[2] = {0.f, 0.f}, S1[2] = {0.f, 0.f}, C1[2] = {0.f, 0.f};
  float p0[2] = {0.f, 0.f}, p1[2] = {0.f, 0.f};
#pragma unroll
  for (int k = 0; k < 2; k++) {
    ui[k] = sp[QI<M>(r0 + k, c)];
    ab_i[k] = sab[QI<M>(r0 + k, c)];
  }
  for_each_pair<M>(
      [&](auto ac, auto bc) {
        constexpr int a = decltype(ac)::value, b = decltype(bc)::value;
        constexpr float hx = sten_q(kHx, M, a, b), hy = sten_q(kHy, M, a, b), L = sten_q(kR, M, a, b);
        constexpr float gx = sten_q(kGx, M, a, b), gy = sten_q(kGy, M, a, b);
#pragma unroll
        for (int k = 0; k < 2; k++) {
          const int r = r0 + k;
          const int qp = QI<M>(r + a, c + b), qm = QI<M>(r - a, c - b);
          const float2 abp = sab[qp], abm = sab[qm];
          const float2 d1 = f2_unpack(f2_sub(sp[qp], ui[k]));  // u(+) - u_i
          const float2 d2 = f2_unpack(f2_sub(ui[k], sp[qm]));  // u_i - u(-)
          const float e1 = fmaf(hx, d1.x, hy * d1.y);
          const float e2 = fmaf(hx, d2.x, hy * d2.y);
          float T, wp, wm;
          if (FULL) {
            T = (abp.x - abm.x) * L;
            wp = ab_i[k].y + abp.y;
            wm = ab_i[k].y + abm.y;
          } else {
            // a valid neighbour has B > 0; an absent one has A = B = 0
            const float mp = abp.y > 0.f ? 1.f : 0.f, mm = abm.y > 0.f ? 1.f : 0.f;
            T = fmaf(mp - mm, ab_i[k].x, abp.x - abm.x) * L;
            wp = fmaf(mp, ab_i[k].y, abp.y);
            wm = fmaf(mm, ab_i[k].y, abm.y);
          }
          T = fmaf(wp, e1, T);
          T = fmaf(-wm, e2, T);
          p0[k] = fmaf(T, gx, p0[k]);
          p1[k] = fmaf(T, gy, p1[k]);
        }
      },
      [&](auto) {
#pragma unroll
        for (int k = 0; k < 2; k++) {
          kahan_add(S0[k], C0[k], p0[k]);
          kahan_add(S1[k], C1[k], p1[k]);
          p0[k] = p1[k] = 0.f;
        }
      });
#pragma unroll
  for (int k = 0; k < 2; k++) {
    F[k][0] = S0[k] - C0[k];
    F[k][1] = S1[k] - C1[k];
  }
}

// ---------------------------------------------------------------------------
// Predicted displacements (FP32 copy) -> dilatation, persistent over tiles.
template <int M, int K>
__global__ void __launch_bounds__(th32_threads(K), K == 4 ? 6 : 4)
    k_theta32(const __grid_constant__ CUtensorMap map_u, const __grid_constant__ CUtensorMap map_type, Geo g,
              const DenseTile *__restrict__ tiles, int tile_begin, int n_tiles, StepPtrs p, int pitch, int skip_abc,
              int *sched, int *err) {
  using R = Region32<M>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * R::THETA_STAGE);
  int *s_tile = reinterpret_cast<int *>(bar + 2);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (*(volatile int *)err) return;  // an earlier wait timed out: do nothing
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
    s_tile[0] = sched_next(sched);
  }
  __syncthreads();
  auto issue = [&](int stage, int tile) {
    const DenseTile t = tiles[tile_begin + tile];
    unsigned char *base = smem + stage * R::THETA_STAGE;
    mbar_expect_tx(&bar[stage], R::THETA_TX);
    tma_load_2d(base, &map_u, 2 * t.col, t.row, &bar[stage]);
    tma_load_2d(base + R::T_TY, &map_type, t.col, t.row, &bar[stage]);
  };
  int tile = s_tile[0];
  if (tid == 0 && tile < n_tiles) issue(0, tile);
  int it = 0;
  bool failed = false;
  for (; tile < n_tiles; it++, tile = s_tile[it & 1]) {
    const int stage = it & 1;
    if (tid == 0) {
      const int nx = sched_next(sched);
      s_tile[stage ^ 1] = nx;
      if (nx < n_tiles) issue(stage ^ 1, nx);
    }
    const DenseTile t = tiles[tile_begin + tile];
    const InstParams &P = c_inst[t.inst];
    const float2 *su = reinterpret_cast<const float2 *>(smem + stage * R::THETA_STAGE);
    const uint8_t *sty = reinterpret_cast<const uint8_t *>(smem + stage * R::THETA_STAGE + R::T_TY);
    const int r0 = K * warp;
    const size_t cell0 = (size_t)(t.row + M + r0) * pitch + t.col + M + lane;
    double mi[K];
#pragma unroll
    for (int k = 0; k < K; k++) mi[k] = g.m[cell0 + (size_t)k * pitch];
    const bool landed = mbar_wait_bounded(&bar[stage], (it >> 1) & 1, err);
    if (__syncthreads_or(!landed)) {  // a copy timed out: leave the loop together
      failed = true;
      break;
    }
    float th[K];
    if (t.flags & kTileFull)
      theta_tile32<M, true, K>(su, sty, r0, lane, th);
    else
      theta_tile32<M, false, K>(su, sty, r0, lane, th);
    const double scale = 2.0 * P.dx * P.dy * P.dx;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const uint8_t ty = sty[(r0 + k + M) * R::RT + lane + M];
      if (!(ty & kExists)) continue;
      if (skip_abc && (ty & kActiveAbc)) continue;  // the G_theta kernel writes it
      p.th_np1[cell0 + (size_t)k * pitch] = (mi[k] > 0.0) ? (scale / mi[k]) * (double)th[k] : 0.0;
    }
    fence_proxy_async_smem();
    __syncthreads();  // the stage is refilled at the start of the next-but-one iteration
  }
  if (failed && tid == 0) drain_stages(bar, it, s_tile[(it & 1) ^ 1] < n_tiles, err);
  if (tid == 0) sched_finish(sched);
}

// ---------------------------------------------------------------------------
// Force (FP32) + corrector + next predictor (FP64), persistent over tiles.
// The FP32 sum is F / alpha with alpha = 8 mu / m_ref: coef32 holds
// q = m_ref / m_i for both coefficients, so after the copy lands (theta, coef)
// become (A', B') = (q (lambda_PD / alpha) theta dx, q) in the coef slot --
// B' = 1 exactly at full-horizon nodes -- and the per-instance constants are
// applied once, in FP64, to the finished sum.  Absent neighbours and m <= 0
// get A' = B' = 0.
template <int M>
__global__ void __launch_bounds__(kTileThreads, 3)
    k_force32(const __grid_constant__ CUtensorMap map_u, const __grid_constant__ CUtensorMap map_th,
              const __grid_constant__ CUtensorMap map_coef, const __grid_constant__ CUtensorMap map_type, Geo g,
              const DenseTile *__restrict__ tiles, int tile_begin, int n_tiles, StepPtrs p, int pitch, int abc_on,
              int bump_step, int *d_step, int *sched, int *err) {
  using R = Region32<M>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * R::FORCE_STAGE);
  int *s_tile = reinterpret_cast<int *>(bar + 2);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (*(volatile int *)err) return;  // an earlier wait timed out: do nothing
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
    if (bump_step && blockIdx.x == 0) *d_step += 1;
    s_tile[0] = sched_next(sched);
  }
  __syncthreads();
  auto issue = [&](int stage, int tile) {
    const DenseTile t = tiles[tile_begin + tile];
    unsigned char *base = smem + stage * R::FORCE_STAGE;
    mbar_expect_tx(&bar[stage], R::FORCE_TX);
    tma_load_2d(base, &map_u, 2 * t.col, t.row, &bar[stage]);
    tma_load_2d(base + R::F_TH, &map_th, t.col, t.row, &bar[stage]);
    tma_load_2d(base + R::F_CO, &map_coef, 2 * t.col, t.row, &bar[stage]);
    tma_load_2d(base + R::F_TY, &map_type, t.col, t.row, &bar[stage]);
  };
  int tile = s_tile[0];
  if (tid == 0 && tile < n_tiles) issue(0, tile);
  int it = 0;
  bool failed = false;
  for (; tile < n_tiles; it++, tile = s_tile[it & 1]) {
    const int stage = it & 1;
    if (tid == 0) {
      const int nx = sched_next(sched);
      s_tile[stage ^ 1] = nx;
      if (nx < n_tiles) issue(stage ^ 1, nx);
    }
    const DenseTile t = tiles[tile_begin + tile];
    const InstParams &P = c_inst[t.inst];
    unsigned char *base = smem + stage * R::FORCE_STAGE;
    const float2 *su = reinterpret_cast<const float2 *>(base);
    const double *sth = reinterpret_cast<const double *>(base + R::F_TH);
    float2 *sab = reinterpret_cast<float2 *>(base + R::F_CO);
    const uint8_t *sty = reinterpret_cast<const uint8_t *>(base + R::F_TY);
    const int r0 = 2 * warp;
    const size_t cell0 = (size_t)(t.row + M + r0) * pitch + t.col + M + lane;
    // corrector / predictor inputs of the owned cells, fetched while the copy lands
    const double2 vh0 = p.vh[cell0], vh1 = p.vh[cell0 + pitch];
    const double2 un0 = p.u_np1[cell0], un1 = p.u_np1[cell0 + pitch];
    const bool landed = mbar_wait_bounded(&bar[stage], (it >> 1) & 1, err);
    if (__syncthreads_or(!landed)) {  // a copy timed out: leave the loop together
      failed = true;
      break;
    }
    const float dxf = (float)P.dx;
    for (int q = tid; q < R::CELLS; q += kTileThreads) {
      const int rr = q / R::RC, cc = q - rr * R::RC;
      const float2 co = sab[q];
      const bool valid = (sty[rr * R::RT + cc] & kExists) && co.y >= 0.f;
      sab[q] = valid ? make_float2(co.x * (float)(sth[q] * P.f32_ab) * dxf, co.y) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float F[2][2];
    if (t.flags & kTileFull)
      force_tile32<M, true>(su, sab, r0, lane, F);
    else
      force_tile32<M, false>(su, sab, r0, lane, F);
    const double scale = P.f32_b0 * P.dx * P.dy / P.rho;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const uint8_t ty = sty[(r0 + k + M) * R::RT + lane + M];
      if (!(ty & kExists)) continue;
      const size_t cell = cell0 + (size_t)k * pitch;
      const bool valid = sab[QI<M>(r0 + k, lane)].y > 0.f;  // m_i > 0 (:827-831)
      const double2 acc =
          valid ? make_double2((double)F[k][0] * scale, (double)F[k][1] * scale) : make_double2(0.0, 0.0);
      p.a_np1[cell] = acc;
      if (abc_on && (ty & kActiveAbc)) continue;  // G_v writes v; the next theta kernel predicts u
      // corrector (:924) then the next predictor (:727), FP64
      const double2 vh = k == 0 ? vh0 : vh1;
      double2 v, vh2, un;
      v.x = vh.x + P.half_dt * acc.x;
      v.y = vh.y + P.half_dt * acc.y;
      vh2.x = v.x + P.half_dt * acc.x;
      vh2.y = v.y + P.half_dt * acc.y;
      const double2 u = k == 0 ? un0 : un1;
      un.x = u.x + P.dt * vh2.x;
      un.y = u.y + P.dt * vh2.y;
      p.v_np1[cell] = v;
      p.vh[cell] = vh2;
      p.u_np2[cell] = un;
      p.u32_np2[cell] = make_float2((float)un.x, (float)un.y);
    }
    fence_proxy_async_smem();
    __syncthreads();
  }
  if (failed && tid == 0) drain_stages(bar, it, s_tile[(it & 1) ^ 1] < n_tiles, err);
  if (tid == 0) sched_finish(sched);
}

// ---------------------------------------------------------------------------
// host side
template <int M>
static void prepare32_m(DenseGroup &gr, int n_sm, cudaError_t *out) {
  using R = Region32<M>;
  cudaError_t e;
  *out = cudaSuccess;
  if ((e = cudaFuncSetAttribute(k_theta32<M, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, R::THETA_SMEM)) ||
      (e = cudaFuncSetAttribute(k_theta32<M, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, R::THETA_SMEM)) ||
      (e = cudaFuncSetAttribute(k_force32<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, R::FORCE_SMEM)) ||
      (e = cudaFuncSetAttribute(k_theta32<M, 4>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared)) ||
      (e = cudaFuncSetAttribute(k_theta32<M, 2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared)) ||
      (e = cudaFuncSetAttribute(k_force32<M>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared))) {
    *out = e;
    return;
  }
  int bt = 0, bt2 = 0, bf = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, k_theta32<M, 4>, th32_threads(4), R::THETA_SMEM)) ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt2, k_theta32<M, 2>, th32_threads(2), R::THETA_SMEM)) ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, k_force32<M>, kTileThreads, R::FORCE_SMEM))) {
    *out = e;
    return;
  }
  bt = std::max(bt, 1);
  bf = std::max(bf, 1);
  gr.theta_rows = 4;
  gr.grid_theta = std::min(gr.n_tiles, bt * n_sm);
  gr.grid_force = std::min(gr.n_tiles, bf * n_sm);
  gr.max_theta_ctas = bt;
  gr.max_theta_ctas2 = std::max(bt2, 1);
  gr.max_force_ctas = bf;
}

cudaError_t dense32_prepare_group(DenseGroup &gr, int n_sm) {
  cudaError_t e = cudaErrorInvalidValue;
  LPS_DISPATCH_M(gr.m, prepare32_m, gr, n_sm, &e);
  return e;
}

template <int M, int K>
static void theta32_k(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                      int ring_u, bool skip_abc, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(gr.grid_theta);
  cfg.blockDim = dim3(th32_threads(K));
  cfg.dynamicSmemBytes = Region32<M>::THETA_SMEM;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributePriority;
  attr[0].val.priority = dg.tile_priority;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_theta32<M, K>, gr.maps.u32[ring_u & 1], gr.maps.type, lg.geo, dg.tiles, gr.tile_begin,
                     gr.n_tiles, p, dg.pitch, skip_abc ? 1 : 0, gr.sched, dg.d_err);
}

template <int M>
static void theta32_m(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                      int ring_u, bool skip_abc, cudaStream_t st) {
  if (gr.theta_rows == 2)
    theta32_k<M, 2>(gr, lg, dg, p, ring_u, skip_abc, st);
  else
    theta32_k<M, 4>(gr, lg, dg, p, ring_u, skip_abc, st);
}

template <int M>
static void force32_m(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                      int ring_u, int ring_th, bool abc_on, bool first, int *d_step, cudaStream_t st) {
  k_force32<M><<<gr.grid_force, kTileThreads, Region32<M>::FORCE_SMEM, st>>>(
      gr.maps.u32[ring_u & 1], gr.maps.th[ring_th], gr.maps.coef32, gr.maps.type, lg.geo, dg.tiles, gr.tile_begin,
      gr.n_tiles, p, dg.pitch, abc_on ? 1 : 0, first ? 1 : 0, d_step, gr.sched + 2, dg.d_err);
}

void launch_theta32_group(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                          int ring_u, bool skip_abc, cudaStream_t st) {
  LPS_DISPATCH_M(gr.m, theta32_m, gr, lg, dg, p, ring_u, skip_abc, st);
}

void launch_force32_group(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                          int ring_u, int ring_th, bool abc_on, bool first, int *d_step, cudaStream_t st) {
  LPS_DISPATCH_M(gr.m, force32_m, gr, lg, dg, p, ring_u, ring_th, abc_on, first, d_step, st);
}

}  // namespace lps
