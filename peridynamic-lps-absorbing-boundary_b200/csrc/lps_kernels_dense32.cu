// lps_kernels_dense32.cu -- FP32-mixed form of the dense tile kernels, sm_100a.
//
// Same two persistent passes as the FP64 form (lps_kernels_dense.cu), with
// the bond arithmetic in FP32:
//   k_theta32<M,K>  dilatation (src/main.cpp:736-761) from an FP32 copy of the
//                   predicted displacements; its epilogue also writes the force
//                   pass's per-cell coefficient A' (B' is static)
//   k_force32<M,K>  force (:821-874) in FP32; corrector (:922-925) and the
//                   next predictor (:725-728) in FP64, which also writes the
//                   FP32 copy of the next predicted level
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
//
// No per-neighbour existence test.  Absent cells hold u = 0 and A' = B' = 0,
// so every stencil pair is evaluated the same way, and the terms that an
// absent neighbour contributes wrongly are removed by two static per-cell
// quantities, zero at full-horizon cells:
//   W_i  = sum over present offsets of beta (a, b)
//   Ka_i = sum over absent offsets of beta xi_hat xi_hat^T
// -- theta_i gets -W_i . u_i, F_i gets A'_i W_i + B'_i Ka_i u_i.  Tiles whose
// cells and neighbours all have B' = 1 ("deep" tiles, the interior) use
//   F_i = sum beta xi_hat [ (A'+ - A'-) r + 2 xi_hat . (u(+) + u(-) - 2 u_i) ],
// the same sum with the coefficients folded.  Each stencil column's partial
// sum is added to the cell's total with Kahan compensation.
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

__host__ __device__ constexpr double sten_qd(int Q, int M, int a, int b) {
  const double r = ct_sqrt((double)(a * a + b * b));
  const double beta = r <= M - 0.5 ? 1.0 : (r <= M + 0.5 ? M + 0.5 - r : 0.0);
  switch (Q) {
    case kHx: return a / r;           // xi_hat
    case kHy: return b / r;
    case kR: return r;                // |xi| / dx
    case kGx: return beta * a / r;    // beta xi_hat
    case kGy: return beta * b / r;
    case kWx: return beta * a;        // beta (a, b)
    default: return beta * b;
  }
}
__host__ __device__ constexpr float sten_q(int Q, int M, int a, int b) { return (float)sten_qd(Q, M, a, b); }

// Staged-region geometry of the FP32 tile kernels: the dilatation stages the
// FP32 displacements, the force pass the displacements and the coefficient
// planes A' and B' (one float per cell; B' only for tiles that are not deep).
// The planes' staged rows are RCA floats wide, RC rounded up to 16 bytes, as a
// TMA box's inner extent must be.
template <int M>
struct Region32 {
  static constexpr int RR = kTileRows + 2 * M;
  static constexpr int RC = kTileCols + 2 * M;
  static constexpr int RCA = (RC + 3) / 4 * 4;
  static constexpr int CELLS = RR * RC;
  static constexpr int align128(int x) { return (x + 127) / 128 * 128; }
  static constexpr int U_BYTES = CELLS * 8;
  static constexpr int P_BYTES = RR * RCA * 4;
  static constexpr int THETA_STAGE = align128(U_BYTES);
  static constexpr int THETA_TX = U_BYTES;
  static constexpr int F_A = align128(U_BYTES);
  static constexpr int F_B = align128(F_A + P_BYTES);
  static constexpr int FORCE_STAGE = align128(F_B + P_BYTES);
  static constexpr int FORCE_TX_DEEP = U_BYTES + P_BYTES;
  static constexpr int FORCE_TX = U_BYTES + 2 * P_BYTES;
  static constexpr int THETA_SMEM = 2 * THETA_STAGE + 64;
  static constexpr int FORCE_SMEM = 2 * FORCE_STAGE + 64;
};
// staged coefficient-plane index of tile-relative cell (r, c)
template <int M>
__device__ __forceinline__ int QA(int r, int c) {
  return (r + M) * Region32<M>::RCA + (c + M);
}

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
__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
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

// The same for an (x, y) pair in paired instructions (each lane as kahan_add).
__device__ __forceinline__ void kahan_add2(f32x2 &s, f32x2 &c, f32x2 x) {
  const f32x2 y = f2_sub(x, c);
  const f32x2 t = f2_add(s, y);
  c = f2_sub(f2_sub(t, s), y);
  s = t;
}

// The dilatation thread owns K (4 or 2) adjacent rows of one column, so a
// staged value it loads feeds the pairs of up to K cells; each cell's sums
// are the same whatever K.  The x and y parts of a bond pair's displacement
// difference and of the column's partial sums travel together in paired FP32
// instructions.  The force thread owns cells (r0, c) and (r0 + 1, c).
constexpr int th32_threads(int K) { return kTileRows * kTileCols / K; }

// sum over pairs of beta (a, b) . (u(+) - u(-)), per owned row; absent cells
// contribute u = 0 (the -W . u_i correction is applied by the caller).
template <int M, int K>
__device__ __forceinline__ void theta_tile32(const float2 *__restrict__ su, int r0, int c, float th[K]) {
  const f32x2 *__restrict__ sp = reinterpret_cast<const f32x2 *>(su);
  f32x2 part[K];  // (x, y) partial sums of the column
  float S[K], C[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
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
          const f32x2 d = f2_sub(sp[QI<M>(r + a, c + b)], sp[QI<M>(r - a, c - b)]);
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

// Force sums of cells (r0 + k, c), k < K.  DEEP: every coefficient B' is 1
// (folded form); otherwise the general pair form, whose absent-neighbour terms
// the caller corrects.  Column by column (stencil offset b), the thread walks
// the pairs (a, b) / (-a, -b) in order of a and keeps two sliding windows of K
// staged cells: rows r0 + a + k of column c + b and rows r0 - a + k of column
// c - b.  Each step of a moves both windows by one row, so every staged value
// is loaded once per column and feeds up to K cells from registers.
template <int M, int K, bool DEEP>
__device__ __forceinline__ void force_tile32(const float2 *__restrict__ su, const float *__restrict__ sa,
                                             const float *__restrict__ sb, int r0, int c, float F[K][2]) {
  const f32x2 *__restrict__ sp = reinterpret_cast<const f32x2 *>(su);
  f32x2 ui[K], S[K], Cc[K];
  float bi[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    ui[k] = sp[QI<M>(r0 + k, c)];
    bi[k] = DEEP ? 1.f : sb[QA<M>(r0 + k, c)];
    S[k] = Cc[k] = 0ull;
  }
  const f32x2 m2 = f2_pack(-2.f, -2.f);
  static_for<0, M + 1>([&](auto bc) {
    constexpr int b = decltype(bc)::value;
    constexpr int A = amax(M, b);
    constexpr int a0 = b == 0 ? 1 : -A;  // b = 0: pairs (a, 0) with a > 0
    f32x2 wp[K], wm[K];                  // u at rows r0 + a + k (column c + b), r0 - a + k (column c - b)
    float ap[K], am[K], bp[K], bm[K];    // A', B' there
    float p0[K], p1[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      wp[k] = sp[QI<M>(r0 + a0 + k, c + b)];
      wm[k] = sp[QI<M>(r0 - a0 + k, c - b)];
      ap[k] = sa[QA<M>(r0 + a0 + k, c + b)];
      am[k] = sa[QA<M>(r0 - a0 + k, c - b)];
      if (!DEEP) {
        bp[k] = sb[QA<M>(r0 + a0 + k, c + b)];
        bm[k] = sb[QA<M>(r0 - a0 + k, c - b)];
      }
      p0[k] = p1[k] = 0.f;
    }
    static_for<a0, A + 1>([&](auto ac) {
      constexpr int a = decltype(ac)::value;
      constexpr float hx = sten_q(kHx, M, a, b), hy = sten_q(kHy, M, a, b), L = sten_q(kR, M, a, b);
      constexpr float gx = sten_q(kGx, M, a, b), gy = sten_q(kGy, M, a, b);
#pragma unroll
      for (int k = 0; k < K; k++) {
        float T;
        if (DEEP) {
          // 2 xi_hat . (u(+) + u(-) - 2 u_i) + (A'+ - A'-) r
          const float2 s = f2_unpack(f2_fma(m2, ui[k], f2_add(wp[k], wm[k])));
          const float e = fmaf(2.f * hx, s.x, (2.f * hy) * s.y);
          T = fmaf(L, ap[k] - am[k], e);
        } else {
          const float2 d1 = f2_unpack(f2_sub(wp[k], ui[k]));  // u(+) - u_i
          const float2 d2 = f2_unpack(f2_sub(ui[k], wm[k]));  // u_i - u(-)
          const float e1 = fmaf(hx, d1.x, hy * d1.y);
          const float e2 = fmaf(hx, d2.x, hy * d2.y);
          T = (ap[k] - am[k]) * L;
          T = fmaf(bi[k] + bp[k], e1, T);
          T = fmaf(-(bi[k] + bm[k]), e2, T);
        }
        p0[k] = fmaf(T, gx, p0[k]);
        p1[k] = fmaf(T, gy, p1[k]);
      }
      if constexpr (a < A) {  // slide: + window down a row, - window up a row
#pragma unroll
        for (int k = 0; k + 1 < K; k++) {
          wp[k] = wp[k + 1];
          ap[k] = ap[k + 1];
          if (!DEEP) bp[k] = bp[k + 1];
        }
#pragma unroll
        for (int k = K - 1; k > 0; k--) {
          wm[k] = wm[k - 1];
          am[k] = am[k - 1];
          if (!DEEP) bm[k] = bm[k - 1];
        }
        wp[K - 1] = sp[QI<M>(r0 + a + K, c + b)];
        ap[K - 1] = sa[QA<M>(r0 + a + K, c + b)];
        wm[0] = sp[QI<M>(r0 - a - 1, c - b)];
        am[0] = sa[QA<M>(r0 - a - 1, c - b)];
        if (!DEEP) {
          bp[K - 1] = sb[QA<M>(r0 + a + K, c + b)];
          bm[0] = sb[QA<M>(r0 - a - 1, c - b)];
        }
      }
    });
#pragma unroll
    for (int k = 0; k < K; k++) kahan_add2(S[k], Cc[k], f2_pack(p0[k], p1[k]));
  });
#pragma unroll
  for (int k = 0; k < K; k++) {
    const float2 f = f2_unpack(f2_sub(S[k], Cc[k]));
    F[k][0] = f.x;
    F[k][1] = f.y;
  }
}

// ---------------------------------------------------------------------------
// Predicted displacements (FP32 copy) -> dilatation and the force pass's
// coefficients, persistent over tiles.
template <int M, int K>
__global__ void __launch_bounds__(th32_threads(K), K == 4 ? 6 : 4)
    k_theta32(const __grid_constant__ CUtensorMap map_u, Geo g, const DenseTile *__restrict__ tiles, int tile_begin,
              int n_tiles, StepPtrs p, Dense32 d32, int pitch, int skip_abc, int *sched, int *err) {
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
    mbar_expect_tx(&bar[stage], R::THETA_TX);
    tma_load_2d(smem + stage * R::THETA_STAGE, &map_u, 2 * t.col, t.row, &bar[stage]);
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
    const InstParams &P = g.ip[t.inst];
    const float2 *su = reinterpret_cast<const float2 *>(smem + stage * R::THETA_STAGE);
    const int r0 = K * warp;
    const size_t cell0 = (size_t)(t.row + M + r0) * pitch + t.col + M + lane;
    // the owned cells' static data, fetched while the copy lands; in a full
    // tile every owned cell has m_i = m_ref and B' = 1, so only the types
    const bool full = t.flags & kTileFull;
    double mi[K];
    uint8_t ty[K];
    float q[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      const size_t cell = cell0 + (size_t)k * pitch;
      ty[k] = g.type[cell];
      mi[k] = full ? P.mref : g.m[cell];
      q[k] = full ? 1.f : d32.bp32[cell];
    }
    const bool landed = mbar_wait_bounded(&bar[stage], (it >> 1) & 1, err);
    if (__syncthreads_or(!landed)) {  // a copy timed out: leave the loop together
      failed = true;
      break;
    }
    float th[K];
    theta_tile32<M, K>(su, r0, lane, th);
    const double scale = 2.0 * P.dx * P.dy * P.dx;
    const float dxf = (float)P.dx;
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (!(ty[k] & kExists)) continue;
      const size_t cell = cell0 + (size_t)k * pitch;
      double thd;
      if (skip_abc && (ty[k] & kActiveAbc)) {
        thd = p.th_np1[cell];  // G_theta wrote it a step ahead
      } else {
        float tk = th[k];
        if (!full) {  // absent neighbours: remove their -u_i terms
          const float2 w = d32.w32[cell], ui = su[QI<M>(r0 + k, lane)];
          tk -= fmaf(w.x, ui.x, w.y * ui.y);
        }
        thd = (mi[k] > 0.0) ? (scale / mi[k]) * (double)tk : 0.0;
        if (p.full || (ty[k] & kKeepState)) p.th_np1[cell] = thd;  // the force pass reads A'
      }
      d32.ap32[cell] = q[k] > 0.f ? (float)(thd * P.f32_ab) * q[k] * dxf : 0.f;
    }
    fence_proxy_async_smem();
    __syncthreads();  // the stage is refilled at the start of the next-but-one iteration
  }
  if (failed && tid == 0) drain_stages(bar, it, s_tile[(it & 1) ^ 1] < n_tiles, err);
  if (tid == 0) sched_finish(sched);
}

// ---------------------------------------------------------------------------
// Force (FP32) + corrector + next predictor (FP64), persistent over tiles.
// The FP32 sum is F / alpha with alpha = 8 mu / m_ref; the per-instance
// constants are applied once, in FP64, to the finished sum.  A thread owns K
// (2 or 4) adjacent rows of one column.  Deep tiles stage u and A' only.
constexpr int f32_threads(int K) { return kTileRows * kTileCols / K; }

template <int M, int K>
__global__ void __launch_bounds__(f32_threads(K), K == 4 ? 4 : 3)
    k_force32(const __grid_constant__ CUtensorMap map_u, const __grid_constant__ CUtensorMap map_a,
              const __grid_constant__ CUtensorMap map_b, Geo g, const DenseTile *__restrict__ tiles, int tile_begin,
              int n_tiles, StepPtrs p, Dense32 d32, int pitch, int abc_on, int bump_step, int *d_step, int *sched,
              int *err) {
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
    const bool deep = t.flags & kTileDeep32;
    mbar_expect_tx(&bar[stage], deep ? R::FORCE_TX_DEEP : R::FORCE_TX);
    tma_load_2d(base, &map_u, 2 * t.col, t.row, &bar[stage]);
    tma_load_2d(base + R::F_A, &map_a, t.col, t.row, &bar[stage]);
    if (!deep) tma_load_2d(base + R::F_B, &map_b, t.col, t.row, &bar[stage]);
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
    const InstParams &P = g.ip[t.inst];
    unsigned char *base = smem + stage * R::FORCE_STAGE;
    const float2 *su = reinterpret_cast<const float2 *>(base);
    const float *sa = reinterpret_cast<const float *>(base + R::F_A);
    const float *sb = reinterpret_cast<const float *>(base + R::F_B);
    const bool deep = t.flags & kTileDeep32, full = t.flags & kTileFull;
    const int r0 = K * warp;
    const size_t cell0 = (size_t)(t.row + M + r0) * pitch + t.col + M + lane;
    // corrector / predictor inputs of the owned cells, fetched while the copy
    // lands (two rows per thread; with four, after the sums, to save registers)
    constexpr int KP = K == 2 ? 2 : 0;
    double2 vhp[KP > 0 ? KP : 1], unp[KP > 0 ? KP : 1];
    uint8_t ty[K];
#pragma unroll
    for (int k = 0; k < K; k++) ty[k] = g.type[cell0 + (size_t)k * pitch];
#pragma unroll
    for (int k = 0; k < KP; k++) {
      vhp[k] = p.vh[cell0 + (size_t)k * pitch];
      unp[k] = p.u_np1[cell0 + (size_t)k * pitch];
    }
    const bool landed = mbar_wait_bounded(&bar[stage], (it >> 1) & 1, err);
    if (__syncthreads_or(!landed)) {  // a copy timed out: leave the loop together
      failed = true;
      break;
    }
    float F[K][2];
    if (deep)
      force_tile32<M, K, true>(su, sa, sb, r0, lane, F);
    else
      force_tile32<M, K, false>(su, sa, sb, r0, lane, F);
    const double scale = P.f32_b0 * P.dx * P.dy / P.rho;
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (!(ty[k] & kExists)) continue;
      const size_t cell = cell0 + (size_t)k * pitch;
      const float ai = sa[QA<M>(r0 + k, lane)], bi = deep ? 1.f : sb[QA<M>(r0 + k, lane)];
      if (!full) {  // absent neighbours: A'_i W_i + B'_i Ka_i u_i
        const float2 w = d32.w32[cell], ui = su[QI<M>(r0 + k, lane)];
        const float4 ka = d32.ka32[cell];
        F[k][0] += fmaf(ai, w.x, bi * fmaf(ka.x, ui.x, ka.y * ui.y));
        F[k][1] += fmaf(ai, w.y, bi * fmaf(ka.y, ui.x, ka.z * ui.y));
      }
      const bool valid = bi > 0.f;  // m_i > 0 (:827-831)
      const double2 acc =
          valid ? make_double2((double)F[k][0] * scale, (double)F[k][1] * scale) : make_double2(0.0, 0.0);
      if (p.full || (ty[k] & (kKeepState | kActiveAbc))) p.a_np1[cell] = acc;
      if (abc_on && (ty[k] & kActiveAbc)) continue;  // G_v writes v; the end-of-step kernel predicts u
      // corrector (:924) then the next predictor (:727), FP64
      const double2 vh = KP > 0 ? vhp[k < KP ? k : 0] : p.vh[cell];
      const double2 u = KP > 0 ? unp[k < KP ? k : 0] : p.u_np1[cell];
      double2 v, vh2, un;
      v.x = vh.x + P.half_dt * acc.x;
      v.y = vh.y + P.half_dt * acc.y;
      vh2.x = v.x + P.half_dt * acc.x;
      vh2.y = v.y + P.half_dt * acc.y;
      un.x = u.x + P.dt * vh2.x;
      un.y = u.y + P.dt * vh2.y;
      if (p.full || (ty[k] & kKeepState)) p.v_np1[cell] = v;
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

// Static per-cell data of ratio M (see the top of this file): W_i, Ka_i and
// whether the cell, all its stencil neighbours present, has B' = 1.
template <int M>
static void static32_m(const std::vector<uint8_t> &type, int pitch, long first, long count, std::vector<float2> &w32,
                       std::vector<float4> &ka32) {
  constexpr Sten<M> sten = make_sten<M>();
  constexpr int N = Sten<M>::N;
  // per-offset terms, evaluated once (sten_qd's square root is an iteration
  // meant for compile-time tables)
  double tw[N][2], tk[N][3];
  long nb_off[N];
  for (int j = 0; j < N; j++) {
    const int a = sten.a[j], b = sten.b[j];
    tw[j][0] = sten_qd(kWx, M, a, b);
    tw[j][1] = sten_qd(kWy, M, a, b);
    // beta xi_hat xi_hat^T = g xi_hat^T with g = beta xi_hat
    const double gx = sten_qd(kGx, M, a, b), gy = sten_qd(kGy, M, a, b);
    const double hx = sten_qd(kHx, M, a, b), hy = sten_qd(kHy, M, a, b);
    tk[j][0] = gx * hx;
    tk[j][1] = gx * hy;
    tk[j][2] = gy * hy;
    nb_off[j] = (long)a * pitch + b;
  }
#pragma omp parallel for schedule(static)
  for (long c = first; c < first + count; c++) {
    if (!(type[c] & kExists)) continue;
    double wx = 0, wy = 0, kxx = 0, kxy = 0, kyy = 0;
    for (int j = 0; j < N; j++) {
      if (type[c + nb_off[j]] & kExists) {
        wx += tw[j][0];
        wy += tw[j][1];
      } else {
        kxx += tk[j][0];
        kxy += tk[j][1];
        kyy += tk[j][2];
      }
    }
    w32[c] = make_float2((float)wx, (float)wy);
    ka32[c] = make_float4((float)kxx, (float)kxy, (float)kyy, 0.f);
  }
}

void dense32_static(int m, const std::vector<uint8_t> &type, int pitch, long first, long count,
                    std::vector<float2> &w32, std::vector<float4> &ka32) {
  LPS_DISPATCH_M(m, static32_m, type, pitch, first, count, w32, ka32);
}

template <int M>
static void deep32_m(const std::vector<uint8_t> &type, const std::vector<float2> &coef32, int pitch, long first_owned,
                     bool *deep) {
  constexpr Sten<M> sten = make_sten<M>();
  bool ok = true;
  for (int r = 0; r < kTileRows && ok; r++)
    for (int q = 0; q < kTileCols && ok; q++) {
      const long c = first_owned + (long)r * pitch + q;
      if (!(type[c] & kExists)) continue;
      if (coef32[c].y != 1.0f) ok = false;
      for (int j = 0; j < Sten<M>::N && ok; j++) {
        const long nb = c + (long)sten.a[j] * pitch + sten.b[j];
        if (!(type[nb] & kExists) || coef32[nb].y != 1.0f) ok = false;
      }
    }
  *deep = ok;
}

bool dense32_tile_deep(int m, const std::vector<uint8_t> &type, const std::vector<float2> &coef32, int pitch,
                       long first_owned) {
  bool deep = false;
  LPS_DISPATCH_M(m, deep32_m, type, coef32, pitch, first_owned, &deep);
  return deep;
}

template <int M>
static void prepare32_m(DenseGroup &gr, int n_sm, cudaError_t *out) {
  using R = Region32<M>;
  cudaError_t e;
  *out = cudaSuccess;
  const auto smem = cudaFuncAttributeMaxDynamicSharedMemorySize;
  const auto carve = cudaFuncAttributePreferredSharedMemoryCarveout;
  const int maxs = cudaSharedmemCarveoutMaxShared;
  if ((e = cudaFuncSetAttribute(k_theta32<M, 4>, smem, R::THETA_SMEM)) ||
      (e = cudaFuncSetAttribute(k_theta32<M, 2>, smem, R::THETA_SMEM)) ||
      (e = cudaFuncSetAttribute(k_force32<M, 2>, smem, R::FORCE_SMEM)) ||
      (e = cudaFuncSetAttribute(k_force32<M, 4>, smem, R::FORCE_SMEM)) ||
      (e = cudaFuncSetAttribute(k_theta32<M, 4>, carve, maxs)) || (e = cudaFuncSetAttribute(k_theta32<M, 2>, carve, maxs)) ||
      (e = cudaFuncSetAttribute(k_force32<M, 2>, carve, maxs)) || (e = cudaFuncSetAttribute(k_force32<M, 4>, carve, maxs))) {
    *out = e;
    return;
  }
  int bt = 0, bt2 = 0, bf = 0, bf4 = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, k_theta32<M, 4>, th32_threads(4), R::THETA_SMEM)) ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt2, k_theta32<M, 2>, th32_threads(2), R::THETA_SMEM)) ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, k_force32<M, 2>, f32_threads(2), R::FORCE_SMEM)) ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf4, k_force32<M, 4>, f32_threads(4), R::FORCE_SMEM))) {
    *out = e;
    return;
  }
  bt = std::max(bt, 1);
  bf = std::max(bf, 1);
  gr.theta_rows = 4;
  gr.force_rows = 2;
  gr.grid_theta = std::min(gr.n_tiles, bt * n_sm);
  gr.grid_force = std::min(gr.n_tiles, bf * n_sm);
  gr.max_theta_ctas = bt;
  gr.max_theta_ctas2 = std::max(bt2, 1);
  gr.max_force_ctas = bf;
  gr.max_force_ctas4 = std::max(bf4, 1);
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
  cudaLaunchKernelEx(&cfg, k_theta32<M, K>, gr.maps.u32[ring_u & 1], lg.geo, dg.tiles, gr.tile_begin, gr.n_tiles, p,
                     dg.d32, dg.pitch, skip_abc ? 1 : 0, gr.sched, dg.d_err);
}

template <int M>
static void theta32_m(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                      int ring_u, bool skip_abc, cudaStream_t st) {
  if (gr.theta_rows == 2)
    theta32_k<M, 2>(gr, lg, dg, p, ring_u, skip_abc, st);
  else
    theta32_k<M, 4>(gr, lg, dg, p, ring_u, skip_abc, st);
}

template <int M, int K>
static void force32_k(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p, int ring_u,
                      bool abc_on, bool first, int *d_step, cudaStream_t st) {
  k_force32<M, K><<<gr.grid_force, f32_threads(K), Region32<M>::FORCE_SMEM, st>>>(
      gr.maps.u32[ring_u & 1], gr.maps.ap32, gr.maps.bp32, lg.geo, dg.tiles, gr.tile_begin, gr.n_tiles, p, dg.d32,
      dg.pitch, abc_on ? 1 : 0, first ? 1 : 0, d_step, gr.sched + 2, dg.d_err);
}

template <int M>
static void force32_m(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                      int ring_u, int, bool abc_on, bool first, int *d_step, cudaStream_t st) {
  if (gr.force_rows == 4)
    force32_k<M, 4>(gr, lg, dg, p, ring_u, abc_on, first, d_step, st);
  else
    force32_k<M, 2>(gr, lg, dg, p, ring_u, abc_on, first, d_step, st);
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
