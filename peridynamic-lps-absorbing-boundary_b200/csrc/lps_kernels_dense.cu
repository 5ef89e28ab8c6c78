// lps_kernels_dense.cu -- masked dense-grid stencil kernels, FP64, sm_100a.
//
// One time step is two persistent tile kernels on the main stream and the
// absorbing-boundary kernels:
//   k_theta_tma<M>   dilatation (src/main.cpp:736-761) of the predicted
//                    displacements
//   k_force_tma<M>   force (:821-874), corrector (:922-925) and the next
//                    step's predictor (:725-728)
//   k_abc_sell       G_u, G_v (:883-916, :933-974) of the step and G_theta
//                    (:792-812) of the next, on a side stream beside the force
//                    tiles
//   k_abc_predict    the ABC nodes' merge and prediction at the end of the step
// Tile kernels stage a 16 x 32 tile plus its m-cell halo with TMA
// (cp.async.bulk.tensor) into one of two shared-memory buffers while the
// other buffer is being computed; every wait on the transaction barrier is
// bounded and reports a timeout through an error flag.  Each thread owns 2
// adjacent rows of one column and walks the stencil, pairing offset (a, b)
// with (-a, -b), so every staged value it loads feeds several bonds.
#include <cmath>
#include <cstdio>

#include "lps_abc.cuh"
#include "lps_common.cuh"
#include "lps_dense.cuh"
#include "lps_tile.cuh"

namespace lps {

// Per-offset constants, 7 rows of N doubles per supported M:
//   0: xi_hat_x  1: xi_hat_y  2: |xi|  3: g_x = beta dV xi_hat_x
//   4: g_y       5: c_x = beta dV xi_x  6: c_y = beta dV xi_y
constexpr int kStenRows = 7;
__host__ __device__ constexpr int sten_base(int M) {
  int base = 0;
  for (int m : {2, 3, 4, 5, 6, 8}) {
    if (m == M) return base;
    base += kStenRows * sten_count(m);
  }
  return -1;
}
constexpr int kStenDoubles = sten_base(8) + kStenRows * sten_count(8);
__constant__ double c_sten[kStenDoubles];

template <int M>
__device__ __forceinline__ double SC(int row, int j) {
  return c_sten[sten_base(M) + row * Sten<M>::N + j];
}

bool dense_m_supported(int m) {
  for (int x : kDenseM)
    if (x == m) return true;
  return false;
}

template <int M>
static void offsets_of(std::vector<int> &a, std::vector<int> &b) {
  constexpr Sten<M> s = make_sten<M>();
  a.assign(s.a, s.a + Sten<M>::N);
  b.assign(s.b, s.b + Sten<M>::N);
}

void dense_offsets(int m, std::vector<int> &a, std::vector<int> &b) {
  a.clear();
  b.clear();
  LPS_DISPATCH_M(m, offsets_of, a, b);
}

cudaError_t upload_dense_constants(int m, double dx, double dy, double delta, cudaStream_t st) {
  std::vector<int> A, B;
  dense_offsets(m, A, B);
  const int N = (int)A.size();
  std::vector<double> c(kStenRows * N);
  for (int j = 0; j < N; j++) {
    // the reference's bond geometry, src/main.cpp:837-848
    const double xi_x = A[j] * dx, xi_y = B[j] * dy;
    const double xi_norm = std::sqrt(xi_x * xi_x + xi_y * xi_y);
    double beta;
    if (xi_norm <= delta - dx / 2.0) beta = 1.0;
    else if (xi_norm <= delta + dx / 2.0) beta = (delta + dx / 2.0 - xi_norm) / dx;
    else beta = 0.0;
    const double bdv = beta * dx * dy;
    c[0 * N + j] = xi_x / xi_norm;
    c[1 * N + j] = xi_y / xi_norm;
    c[2 * N + j] = xi_norm;
    c[3 * N + j] = bdv * (xi_x / xi_norm);
    c[4 * N + j] = bdv * (xi_y / xi_norm);
    c[5 * N + j] = bdv * xi_x;
    c[6 * N + j] = bdv * xi_y;
  }
  return cudaMemcpyToSymbolAsync(c_sten, c.data(), sizeof(double) * c.size(), sizeof(double) * sten_base(m),
                                 cudaMemcpyHostToDevice, st);
}

// ---------------------------------------------------------------------------
// Tile compute.  A force thread owns cells (r0, c) and (r0 + 1, c), a
// dilatation thread K rows of column c; for every pair of opposite
// offsets (a, b) / (-a, -b) it reads the two staged neighbours of each cell --
// the row-(r0+1) reads of one offset are the row-r0 reads of the next, so
// most of them come from registers.
//   dilatation pair:  c_j . (u(+) - u(-))                    (src/main.cpp:757)
//   force pair:       g_j [ (A+ - A-) |xi| + (B_i + B+) e+ - (B_i + B-) e- ]
// with e+ = (u(+) - u_i) . xi_hat, e- = (u_i - u(-)) . xi_hat, A = 2(l-m)/m
// theta, B = 8 mu / m (:857-869).  Masked tiles (near the domain edge) use the
// same pairs with absent neighbours zeroed: u = A = B = 0 there, and the
// owned node's own terms are weighted by which side is present.
// The dilatation thread owns K adjacent rows of one column (the force thread
// two), so a staged value it loads feeds the pairs of up to K cells; each
// cell's sums are the same whatever the rows per thread.  K is 4 or 2, picked
// per batch (the autotuner's choice; 4 by default); a CTA has th_threads(K)
// threads.
constexpr int th_threads(int K) { return kTileRows * kTileCols / K; }

template <int M, bool FULL, int K>
__device__ __forceinline__ void theta_tile(const double2 *__restrict__ su, const uint8_t *__restrict__ sty, int r0,
                                           int c, double th[K]) {
  using R = Region<M>;
  double s0[K], s1[K];
#pragma unroll
  for (int k = 0; k < K; k++) s0[k] = s1[k] = 0.0;
  for_each_pair<M>(
      [&](auto ac, auto bc) {
        constexpr int a = decltype(ac)::value, b = decltype(bc)::value;
        constexpr int j = sten_index(M, a, b);
        const double cx = SC<M>(5, j), cy = SC<M>(6, j);
#pragma unroll
        for (int k = 0; k < K; k++) {
          const int r = r0 + k;
          const double2 up = su[QI<M>(r + a, c + b)], um = su[QI<M>(r - a, c - b)];
          double dx = up.x - um.x, dy = up.y - um.y;
          if (!FULL) {
            // absent neighbours hold u = 0; restore the -u_i of the present side
            const double mp = (sty[(r + a + M) * R::RT + c + b + M] & kExists) ? 1.0 : 0.0;
            const double mm = (sty[(r - a + M) * R::RT + c - b + M] & kExists) ? 1.0 : 0.0;
            const double2 ui = su[QI<M>(r, c)];
            dx = fma(mm - mp, ui.x, dx);
            dy = fma(mm - mp, ui.y, dy);
          }
          s0[k] = fma(cx, dx, s0[k]);
          s1[k] = fma(cy, dy, s1[k]);
        }
      },
      [](auto) {});
#pragma unroll
  for (int k = 0; k < K; k++) th[k] = s0[k] + s1[k];
}

template <int M, bool FULL>
__device__ __forceinline__ void force_tile(const double2 *__restrict__ su, const double2 *__restrict__ sab, int r0,
                                           int c, double2 F[2]) {
  double2 ui[2], ab_i[2];
  double F0[2] = {0.0, 0.0}, F1[2] = {0.0, 0.0};
#pragma unroll
  for (int k = 0; k < 2; k++) {
    ui[k] = su[QI<M>(r0 + k, c)];
    ab_i[k] = sab[QI<M>(r0 + k, c)];
  }
  for_each_pair<M>(
      [&](auto ac, auto bc) {
        constexpr int a = decltype(ac)::value, b = decltype(bc)::value;
        constexpr int j = sten_index(M, a, b);
        const double hx = SC<M>(0, j), hy = SC<M>(1, j), L = SC<M>(2, j);
        const double gx = SC<M>(3, j), gy = SC<M>(4, j);
#pragma unroll
        for (int k = 0; k < 2; k++) {
          const int r = r0 + k;
          const int qp = QI<M>(r + a, c + b), qm = QI<M>(r - a, c - b);
          const double2 up = su[qp], um = su[qm], abp = sab[qp], abm = sab[qm];
          const double e1 = hx * (up.x - ui[k].x) + hy * (up.y - ui[k].y);
          const double e2 = hx * (ui[k].x - um.x) + hy * (ui[k].y - um.y);
          double T, wp, wm;
          if (FULL) {
            T = (abp.x - abm.x) * L;
            wp = ab_i[k].y + abp.y;
            wm = ab_i[k].y + abm.y;
          } else {
            // a valid neighbour has B > 0; an absent one has A = B = 0
            const double mp = abp.y > 0.0 ? 1.0 : 0.0, mm = abm.y > 0.0 ? 1.0 : 0.0;
            T = fma(mp - mm, ab_i[k].x, abp.x - abm.x) * L;
            wp = fma(mp, ab_i[k].y, abp.y);
            wm = fma(mm, ab_i[k].y, abm.y);
          }
          T = fma(wp, e1, T);
          T = fma(-wm, e2, T);
          F0[k] = fma(T, gx, F0[k]);
          F1[k] = fma(T, gy, F1[k]);
        }
      },
      [](auto) {});
#pragma unroll
  for (int k = 0; k < 2; k++) F[k] = make_double2(F0[k], F1[k]);
}

// ---------------------------------------------------------------------------
// Predicted displacements -> dilatation, persistent over tiles.
template <int M, int K>
__global__ void __launch_bounds__(th_threads(K), K == 4 ? 4 : 3)
    k_theta_tma(const __grid_constant__ CUtensorMap map_u, const __grid_constant__ CUtensorMap map_type, Geo g,
                const DenseTile *__restrict__ tiles, int tile_begin, int n_tiles, StepPtrs p, int pitch,
                int skip_abc, int *sched, int *err) {
  using R = Region<M>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * R::THETA_STAGE);
  // next tiles of the two stages, beside the barriers: static shared memory
  // would shift the dynamic buffer off its 128-byte alignment
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
    const double2 *su = reinterpret_cast<const double2 *>(smem + stage * R::THETA_STAGE);
    const uint8_t *sty = reinterpret_cast<const uint8_t *>(smem + stage * R::THETA_STAGE + R::T_TY);
    const int r0 = K * warp;
    // m_i of the owned cells, fetched while the copy lands
    const size_t cell0 = (size_t)(t.row + M + r0) * pitch + t.col + M + lane;
    double mi[K];
#pragma unroll
    for (int k = 0; k < K; k++) mi[k] = g.m[cell0 + (size_t)k * pitch];
    const bool landed = mbar_wait_bounded(&bar[stage], (it >> 1) & 1, err);
    if (__syncthreads_or(!landed)) {  // a copy timed out: leave the loop together
      failed = true;
      break;
    }
    double th[K];
    if (t.flags & kTileFull)
      theta_tile<M, true, K>(su, sty, r0, lane, th);
    else
      theta_tile<M, false, K>(su, sty, r0, lane, th);
#pragma unroll
    for (int k = 0; k < K; k++) {
      const uint8_t ty = sty[(r0 + k + M) * R::RT + lane + M];
      if (!(ty & kExists)) continue;
      if (skip_abc && (ty & kActiveAbc)) continue;  // the G_theta kernel writes it
      p.th_np1[cell0 + (size_t)k * pitch] = (mi[k] > 0.0) ? (2.0 / mi[k]) * th[k] : 0.0;
    }
    fence_proxy_async_smem();
    __syncthreads();  // the stage is refilled at the start of the next-but-one iteration
  }
  if (failed && tid == 0) drain_stages(bar, it, s_tile[(it & 1) ^ 1] < n_tiles, err);
  if (tid == 0) sched_finish(sched);
}

// ---------------------------------------------------------------------------
// Force + corrector + next predictor, persistent over tiles.  After the copy
// lands, (theta, coef) become (A, B) = (2(l-m)/m theta, 8 mu/m) in the coef
// slot; absent neighbours and m <= 0 (src/main.cpp:852) get A = B = 0.
template <int M>
__global__ void __launch_bounds__(kTileThreads, 2)
    k_force_tma(const __grid_constant__ CUtensorMap map_u, const __grid_constant__ CUtensorMap map_th,
                const __grid_constant__ CUtensorMap map_coef, const __grid_constant__ CUtensorMap map_type, Geo g,
                const DenseTile *__restrict__ tiles, int tile_begin, int n_tiles, StepPtrs p, int pitch, int abc_on,
                int bump_step, int *d_step, int *sched, int *err) {
  using R = Region<M>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * R::FORCE_STAGE);
  // next tiles of the two stages, beside the barriers: static shared memory
  // would shift the dynamic buffer off its 128-byte alignment
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
    const InstParams &P = g.ip[t.inst];
    unsigned char *base = smem + stage * R::FORCE_STAGE;
    double2 *su = reinterpret_cast<double2 *>(base);
    const double *sth = reinterpret_cast<const double *>(base + R::F_TH);
    double2 *sab = reinterpret_cast<double2 *>(base + R::F_CO);
    const uint8_t *sty = reinterpret_cast<const uint8_t *>(base + R::F_TY);
    const int r0 = 2 * warp;
    // corrector inputs of the owned cells, fetched while the copy lands
    const size_t cell0 = (size_t)(t.row + M + r0) * pitch + t.col + M + lane;
    const double2 vh0 = p.vh[cell0], vh1 = p.vh[cell0 + pitch];
    const bool landed = mbar_wait_bounded(&bar[stage], (it >> 1) & 1, err);
    if (__syncthreads_or(!landed)) {  // a copy timed out: leave the loop together
      failed = true;
      break;
    }
    for (int q = tid; q < R::CELLS; q += kTileThreads) {
      const int rr = q / R::RC, cc = q - rr * R::RC;
      const double2 co = sab[q];
      const bool valid = (sty[rr * R::RT + cc] & kExists) && co.y >= 0.0;
      sab[q] = valid ? make_double2(co.x * sth[q], co.y) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double2 F[2];
    if (t.flags & kTileFull)
      force_tile<M, true>(su, sab, r0, lane, F);
    else
      force_tile<M, false>(su, sab, r0, lane, F);
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const uint8_t ty = sty[(r0 + k + M) * R::RT + lane + M];
      if (!(ty & kExists)) continue;
      const size_t cell = cell0 + (size_t)k * pitch;
      const bool valid = sab[QI<M>(r0 + k, lane)].y > 0.0;  // m_i > 0 (:827-831)
      const double2 acc = valid ? make_double2(F[k].x / P.rho, F[k].y / P.rho) : make_double2(0.0, 0.0);
      if (p.full || (ty & (kKeepState | kActiveAbc))) p.a_np1[cell] = acc;
      if (abc_on && (ty & kActiveAbc)) continue;  // G_v writes v; the next theta kernel predicts u
      // corrector (:924) then the next predictor (:727) from the same values
      const double2 vh = k == 0 ? vh0 : vh1;
      double2 v, vh2, un;
      v.x = vh.x + P.half_dt * acc.x;
      v.y = vh.y + P.half_dt * acc.y;
      vh2.x = v.x + P.half_dt * acc.x;
      vh2.y = v.y + P.half_dt * acc.y;
      const double2 u = su[QI<M>(r0 + k, lane)];
      un.x = u.x + P.dt * vh2.x;
      un.y = u.y + P.dt * vh2.y;
      if (p.full || (ty & kKeepState)) p.v_np1[cell] = v;
      p.vh[cell] = vh2;
      p.u_np2[cell] = un;
    }
    fence_proxy_async_smem();
    __syncthreads();
  }
  if (failed && tid == 0) drain_stages(bar, it, s_tile[(it & 1) ^ 1] < n_tiles, err);
  if (tid == 0) sched_finish(sched);
}

// ---------------------------------------------------------------------------
// Absorbing-boundary kernels of the dense path.
// The absorbing boundary of a dense step over the sliced-ELL operators: one
// CTA per slice of 32 writing entries (one per lane), kSellWarps warps that
// split the slice's cloud positions; a warp's operator reads are 256-byte
// rows of one contiguous run, so the operator stream reaches DRAM in long
// sequential pieces.  Per entry: G_u and G_v of this step (src/main.cpp:
// 883-916, :933-974) from u^n, u^{n-1}, v^n, v^{n-1}, and, one step ahead,
// G_theta (:792-812): theta^{n+2} from theta^{n+1} (p.th_np1) and theta^n
// (p.th_n) into the ring slot that theta^{n-1} (p.th_nm1) frees.  Warps add
// their partial sums through shared memory.
// Measured (7-instance batch, standalone): 4 warps 68.3 us without and
// 60.7 us with the cloud index loaded one position ahead; 8 warps 63.6 us;
// 4 or 8 warps at 46 registers 67.1 / 60.5 us.
constexpr int kSellWarps = 4;

__global__ void __launch_bounds__(32 * kSellWarps) k_abc_sell(Abc ab, StepPtrs p, int do_uv, int do_theta) {
  constexpr int W = kSellWarps;
  __shared__ double red[W - 1][5][32];
  const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
  const SellSlice sl = ab.slices[blockIdx.x];
  const int a = ab.sell_a[blockIdx.x * 32 + lane];
  const int inst = a >= 0 ? ab.inst[a] : 0;
  const bool kin = ab.ip[inst].kinematic != 0;
  const double *__restrict__ g = ab.sell_g + sl.goff + lane;
  const int *__restrict__ ix = ab.sell_idx + sl.ioff + lane;
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // ux, uy, vx, vy, theta
  // warp q takes positions q, q + W, ...: which warp sums a position does
  // not depend on the slice's length, so an entry's result does not depend on
  // the entries it shares a slice with (past its own length it adds zeros)
  int k_next = q < sl.len ? __ldg(ix + 32 * q) : 0;
#pragma unroll 2
  for (int e = q; e < sl.len; e += W) {
    const int k = k_next;  // this position's cloud index, loaded one position ahead
    if (e + W < sl.len) k_next = __ldg(ix + 32 * (e + W));
    const double *__restrict__ ge = g + (size_t)e * 18 * 32;
    if (do_uv) {
      const double2 un = p.u_n[k], um = p.u_nm1[k];
      s[0] += __ldcs(ge + 0 * 32) * un.x + __ldcs(ge + 1 * 32) * un.y + __ldcs(ge + 2 * 32) * um.x +
              __ldcs(ge + 3 * 32) * um.y;
      s[1] += __ldcs(ge + 4 * 32) * un.x + __ldcs(ge + 5 * 32) * un.y + __ldcs(ge + 6 * 32) * um.x +
              __ldcs(ge + 7 * 32) * um.y;
      if (!kin) {
        const double2 vn = p.v_n[k], vm = p.v_nm1[k];
        s[2] += __ldcs(ge + 8 * 32) * vn.x + __ldcs(ge + 9 * 32) * vn.y + __ldcs(ge + 10 * 32) * vm.x +
                __ldcs(ge + 11 * 32) * vm.y;
        s[3] += __ldcs(ge + 12 * 32) * vn.x + __ldcs(ge + 13 * 32) * vn.y + __ldcs(ge + 14 * 32) * vm.x +
                __ldcs(ge + 15 * 32) * vm.y;
      }
    }
    if (do_theta) s[4] += __ldcs(ge + 16 * 32) * p.th_np1[k] + __ldcs(ge + 17 * 32) * p.th_n[k];
  }
  if (q > 0)
#pragma unroll
    for (int j = 0; j < 5; j++) red[q - 1][j][lane] = s[j];
  __syncthreads();
  if (q > 0 || a < 0) return;
#pragma unroll
  for (int w = 0; w < W - 1; w++)
#pragma unroll
    for (int j = 0; j < 5; j++) s[j] += red[w][j][lane];
  const int node = ab.node[a];
  if (do_uv) {
    p.s_abc[a] = make_double2(s[0], s[1]);
    if (kin) {
      // v = (u^{n+1} - u^n) / dt with this node's u^n, src/main.cpp:940-943
      const double2 un = p.u_n[node];
      const double dt = ab.ip[inst].dt;
      p.v_np1[node] = make_double2((s[0] - un.x) / dt, (s[1] - un.y) / dt);
    } else {
      p.v_np1[node] = make_double2(s[2], s[3]);
    }
  }
  if (do_theta) const_cast<double *>(p.th_nm1)[node] = s[4];
}

static void launch_abc_sell(const Abc &ab, const StepPtrs &p, int do_uv, int do_theta, cudaStream_t st) {
  k_abc_sell<<<ab.n_slices, 32 * kSellWarps, 0, st>>>(ab, p, do_uv, do_theta);
}

// End of a dense step at the absorbing boundary, after the force tiles and
// G_u/G_v: this step's G_u result u^{n+1} goes into the displacement ring,
// and u^{n+2} is predicted there from it, the G_v velocity and the new
// acceleration (src/main.cpp:725-728), so the next step's tiles stage every
// cell straight from the rings.
__global__ void __launch_bounds__(256) k_abc_predict(Abc ab, StepPtrs p) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= ab.n_abc || !ab.writes[a]) return;
  const int node = ab.node[a];
  const InstParams &P = ab.ip[ab.inst[a]];
  const double2 u = p.s_abc[a], v = p.v_np1[node], acc = p.a_np1[node];
  double2 vh, up;
  vh.x = v.x + P.half_dt * acc.x;
  vh.y = v.y + P.half_dt * acc.y;
  up.x = u.x + P.dt * vh.x;
  up.y = u.y + P.dt * vh.y;
  p.u_np1[node] = u;
  p.u_np2[node] = up;
  p.vh[node] = vh;
  if (p.u32_np2) p.u32_np2[node] = make_float2((float)up.x, (float)up.y);
}

// ---------------------------------------------------------------------------
// Per-cell kernels with direct global loads (run once per reset or at the
// diagnostics cadence): theta history init (src/main.cpp:664-682) and the
// energy/momentum partial sums (:986-1062).
template <int M>
__device__ __forceinline__ double theta_cell(const Geo &g, const double2 *u, size_t cell, int pitch) {
  const double2 ui = u[cell];
  double s0 = 0.0, s1 = 0.0;
  static_for<0, Sten<M>::N>([&](auto jc) {
    constexpr int j = decltype(jc)::value;
    constexpr int a = make_sten<M>().a[j], b = make_sten<M>().b[j];
    const size_t nb = (size_t)((ptrdiff_t)cell + (ptrdiff_t)a * pitch + b);
    if (g.type[nb] & kExists) {
      const double2 uj = u[nb];
      s0 = fma(SC<M>(5, j), uj.x - ui.x, s0);
      s1 = fma(SC<M>(6, j), uj.y - ui.y, s1);
    }
  });
  const double mi = g.m[cell];
  return (mi > 0.0) ? (2.0 / mi) * (s0 + s1) : 0.0;
}

template <int M>
__device__ __forceinline__ void theta_cell_into(const Geo &g, const double2 *u, size_t cell, int pitch, double *out) {
  *out = theta_cell<M>(g, u, cell, pitch);
}

__global__ void __launch_bounds__(256) k_theta_dense_init(Geo g, const double2 *u, double *theta) {
  const size_t cell = (size_t)blockIdx.x * 256 + threadIdx.x;
  if (cell >= (size_t)g.n_total || !(g.type[cell] & kExists)) return;
  const InstParams &P = g.ip[g.blk_inst[blockIdx.x]];
  double th = 0.0;
  LPS_DISPATCH_M(P.stencil, theta_cell_into, g, u, cell, P.pitch, &th);
  theta[cell] = th;
}

// Diagnostics of the dense path (src/main.cpp:986-1062), one CTA per tile:
// the tile's displacements and node types are staged with TMA (as for the
// dilatation), and each thread sums the deviatoric strain energy of its two
// cells over the opposite-offset pairs -- for offset (a, b) the bond
// extension e+ = xi_hat . (u(+) - u_i), for (-a, -b) it is
// e- = xi_hat . (u_i - u(-)), each with e^d = e - theta_i |xi| / 2 (:1027-1038)
// -- then kinetic energy, momentum and the maxima from its own cells.  Each
// tile leaves one partial; k_diag_abc adds the boundary norms (:1050-1062).
template <int M>
__global__ void __launch_bounds__(kTileThreads, 2)
    k_diag_tiles(const __grid_constant__ CUtensorMap map_u, const __grid_constant__ CUtensorMap map_type, Geo g,
                 const DenseTile *__restrict__ tiles, int tile_begin, const double2 *__restrict__ v,
                 const double2 *__restrict__ acc_n, const double *__restrict__ theta, DiagPartial *partials,
                 int pitch, int *err) {
  using R = Region<M>;
  static_assert(R::THETA_STAGE + 64 <= 48 * 1024, "one stage fits the default shared-memory limit");
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + R::THETA_STAGE);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const DenseTile t = tiles[tile_begin + blockIdx.x];
  DiagAcc acc;
  acc.init();
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
    mbar_expect_tx(bar, R::THETA_TX);
    tma_load_2d(smem, &map_u, 2 * t.col, t.row, bar);
    tma_load_2d(smem + R::T_TY, &map_type, t.col, t.row, bar);
  }
  const InstParams &P = g.ip[t.inst];
  const int r0 = 2 * warp;
  const size_t cell0 = (size_t)(t.row + M + r0) * pitch + t.col + M + lane;
  // the owned cells' other fields, fetched while the copy lands
  double2 vv[2], aa[2], xy[2];
  double th[2], mi[2];
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const size_t cell = cell0 + (size_t)k * pitch;
    vv[k] = v[cell];
    aa[k] = acc_n[cell];
    xy[k] = g.xy[cell];
    th[k] = theta[cell];
    mi[k] = g.m[cell];
  }
  __syncthreads();  // barrier initialised before any thread waits on it
  const bool ok = mbar_wait_bounded(bar, 0, err);
  const double2 *su = reinterpret_cast<const double2 *>(smem);
  const uint8_t *sty = smem + R::T_TY;
  if (ok) {
    const bool full = t.flags & kTileFull;
    const double2 ui[2] = {su[QI<M>(r0, lane)], su[QI<M>(r0 + 1, lane)]};
    double w[2] = {0.0, 0.0};
    for_each_pair<M>(
        [&](auto ac, auto bc) {
          constexpr int a = decltype(ac)::value, b = decltype(bc)::value;
          constexpr int j = sten_index(M, a, b);
          const double hx = SC<M>(0, j), hy = SC<M>(1, j), L = SC<M>(2, j);
          const double bdv = SC<M>(3, j) * SC<M>(0, j) + SC<M>(4, j) * SC<M>(1, j);  // beta dV
#pragma unroll
          for (int k = 0; k < 2; k++) {
            const int r = r0 + k;
            const double2 up = su[QI<M>(r + a, lane + b)], um = su[QI<M>(r - a, lane - b)];
            const double hl = th[k] * L / 2.0;
            const double e1 = hx * (up.x - ui[k].x) + hy * (up.y - ui[k].y) - hl;
            const double e2 = hx * (ui[k].x - um.x) + hy * (ui[k].y - um.y) - hl;
            if (full) {
              w[k] += bdv * (e1 * e1 + e2 * e2);
            } else {
              if (sty[(r + a + M) * R::RT + lane + b + M] & kExists) w[k] += bdv * (e1 * e1);
              if (sty[(r - a + M) * R::RT + lane - b + M] & kExists) w[k] += bdv * (e2 * e2);
            }
          }
        },
        [](auto) {});
#pragma unroll
    for (int k = 0; k < 2; k++) {
      if (!(sty[(r0 + k + M) * R::RT + lane + M] & kExists)) continue;
      const size_t cell = cell0 + (size_t)k * pitch;
      acc.add_maxima(ui[k], vv[k], aa[k], th[k], (int)cell);
      const double rr = sqrt(xy[k].x * xy[k].x + xy[k].y * xy[k].y);
      if (P.out_r > 0.0 && rr > P.out_r) continue;  // energy only in the near field (:1010)
      acc.Px += P.rho * vv[k].x * P.dx * P.dy;
      acc.Py += P.rho * vv[k].y * P.dx * P.dy;
      const double ek = 0.5 * P.rho * (vv[k].x * vv[k].x + vv[k].y * vv[k].y) * P.dx * P.dy;
      const double W_i = 0.5 * P.kappa * th[k] * th[k] + (P.c_mu4 / mi[k]) * w[k];
      const double ep = W_i * P.dx * P.dy;
      acc.Ek += ek;
      acc.Ep += ep;
      acc.E += ek + ep;
    }
  }
  // a copy that timed out may still land: wait it out before the CTA leaves
  if (!ok && tid == 0) mbar_wait_bounded(bar, 0, err);
  acc.block_reduce_store(partials + tile_begin + blockIdx.x);
}

// Boundary norms at the active ABC nodes (src/main.cpp:1050-1062).
__global__ void __launch_bounds__(kNodeBlock)
    k_diag_abc(Abc ab, const double2 *__restrict__ u, const double2 *__restrict__ v, DiagPartial *partials) {
  DiagAcc acc;
  acc.init();
  const int e = blockIdx.x * kNodeBlock + threadIdx.x;
  if (e < ab.n_abc && ab.active[e]) {
    const int node = ab.node[e];
    const double2 un = u[node], vn = v[node];
    acc.uB = un.x * un.x + un.y * un.y;
    acc.vB = vn.x * vn.x + vn.y * vn.y;
    acc.nact = 1;
  }
  acc.block_reduce_store(partials + blockIdx.x);
}

// u^1 = u^0 + dt (v^0 + dt/2 a^0) with a^0 = 0, and vh = v^0, src/main.cpp:727.
__global__ void __launch_bounds__(256) k_dense_reset_predict(Geo g, const double2 *u0, const double2 *v0,
                                                              double2 *u1, float2 *u32_1, double2 *vh) {
  const size_t cell = (size_t)blockIdx.x * 256 + threadIdx.x;
  if (cell >= (size_t)g.n_total) return;
  if (!(g.type[cell] & kExists)) {
    u1[cell] = make_double2(0.0, 0.0);
    if (u32_1) u32_1[cell] = make_float2(0.f, 0.f);
    vh[cell] = make_double2(0.0, 0.0);
    return;
  }
  const InstParams &P = g.ip[g.blk_inst[blockIdx.x]];
  const double2 u = u0[cell], v = v0[cell];
  double2 h, up;
  h.x = v.x + P.half_dt * 0.0;
  h.y = v.y + P.half_dt * 0.0;
  up.x = u.x + P.dt * h.x;
  up.y = u.y + P.dt * h.y;
  u1[cell] = up;
  if (u32_1) u32_1[cell] = make_float2((float)up.x, (float)up.y);
  vh[cell] = h;
}

// ---------------------------------------------------------------------------
// host side
template <int M>
static cudaError_t prepare_m(DenseGroup &gr, int n_sm) {
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_theta_tma<M, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Region<M>::THETA_SMEM)) ||
      (e = cudaFuncSetAttribute(k_theta_tma<M, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Region<M>::THETA_SMEM)))
    return e;
  if ((e = cudaFuncSetAttribute(k_force_tma<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Region<M>::FORCE_SMEM)))
    return e;
  if ((e = cudaFuncSetAttribute(k_theta_tma<M, 4>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared)) ||
      (e = cudaFuncSetAttribute(k_theta_tma<M, 2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared)) ||
      (e = cudaFuncSetAttribute(k_force_tma<M>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared)))
    return e;
  int bt = 0, bt2 = 0, bf = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, k_theta_tma<M, 4>, th_threads(4),
                                                         Region<M>::THETA_SMEM)) ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt2, k_theta_tma<M, 2>, th_threads(2),
                                                         Region<M>::THETA_SMEM)))
    return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf, k_force_tma<M>, kTileThreads, Region<M>::FORCE_SMEM)))
    return e;
  bt = std::max(bt, 1);
  bf = std::max(bf, 1);
  gr.theta_rows = 4;
  gr.grid_theta = std::min(gr.n_tiles, bt * n_sm);
  gr.grid_force = std::min(gr.n_tiles, bf * n_sm);
  gr.max_theta_ctas = bt;
  gr.max_theta_ctas2 = std::max(bt2, 1);
  gr.max_force_ctas = bf;
  gr.force_rows = 2;
  gr.max_force_ctas4 = 0;  // the FP64 force pass has the two-row form only
  return cudaSuccess;
}

template <int M>
static void prepare_dispatch(DenseGroup &gr, int n_sm, cudaError_t *e) {
  *e = prepare_m<M>(gr, n_sm);
}

void dense_set_ctas(DenseGeo &dg, int theta_rows, int theta_ctas, int force_ctas, int force_rows) {
  int dev = 0, n_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  for (auto &gr : dg.groups) {
    gr.theta_rows = theta_rows == 2 ? 2 : 4;
    gr.force_rows = (force_rows == 4 && gr.max_force_ctas4 > 0) ? 4 : 2;
    const int t = std::max(1, std::min(theta_ctas, gr.theta_rows == 2 ? gr.max_theta_ctas2 : gr.max_theta_ctas));
    const int f = std::max(1, std::min(force_ctas, gr.force_rows == 4 ? gr.max_force_ctas4 : gr.max_force_ctas));
    gr.grid_theta = std::min(gr.n_tiles, t * n_sm);
    gr.grid_force = std::min(gr.n_tiles, f * n_sm);
  }
}

cudaError_t dense_prepare(DenseGeo &dg) {
  int dev = 0, n_sm = 0, least = 0, greatest = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  dg.tile_priority = greatest;  // tile CTAs are dispatched ahead of the ABC kernel's blocks
  for (auto &gr : dg.groups) {
    cudaError_t e = cudaErrorInvalidValue;
    if (dg.fp32)
      e = dense32_prepare_group(gr, n_sm);
    else
      LPS_DISPATCH_M(gr.m, prepare_dispatch, gr, n_sm, &e);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

bool encode(CUtensorMap *map, CUtensorMapDataType dt, size_t elem, const void *base, uint64_t inner,
            uint64_t rows, uint32_t box_inner, uint32_t box_rows) {
  auto fn = get_encode();
  if (!fn) return false;
  const cuuint64_t dims[2] = {inner, rows};
  const cuuint64_t strides[1] = {inner * elem};
  const cuuint32_t box[2] = {box_inner, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, dt, 2, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int M>
void encode_m(DenseGroup &g, int pitch, int rows, double2 *const *U, double *const *TH, const double2 *coef,
              const uint8_t *type, float2 *const *U32, const float *ap32, const float *bp32, bool *ok) {
  using R = Region<M>;
  bool good = true;
  if (U32) {
    // FP32-mixed planes; the coefficient boxes are RC rounded up to 16 bytes
    const uint32_t rca = (R::RC + 3) / 4 * 4;
    for (int r = 0; r < 2; r++)
      good &= encode(&g.maps.u32[r], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, U32[r], 2ull * pitch, rows, 2 * R::RC,
                     R::RR);
    good &= encode(&g.maps.ap32, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ap32, pitch, rows, rca, R::RR);
    good &= encode(&g.maps.bp32, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, bp32, pitch, rows, rca, R::RR);
  }
  for (int r = 0; r < kUring; r++)
    good &= encode(&g.maps.u[r], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, U[r], 2ull * pitch, rows, 2 * R::RC, R::RR);
  for (int r = 0; r < 3; r++)
    good &= encode(&g.maps.th[r], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, TH[r], pitch, rows, R::RC, R::RR);
  good &= encode(&g.maps.coef, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, coef, 2ull * pitch, rows, 2 * R::RC, R::RR);
  good &= encode(&g.maps.type, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, type, pitch, rows, R::RT, R::RR);
  *ok = good;
}
}  // namespace

int dense_encode_maps(DenseGroup &g, int pitch, int total_rows, double2 *const *U, double *const *TH,
                      const double2 *coef, const uint8_t *type, float2 *const *U32, const float *ap32,
                      const float *bp32, std::string &err) {
  bool ok = false;
  LPS_DISPATCH_M(g.m, encode_m, g, pitch, total_rows, U, TH, coef, type, U32, ap32, bp32, &ok);
  if (!ok) {
    err = "cuTensorMapEncodeTiled failed for the dense layout";
    return LPS_ERR_CUDA;
  }
  return LPS_OK;
}

template <int M, int K>
static void launch_theta_k(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                           int ring_u, bool skip_abc, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(gr.grid_theta);
  cfg.blockDim = dim3(th_threads(K));
  cfg.dynamicSmemBytes = Region<M>::THETA_SMEM;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributePriority;
  attr[0].val.priority = dg.tile_priority;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_theta_tma<M, K>, gr.maps.u[ring_u], gr.maps.type, lg.geo, dg.tiles, gr.tile_begin,
                     gr.n_tiles, p, dg.pitch, skip_abc ? 1 : 0, gr.sched, dg.d_err);
}

template <int M>
static void launch_theta_group(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                               int ring_u, bool skip_abc, cudaStream_t st) {
  if (gr.theta_rows == 2)
    launch_theta_k<M, 2>(gr, lg, dg, p, ring_u, skip_abc, st);
  else
    launch_theta_k<M, 4>(gr, lg, dg, p, ring_u, skip_abc, st);
}

template <int M>
static void launch_force_group(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                               int ring_u, int ring_th, bool abc_on, bool first, int *d_step, cudaStream_t st) {
  k_force_tma<M><<<gr.grid_force, kTileThreads, Region<M>::FORCE_SMEM, st>>>(
      gr.maps.u[ring_u], gr.maps.th[ring_th], gr.maps.coef, gr.maps.type, lg.geo, dg.tiles, gr.tile_begin,
      gr.n_tiles, p, dg.pitch, abc_on ? 1 : 0, first ? 1 : 0, d_step, gr.sched + 2, dg.d_err);
}

// ring_u: index of u^{n+1} (the predicted level) in the 4-deep ring;
// p.th_np1 is theta^{n+1}, whose ring index is ring_u' = (n+1) % 3.
int enqueue_dense_step(const DenseGeo &dg, const LaunchGeo &lg, const StepPtrs &p, int *d_step,
                       cudaStream_t st, const Mark *mark, int ring_u) {
  int k = 0;
  const bool abc = lg.abcs_step != -1 && lg.abc.n_abc > 0;
  const bool gth = abc && lg.theta_method == 1;
  const int rth = p.th_ring;
  // With a timing mark the absorbing-boundary kernels run on the main stream
  // (serialised), so each kernel's device time can be read between events.
  const bool fork = mark == nullptr;
  cudaStream_t side = fork ? dg.side : st;
  // The absorbing boundary is one kernel after the dilatation
  // tiles: G_u/G_v of this step and G_theta of the next (theta^{n+2} at ABC
  // nodes from theta^{n+1}, theta^n, into the ring slot theta^{n-1} frees;
  // the reset computes the first one).  It runs on the side stream beside the
  // force tiles; the step joins it at its end, before the ABC prediction that
  // the next step's tiles read.
  for (const auto &gr : dg.groups) {
    if (dg.fp32)
      launch_theta32_group(gr, lg, dg, p, ring_u, gth, st);
    else
      LPS_DISPATCH_M(gr.m, launch_theta_group, gr, lg, dg, p, ring_u, gth, st);
    k++;
  }
  if (mark) (*mark)("theta_tiles");
  if (abc && lg.theta_method == 0) {
    launch_theta_idw(lg, p.th_np1, st, nullptr, nullptr, dg.fp32 ? dg.d32.ap32 : nullptr, dg.d32.bp32);
    if (mark) (*mark)("theta_idw");
    k++;
  }
  const bool pipe = abc && lg.abc.n_slices > 0;
  if (pipe) {
    if (fork) {
      cudaEventRecord(dg.ev_fork[0], st);
      cudaStreamWaitEvent(side, dg.ev_fork[0], 0);
    }
    launch_abc_sell(lg.abc, p, 1, gth ? 1 : 0, side);
    if (mark) (*mark)("abc_sell");
    k++;
    if (fork) cudaEventRecord(dg.ev_join[1], side);
  }
  // pass 2: force tiles
  bool first = true;
  for (const auto &gr : dg.groups) {
    if (dg.fp32)
      launch_force32_group(gr, lg, dg, p, ring_u, rth, abc, first, d_step, st);
    else
      LPS_DISPATCH_M(gr.m, launch_force_group, gr, lg, dg, p, ring_u, rth, abc, first, d_step, st);
    first = false;
    k++;
  }
  if (mark) (*mark)("force_tiles");
  if (abc) {
    if (fork && pipe) cudaStreamWaitEvent(st, dg.ev_join[1], 0);
    k_abc_predict<<<(lg.abc.n_abc + 255) / 256, 256, 0, st>>>(lg.abc, p);
    if (mark) (*mark)("abc_predict");
    k++;
  }
  return k;
}

void launch_dense_reset_predict(const LaunchGeo &lg, const double2 *u0, const double2 *v0, double2 *u1,
                                float2 *u32_1, double2 *vh, cudaStream_t st) {
  k_dense_reset_predict<<<lg.n_node_blocks, 256, 0, st>>>(lg.geo, u0, v0, u1, u32_1, vh);
}

void launch_abc_theta_dense(const DenseGeo &dg, const LaunchGeo &lg, const double *th_n, const double *th_nm1,
                            double *th_np1, cudaStream_t st) {
  if (lg.abc.n_slices == 0) return;
  StepPtrs p = {};
  p.th_np1 = const_cast<double *>(th_n);  // the kernel's "newer" level
  p.th_n = th_nm1;
  p.th_nm1 = th_np1;                       // output slot
  launch_abc_sell(lg.abc, p, 0, 1, st);
}

void launch_theta_dense_init(const DenseGeo &, const LaunchGeo &lg, const double2 *u, double *theta,
                             cudaStream_t st) {
  k_theta_dense_init<<<lg.n_node_blocks, 256, 0, st>>>(lg.geo, u, theta);
}

template <int M>
static void diag_group(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, int ring_u, const double2 *v,
                       const double2 *a, const double *theta, DiagPartial *partials, cudaStream_t st) {
  k_diag_tiles<M><<<gr.n_tiles, kTileThreads, Region<M>::THETA_STAGE + 64, st>>>(
      gr.maps.u[ring_u], gr.maps.type, lg.geo, dg.tiles, gr.tile_begin, v, a, theta, partials, dg.pitch, dg.d_err);
}

void launch_diag_dense(const DenseGeo &dg, const LaunchGeo &lg, int ring_u, const double2 *u, const double2 *v,
                       const double2 *a, const double *theta, DiagPartial *partials, DiagRecord *log,
                       int *log_count, int log_capacity, const int *d_step, cudaStream_t st) {
  int n_tiles = 0;
  for (const auto &gr : dg.groups) {
    LPS_DISPATCH_M(gr.m, diag_group, gr, lg, dg, ring_u, v, a, theta, partials, st);
    n_tiles = std::max(n_tiles, gr.tile_begin + gr.n_tiles);
  }
  const int abc_blocks = (lg.abc.n_abc + kNodeBlock - 1) / kNodeBlock;
  if (abc_blocks > 0) k_diag_abc<<<abc_blocks, kNodeBlock, 0, st>>>(lg.abc, u, v, partials + n_tiles);
  launch_diag_finish_tiles(lg.geo.ip, lg.n_inst, partials, n_tiles, log, log_count, log_capacity, d_step, st);
}

}  // namespace lps
