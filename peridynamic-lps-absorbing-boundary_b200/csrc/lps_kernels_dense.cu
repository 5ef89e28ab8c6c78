// lps_kernels_dense.cu -- masked dense-grid stencil kernels, FP64, sm_100a.
//
// One time step is two launches per stencil group:
//   k_theta_dense<M>: predictor (src/main.cpp:725-728) over a tile plus its
//     m-cell halo staged in shared memory, then the dilatation (:736-761) of
//     the owned cells; extra blocks apply G_theta at ABC nodes (:792-812).
//   k_force_dense<M>: the force (:821-874) over a tile plus halo of predicted
//     displacements and theta coefficients, with the corrector (:922-925)
//     fused; extra blocks apply G_u / G_v (:883-916, :933-974).
// The offsets (a, b) are compile-time constants of M, the per-offset FP64
// weights live in __constant__ memory, so each bond is a handful of FP64
// FMAs on shared-memory operands.
#include <cmath>

#include "lps_abc.cuh"
#include "lps_common.cuh"
#include "lps_dense.cuh"

namespace lps {

// ---------------------------------------------------------------------------
// compile-time stencils: {(a, b) != 0 : a^2 + b^2 <= M^2 + M}
__host__ __device__ constexpr int sten_count(int M) {
  int n = 0;
  for (int a = -M; a <= M; a++)
    for (int b = -M; b <= M; b++)
      if ((a != 0 || b != 0) && a * a + b * b <= M * M + M) n++;
  return n;
}

template <int M>
struct Sten {
  static constexpr int N = sten_count(M);
  int a[N], b[N];
};

template <int M>
__host__ __device__ constexpr Sten<M> make_sten() {
  Sten<M> s{};
  int n = 0;
  for (int a = -M; a <= M; a++)
    for (int b = -M; b <= M; b++)
      if ((a != 0 || b != 0) && a * a + b * b <= M * M + M) {
        s.a[n] = a;
        s.b[n] = b;
        n++;
      }
  return s;
}

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
  switch (m) {
    case 2: offsets_of<2>(a, b); break;
    case 3: offsets_of<3>(a, b); break;
    case 4: offsets_of<4>(a, b); break;
    case 5: offsets_of<5>(a, b); break;
    case 6: offsets_of<6>(a, b); break;
    case 8: offsets_of<8>(a, b); break;
    default: a.clear(); b.clear();
  }
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
template <int M>
struct Region {
  static constexpr int RR = kTileRows + 2 * M;   // staged rows
  static constexpr int RC = kTileCols + 2 * M;   // staged columns
  static constexpr int CELLS = RR * RC;
};

template <int M>
constexpr size_t theta_smem() {
  return Region<M>::CELLS * (sizeof(double2) + 1);
}
template <int M>
constexpr size_t force_smem() {
  return Region<M>::CELLS * (sizeof(double2) + 2 * sizeof(double) + 1);
}

// Predictor + dilatation.  Block = one tile (256 threads: 8 warps x 32
// columns, two owned rows per thread).
template <int M>
__global__ void __launch_bounds__(256)
    k_theta_dense(Geo g, Abc ab, const DenseTile *__restrict__ tiles, StepPtrs p, int tile_begin,
                  int n_tiles, int skip_abc) {
  // blocks past the tiles exist only in the first group's launch
  if ((int)blockIdx.x >= n_tiles) {
    const int a = (blockIdx.x - n_tiles) * kAbcWarpsPerBlock + (threadIdx.x >> 5);
    abc_theta_warp(ab, a, p.th_n, p.th_nm1, p.th_np1);
    return;
  }
  using R = Region<M>;
  extern __shared__ __align__(16) unsigned char smem[];
  double2 *su = reinterpret_cast<double2 *>(smem);
  uint8_t *st = reinterpret_cast<uint8_t *>(su + R::CELLS);
  const DenseTile t = tiles[tile_begin + blockIdx.x];
  const InstParams &P = c_inst[t.inst];
  const int pitch = P.pitch;
  const double dt = P.dt, hdt = P.half_dt;
  for (int q = threadIdx.x; q < R::CELLS; q += 256) {
    const int rr = q / R::RC, cc = q - rr * R::RC;
    const int cell = t.base + (rr - M) * pitch + (cc - M);
    const uint8_t ty = g.type[cell];
    double2 up = make_double2(0.0, 0.0);
    if (ty & kExists) {
      double2 u = p.u_n[cell];
      if (ty & kActiveAbc) u = p.s_abc[g.abc_of[cell]];
      const double2 v = p.v_n[cell], a = p.a_n[cell];
      double2 vh;
      vh.x = v.x + hdt * a.x;
      vh.y = v.y + hdt * a.y;
      up.x = u.x + dt * vh.x;
      up.y = u.y + dt * vh.y;
      if (rr >= M && rr < M + kTileRows && cc >= M && cc < M + kTileCols) {
        p.u_np1[cell] = up;
        p.vh[cell] = vh;
        if (ty & kActiveAbc) p.u_n[cell] = u;
      }
    }
    su[q] = up;
    st[q] = ty;
  }
  __syncthreads();
  constexpr Sten<M> S = make_sten<M>();
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
#pragma unroll 1
  for (int k = 0; k < kTileRows / 8; k++) {
    const int r = ty0 + 8 * k;
    const int q0 = (r + M) * R::RC + (tx + M);
    const uint8_t tc = st[q0];
    if (!(tc & kExists)) continue;
    if (skip_abc && (tc & kActiveAbc)) continue;  // the G_theta warps write it
    const int cell = t.base + r * pitch + tx;
    const double2 ui = su[q0];
    double s0 = 0.0, s1 = 0.0;
    if (t.full) {
#pragma unroll
      for (int j = 0; j < Sten<M>::N; j++) {
        const double2 uj = su[q0 + S.a[j] * R::RC + S.b[j]];
        s0 = fma(SC<M>(5, j), uj.x - ui.x, s0);
        s1 = fma(SC<M>(6, j), uj.y - ui.y, s1);
      }
    } else {
#pragma unroll
      for (int j = 0; j < Sten<M>::N; j++) {
        const int q = q0 + S.a[j] * R::RC + S.b[j];
        if (st[q] & kExists) {
          const double2 uj = su[q];
          s0 = fma(SC<M>(5, j), uj.x - ui.x, s0);
          s1 = fma(SC<M>(6, j), uj.y - ui.y, s1);
        }
      }
    }
    const double mi = g.m[cell];
    p.th_np1[cell] = (mi > 0.0) ? (2.0 / mi) * (s0 + s1) : 0.0;
  }
}

// Force + corrector.  Staged per cell: predicted u, A = 2(l-m)/m theta,
// B = 8 mu / m and a validity byte (exists and m > 0, src/main.cpp:852).
template <int M>
__global__ void __launch_bounds__(256)
    k_force_dense(Geo g, Abc ab, const DenseTile *__restrict__ tiles, StepPtrs p, int tile_begin,
                  int n_tiles, int abc_on, int bump_step, int *d_step) {
  // blocks past the tiles exist only in the first group's launch
  if ((int)blockIdx.x >= n_tiles) {
    const int a = (blockIdx.x - n_tiles) * kAbcWarpsPerBlock + (threadIdx.x >> 5);
    abc_uv_warp(ab, a, p);
    return;
  }
  if (bump_step && blockIdx.x == 0 && threadIdx.x == 0) *d_step += 1;
  using R = Region<M>;
  extern __shared__ __align__(16) unsigned char smem[];
  double2 *su = reinterpret_cast<double2 *>(smem);
  double *sA = reinterpret_cast<double *>(su + R::CELLS);
  double *sB = sA + R::CELLS;
  uint8_t *sv = reinterpret_cast<uint8_t *>(sB + R::CELLS);
  const DenseTile t = tiles[tile_begin + blockIdx.x];
  const InstParams &P = c_inst[t.inst];
  const int pitch = P.pitch;
  for (int q = threadIdx.x; q < R::CELLS; q += 256) {
    const int rr = q / R::RC, cc = q - rr * R::RC;
    const int cell = t.base + (rr - M) * pitch + (cc - M);
    const uint8_t ty = g.type[cell];
    double2 u = make_double2(0.0, 0.0);
    double A = 0.0, B = 0.0;
    uint8_t valid = 0;
    if (ty & kExists) {
      const double2 c = g.coef[cell];
      u = p.u_np1[cell];
      if (c.y >= 0.0) {
        A = c.x * p.th_np1[cell];
        B = c.y;
        valid = 1;
      }
    }
    su[q] = u;
    sA[q] = A;
    sB[q] = B;
    sv[q] = valid;
  }
  __syncthreads();
  constexpr Sten<M> S = make_sten<M>();
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
#pragma unroll 1
  for (int k = 0; k < kTileRows / 8; k++) {
    const int r = ty0 + 8 * k;
    const int q0 = (r + M) * R::RC + (tx + M);
    const int cell = t.base + r * pitch + tx;
    const uint8_t tc = g.type[cell];
    if (!(tc & kExists)) continue;
    double2 acc = make_double2(0.0, 0.0);
    if (sv[q0]) {  // m_i > 0 (:827-831)
      const double2 ui = su[q0];
      const double Ai = sA[q0], Bi = sB[q0];
      double F0 = 0.0, F1 = 0.0;
      if (t.full) {
#pragma unroll
        for (int j = 0; j < Sten<M>::N; j++) {
          const int q = q0 + S.a[j] * R::RC + S.b[j];
          const double2 uj = su[q];
          const double e = SC<M>(0, j) * (uj.x - ui.x) + SC<M>(1, j) * (uj.y - ui.y);
          const double tt = (Ai + sA[q]) * SC<M>(2, j) + (Bi + sB[q]) * e;
          F0 = fma(tt, SC<M>(3, j), F0);
          F1 = fma(tt, SC<M>(4, j), F1);
        }
      } else {
#pragma unroll
        for (int j = 0; j < Sten<M>::N; j++) {
          const int q = q0 + S.a[j] * R::RC + S.b[j];
          if (sv[q]) {
            const double2 uj = su[q];
            const double e = SC<M>(0, j) * (uj.x - ui.x) + SC<M>(1, j) * (uj.y - ui.y);
            const double tt = (Ai + sA[q]) * SC<M>(2, j) + (Bi + sB[q]) * e;
            F0 = fma(tt, SC<M>(3, j), F0);
            F1 = fma(tt, SC<M>(4, j), F1);
          }
        }
      }
      acc.x = F0 / P.rho;
      acc.y = F1 / P.rho;
    }
    p.a_np1[cell] = acc;
    if (!(abc_on && (tc & kActiveAbc))) {
      const double2 vh = p.vh[cell];
      p.v_np1[cell] = make_double2(vh.x + P.half_dt * acc.x, vh.y + P.half_dt * acc.y);
    }
  }
}

// ---------------------------------------------------------------------------
// Per-cell kernels with direct global loads (run once per reset or at the
// diagnostics cadence): theta history init (src/main.cpp:664-682) and the
// energy/momentum partial sums (:986-1062).
template <int M>
__device__ __forceinline__ double theta_cell(const Geo &g, const double2 *u, int cell, int pitch) {
  constexpr Sten<M> S = make_sten<M>();
  const double2 ui = u[cell];
  double s0 = 0.0, s1 = 0.0;
#pragma unroll
  for (int j = 0; j < Sten<M>::N; j++) {
    const int nb = cell + S.a[j] * pitch + S.b[j];
    if (g.type[nb] & kExists) {
      const double2 uj = u[nb];
      s0 = fma(SC<M>(5, j), uj.x - ui.x, s0);
      s1 = fma(SC<M>(6, j), uj.y - ui.y, s1);
    }
  }
  const double mi = g.m[cell];
  return (mi > 0.0) ? (2.0 / mi) * (s0 + s1) : 0.0;
}

__global__ void __launch_bounds__(256) k_theta_dense_init(Geo g, const double2 *u, double *theta) {
  const int cell = blockIdx.x * 256 + threadIdx.x;
  if (cell >= g.n_total || !(g.type[cell] & kExists)) return;
  const InstParams &P = c_inst[g.blk_inst[blockIdx.x]];
  double th = 0.0;
  switch (P.stencil) {
    case 2: th = theta_cell<2>(g, u, cell, P.pitch); break;
    case 3: th = theta_cell<3>(g, u, cell, P.pitch); break;
    case 4: th = theta_cell<4>(g, u, cell, P.pitch); break;
    case 5: th = theta_cell<5>(g, u, cell, P.pitch); break;
    case 6: th = theta_cell<6>(g, u, cell, P.pitch); break;
    case 8: th = theta_cell<8>(g, u, cell, P.pitch); break;
  }
  theta[cell] = th;
}

// Deviatoric strain energy density sum of one cell, src/main.cpp:1025-1038.
template <int M>
__device__ __forceinline__ double wdev_cell(const Geo &g, const double2 *u, int cell, int pitch, double th,
                                            double coef) {
  constexpr Sten<M> S = make_sten<M>();
  const double2 ui = u[cell];
  double W = 0.0;
#pragma unroll
  for (int j = 0; j < Sten<M>::N; j++) {
    const int nb = cell + S.a[j] * pitch + S.b[j];
    if (g.type[nb] & kExists) {
      const double2 uj = u[nb];
      const double e = SC<M>(0, j) * (uj.x - ui.x) + SC<M>(1, j) * (uj.y - ui.y);
      const double ed = e - th * SC<M>(2, j) / 2.0;
      const double bdv = SC<M>(3, j) * SC<M>(0, j) + SC<M>(4, j) * SC<M>(1, j);
      W += coef * ed * ed * bdv;
    }
  }
  return W;
}

__global__ void __launch_bounds__(kNodeBlock)
    k_diag_dense(Geo g, Abc ab, const double2 *__restrict__ u, const double2 *__restrict__ v,
                 const double2 *__restrict__ a, const double *__restrict__ theta, DiagPartial *partials,
                 int n_node_blocks) {
  DiagAcc acc;
  acc.init();
  if ((int)blockIdx.x >= n_node_blocks) {
    const int e = (blockIdx.x - n_node_blocks) * kNodeBlock + threadIdx.x;
    if (e < ab.n_abc && ab.active[e]) {
      const int node = ab.node[e];
      const double2 un = u[node], vn = v[node];
      acc.uB = un.x * un.x + un.y * un.y;
      acc.vB = vn.x * vn.x + vn.y * vn.y;
      acc.nact = 1;
    }
    acc.block_reduce_store(partials + blockIdx.x);
    return;
  }
  const int cell = blockIdx.x * kNodeBlock + threadIdx.x;
  if (cell < g.n_total && (g.type[cell] & kExists)) {
    const InstParams &P = c_inst[g.blk_inst[blockIdx.x]];
    const double2 xy = g.xy[cell], un = u[cell], vn = v[cell], an = a[cell];
    const double th = theta[cell];
    const double r = sqrt(xy.x * xy.x + xy.y * xy.y);
    acc.add_maxima(un, vn, an, th, cell);
    if (!(P.out_r > 0.0 && r > P.out_r)) {
      acc.Px = P.rho * vn.x * P.dx * P.dy;
      acc.Py = P.rho * vn.y * P.dx * P.dy;
      const double ek = 0.5 * P.rho * (vn.x * vn.x + vn.y * vn.y) * P.dx * P.dy;
      const double m_i = g.m[cell];
      const double coef = P.c_mu4 / m_i;
      double W = 0.0;
      switch (P.stencil) {
        case 2: W = wdev_cell<2>(g, u, cell, P.pitch, th, coef); break;
        case 3: W = wdev_cell<3>(g, u, cell, P.pitch, th, coef); break;
        case 4: W = wdev_cell<4>(g, u, cell, P.pitch, th, coef); break;
        case 5: W = wdev_cell<5>(g, u, cell, P.pitch, th, coef); break;
        case 6: W = wdev_cell<6>(g, u, cell, P.pitch, th, coef); break;
        case 8: W = wdev_cell<8>(g, u, cell, P.pitch, th, coef); break;
      }
      const double W_i = 0.5 * P.kappa * th * th + W;
      const double ep = W_i * P.dx * P.dy;
      acc.Ek = ek;
      acc.Ep = ep;
      acc.E = ek + ep;
    }
  }
  acc.block_reduce_store(partials + blockIdx.x);
}

// ---------------------------------------------------------------------------
template <int M>
static cudaError_t set_smem_attrs() {
  cudaError_t e = cudaFuncSetAttribute(k_theta_dense<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)theta_smem<M>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_force_dense<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)force_smem<M>());
}

cudaError_t dense_prepare_kernels() {
  cudaError_t e;
  if ((e = set_smem_attrs<2>()) || (e = set_smem_attrs<3>()) || (e = set_smem_attrs<4>()) ||
      (e = set_smem_attrs<5>()) || (e = set_smem_attrs<6>()) || (e = set_smem_attrs<8>()))
    return e;
  return cudaSuccess;
}

template <int M>
static void launch_group(const DenseGroup &gr, bool first, const LaunchGeo &lg, const DenseGeo &dg,
                         const StepPtrs &p, int *d_step, cudaStream_t st, const Mark *mark) {
  const bool gth = lg.abcs_step != -1 && lg.abc.n_abc > 0 && lg.theta_method == 1;
  const int extra = (first && gth) ? lg.n_abc_blocks : 0;
  k_theta_dense<M><<<gr.n_tiles + extra, 256, theta_smem<M>(), st>>>(lg.geo, lg.abc, dg.tiles, p,
                                                                     gr.tile_begin, gr.n_tiles, gth ? 1 : 0);
  if (mark) (*mark)("theta_dense");
}

template <int M>
static void launch_force_group(const DenseGroup &gr, bool first, const LaunchGeo &lg, const DenseGeo &dg,
                               const StepPtrs &p, int *d_step, cudaStream_t st, const Mark *mark) {
  const bool abc_on = lg.abcs_step != -1 && lg.abc.n_abc > 0;
  const int extra = (first && abc_on) ? lg.n_abc_blocks : 0;
  k_force_dense<M><<<gr.n_tiles + extra, 256, force_smem<M>(), st>>>(
      lg.geo, lg.abc, dg.tiles, p, gr.tile_begin, gr.n_tiles, abc_on ? 1 : 0, first ? 1 : 0, d_step);
  if (mark) (*mark)("force_dense");
}

#define LPS_DISPATCH_M(m, FN, ...)          \
  switch (m) {                              \
    case 2: FN<2>(__VA_ARGS__); break;      \
    case 3: FN<3>(__VA_ARGS__); break;      \
    case 4: FN<4>(__VA_ARGS__); break;      \
    case 5: FN<5>(__VA_ARGS__); break;      \
    case 6: FN<6>(__VA_ARGS__); break;      \
    case 8: FN<8>(__VA_ARGS__); break;      \
  }

int enqueue_dense_step(const DenseGeo &dg, const LaunchGeo &lg, const StepPtrs &p, int *d_step,
                       cudaStream_t st, const Mark *mark) {
  int k = 0;
  for (size_t i = 0; i < dg.groups.size(); i++) {
    LPS_DISPATCH_M(dg.groups[i].m, launch_group, dg.groups[i], i == 0, lg, dg, p, d_step, st, mark);
    k++;
  }
  if (lg.abcs_step != -1 && lg.theta_method == 0 && lg.abc.n_abc > 0) {
    launch_theta_idw(lg, p.th_np1, st);
    if (mark) (*mark)("theta_idw");
    k++;
  }
  for (size_t i = 0; i < dg.groups.size(); i++) {
    LPS_DISPATCH_M(dg.groups[i].m, launch_force_group, dg.groups[i], i == 0, lg, dg, p, d_step, st, mark);
    k++;
  }
  return k;
}

void launch_theta_dense_init(const DenseGeo &, const LaunchGeo &lg, const double2 *u, double *theta,
                             cudaStream_t st) {
  k_theta_dense_init<<<lg.n_node_blocks, 256, 0, st>>>(lg.geo, u, theta);
}

void launch_diag_dense(const DenseGeo &, const LaunchGeo &lg, const double2 *u, const double2 *v,
                       const double2 *a, const double *theta, DiagPartial *partials, DiagRecord *log,
                       int *log_count, int log_capacity, const int *d_step, cudaStream_t st) {
  const int abc_blocks = (lg.abc.n_abc + kNodeBlock - 1) / kNodeBlock;
  k_diag_dense<<<lg.n_node_blocks + abc_blocks, kNodeBlock, 0, st>>>(lg.geo, lg.abc, u, v, a, theta, partials,
                                                                      lg.n_node_blocks);
  launch_diag_finish(lg.n_inst, partials, lg.n_node_blocks, log, log_count, log_capacity, d_step, st);
}

}  // namespace lps
