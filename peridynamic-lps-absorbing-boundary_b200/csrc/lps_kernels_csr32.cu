// lps_kernels_csr32.cu -- FP32-mixed form of the neighbour-list (ELL) kernels,
// sm_100a.
//
// The route for inputs that are not lattices (arbitrary horizon files,
// prenotch-cut horizons): the same per-bond sums as lps_kernels_csr.cu,
//   dilatation  theta_i = (2 dV / m_i) sum_j beta (xi . eta)          (src/main.cpp:736-761)
//   force       F_i = alpha dV sum_j beta xi_hat [(A'_i + A'_j)|xi| + (B'_i + B'_j) e]  (:821-874)
// with e = xi_hat . eta, B' = m_ref / m, A' = (lambda_PD / alpha) B' theta and
// alpha = 8 mu / m_ref, so no material constant enters the FP32 arithmetic.
// FP32: the bond vector (the FP64 coordinate difference, rounded once), |xi|
// and xi_hat (correctly rounded square root and quotients), beta, the
// displacement difference (from the FP32 copy of the predicted level) and the
// sums, which run in chunks of eight bonds added to the node's total with
// Kahan compensation.  FP64: the state, the Verlet update, theta
// storage, the absorbing-boundary operators (the ABC warps are the FP64
// form's) and the diagnostics.
#include "lps_abc.cuh"
#include "lps_common.cuh"
#include "lps_kernels.cuh"

namespace lps {

namespace {

constexpr int kChunk = 8;  // bonds per FP32 partial sum

// s + x with Kahan's running compensation c (the estimate is s - c).
__device__ __forceinline__ void kahan_add(float &s, float &c, float x) {
  const float y = x - c;
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}

// Volume correction of a bond of length r (src/main.cpp:100-107) in FP32.
__device__ __forceinline__ float beta32(float r, float lo, float hi, float inv_dx) {
  return r <= lo ? 1.f : (r <= hi ? (hi - r) * inv_dx : 0.f);
}

}  // namespace

// Dilatation; ABC blocks (blockIdx >= n_node_blocks) apply the G_theta
// override of :792-812 in FP64 and write the force coefficients beside it.
__global__ void __launch_bounds__(kNodeBlock)
    k_theta_csr32(Geo g, Abc ab, const float2 *__restrict__ u32, double *__restrict__ theta,
                  float2 *__restrict__ ab32, const float2 *__restrict__ coef32, const double *__restrict__ th_n,
                  const double *__restrict__ th_nm1, int n_node_blocks, int g_theta_override) {
  if ((int)blockIdx.x >= n_node_blocks) {
    if (!g_theta_override) return;
    const int a = (blockIdx.x - n_node_blocks) * kAbcWarpsPerBlock + (threadIdx.x >> 5);
    abc_theta_warp(ab, a, th_n, th_nm1, theta, ab32, coef32);
    return;
  }
  const int i = blockIdx.x * kNodeBlock + threadIdx.x;
  if (i >= g.n_total) return;
  const uint8_t t = g.type[i];
  if (!(t & kExists)) return;
  if (g_theta_override && (t & kActiveAbc)) return;  // written by the ABC warps
  const InstParams &P = g.ip[g.blk_inst[blockIdx.x]];
  const float blo = (float)P.beta_lo, bhi = (float)P.beta_hi, inv_dx = (float)(1.0 / P.dx);
  const double2 xi_i = g.xy[i];
  const float2 ui = u32[i];
  const int len = g.len[i];
  float S = 0.f, C = 0.f, part = 0.f;
  for (int s0 = 0; s0 < len; s0 += kChunk) {
    const int s1 = min(len, s0 + kChunk);
    for (int s = s0; s < s1; s++) {
      const int j = g.nbr[(size_t)s * g.n_total + i];
      if (j < 0) continue;
      const double2 xj = g.xy[j];
      const float ex = (float)(xj.x - xi_i.x), ey = (float)(xj.y - xi_i.y);
      const float r = __fsqrt_rn(fmaf(ex, ex, ey * ey));
      const float b = beta32(r, blo, bhi, inv_dx);
      const float2 uj = u32[j];
      const float dot = fmaf(ex, uj.x - ui.x, ey * (uj.y - ui.y));  // xi . eta = |xi| e
      part = fmaf(b, dot, part);
    }
    kahan_add(S, C, part);
    part = 0.f;
  }
  const double mi = g.m[i];
  const double th = (mi > 0.0) ? (2.0 * P.dx * P.dy / mi) * (double)(S - C) : 0.0;
  theta[i] = th;
  write_ab32(ab32, coef32, i, th, P);
}

// Force in FP32 with the corrector (:922-925) in FP64.  ABC blocks run the
// FP64 G_u / G_v warps, as k_force_csr does.
__global__ void __launch_bounds__(kNodeBlock)
    k_force_csr32(Geo g, Abc ab, StepPtrs p, const float2 *__restrict__ u32, const float2 *__restrict__ ab32,
                  int n_node_blocks, int abc_on, int *d_step) {
  if ((int)blockIdx.x >= n_node_blocks) {
    if (!abc_on) return;
    const int a = (blockIdx.x - n_node_blocks) * kAbcWarpsPerBlock + (threadIdx.x >> 5);
    abc_uv_warp(ab, a, p);
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *d_step += 1;
  const int i = blockIdx.x * kNodeBlock + threadIdx.x;
  if (i >= g.n_total) return;
  const uint8_t t = g.type[i];
  if (!(t & kExists)) return;
  const InstParams &P = g.ip[g.blk_inst[blockIdx.x]];
  const float2 abi = ab32[i];
  double2 acc = make_double2(0.0, 0.0);
  if (abi.y > 0.f) {  // m_i > 0 (:827-831)
    const float blo = (float)P.beta_lo, bhi = (float)P.beta_hi, inv_dx = (float)(1.0 / P.dx);
    const double2 xi_i = g.xy[i];
    const float2 ui = u32[i];
    const int len = g.len[i];
    float S0 = 0.f, C0 = 0.f, S1 = 0.f, C1 = 0.f, p0 = 0.f, p1 = 0.f;
    for (int s0 = 0; s0 < len; s0 += kChunk) {
      const int s1 = min(len, s0 + kChunk);
      for (int s = s0; s < s1; s++) {
        const int j = g.nbr[(size_t)s * g.n_total + i];
        if (j < 0) continue;
        const float2 abj = ab32[j];
        if (abj.y < 0.f) continue;  // m_j <= 0 (:852)
        const double2 xj = g.xy[j];
        const float ex = (float)(xj.x - xi_i.x), ey = (float)(xj.y - xi_i.y);
        // correctly rounded square root and quotients: an approximate
        // reciprocal square root biases every bond's stiffness the same way
        // each step, and that error grows with the run (about 1e-5 after
        // 4000 steps of configuration 1)
        const float r = __fsqrt_rn(fmaf(ex, ex, ey * ey));
        const float hx = __fdiv_rn(ex, r), hy = __fdiv_rn(ey, r);
        const float b = beta32(r, blo, bhi, inv_dx);
        const float2 uj = u32[j];
        const float e = fmaf(hx, uj.x - ui.x, hy * (uj.y - ui.y));
        const float T = fmaf(abi.y + abj.y, e, (abi.x + abj.x) * r);
        const float bt = b * T;
        p0 = fmaf(bt, hx, p0);
        p1 = fmaf(bt, hy, p1);
      }
      kahan_add(S0, C0, p0);
      kahan_add(S1, C1, p1);
      p0 = p1 = 0.f;
    }
    const double scale = P.f32_b0 * P.dx * P.dy / P.rho;
    acc.x = (double)(S0 - C0) * scale;
    acc.y = (double)(S1 - C1) * scale;
  }
  p.a_np1[i] = acc;
  if (!(abc_on && (t & kActiveAbc))) {
    const double2 vh = p.vh[i];
    p.v_np1[i] = make_double2(vh.x + P.half_dt * acc.x, vh.y + P.half_dt * acc.y);
  }
}

void launch_theta_csr32(const LaunchGeo &g, const float2 *u32, double *theta, float2 *ab32, const float2 *coef32,
                        const double *th_n, const double *th_nm1, cudaStream_t st) {
  const bool gth = g.abcs_step != -1 && g.theta_method == 1 && g.abc.n_abc > 0;
  const int blocks = g.n_node_blocks + (gth ? g.n_abc_blocks : 0);
  k_theta_csr32<<<blocks, kNodeBlock, 0, st>>>(g.geo, g.abc, u32, theta, ab32, coef32, th_n, th_nm1,
                                                g.n_node_blocks, gth ? 1 : 0);
}

void launch_force_csr32(const LaunchGeo &g, const StepPtrs &p, const float2 *ab32, int *d_step, cudaStream_t st) {
  const bool abc_on = g.abcs_step != -1 && g.abc.n_abc > 0;
  const int blocks = g.n_node_blocks + (abc_on ? g.n_abc_blocks : 0);
  k_force_csr32<<<blocks, kNodeBlock, 0, st>>>(g.geo, g.abc, p, p.u32_np1, ab32, g.n_node_blocks, abc_on ? 1 : 0,
                                                d_step);
}

}  // namespace lps
