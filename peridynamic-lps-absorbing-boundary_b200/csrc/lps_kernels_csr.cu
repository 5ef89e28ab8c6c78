// lps_kernels_csr.cu -- neighbour-list (ELL) kernels, FP64, sm_100a.
//
// These kernels take any horizon the host search produced (arbitrary node
// sets, prenotch-cut horizons) and follow the reference's per-bond arithmetic
// (src/main.cpp:736-761 and :821-874) term by term.  The dense-grid kernels
// (lps_kernels_dense.cu) are the fast path for lattice inputs; this path is
// the general one and the fallback.
#include <cstdio>

#include "lps_abc.cuh"
#include "lps_common.cuh"
#include "lps_kernels.cuh"

namespace lps {

// ---------------------------------------------------------------------------
// Predictor, src/main.cpp:725-728, split as u + dt * vh with
// vh = v + dt/2 a (the corrector's first half, :924).  Active ABC nodes first
// take the displacement the previous step's G_u produced (:883-916).
__global__ void __launch_bounds__(kNodeBlock) k_predict_csr(Geo g, StepPtrs p) {
  const int i = blockIdx.x * kNodeBlock + threadIdx.x;
  if (i >= g.n_total) return;
  const uint8_t t = g.type[i];
  if (!(t & kExists)) return;
  const InstParams &P = g.ip[g.blk_inst[blockIdx.x]];
  double2 u = p.u_n[i];
  if (t & kActiveAbc) {
    u = p.s_abc[g.abc_of[i]];
    p.u_n[i] = u;
  }
  const double2 v = p.v_n[i], a = p.a_n[i];
  double2 vh, up;
  vh.x = v.x + P.half_dt * a.x;
  vh.y = v.y + P.half_dt * a.y;
  up.x = u.x + P.dt * vh.x;
  up.y = u.y + P.dt * vh.y;
  p.vh[i] = vh;
  p.u_np1[i] = up;
  if (p.u32_np1) p.u32_np1[i] = make_float2((float)up.x, (float)up.y);  // FP32-mixed form
}

// Dilatation, src/main.cpp:736-761; ABC blocks (blockIdx >= n_node_blocks)
// apply the G_theta override of :792-812 to the same output.
__global__ void __launch_bounds__(kNodeBlock)
    k_theta_csr(Geo g, Abc ab, const double2 *__restrict__ u, double *__restrict__ theta,
                const double *__restrict__ th_n, const double *__restrict__ th_nm1,
                int n_node_blocks, int g_theta_override) {
  if ((int)blockIdx.x >= n_node_blocks) {
    if (!g_theta_override) return;
    const int a = (blockIdx.x - n_node_blocks) * kAbcWarpsPerBlock + (threadIdx.x >> 5);
    abc_theta_warp(ab, a, th_n, th_nm1, theta);
    return;
  }
  const int i = blockIdx.x * kNodeBlock + threadIdx.x;
  if (i >= g.n_total) return;
  const uint8_t t = g.type[i];
  if (!(t & kExists)) return;
  if (g_theta_override && (t & kActiveAbc)) return;  // written by the ABC warps
  const InstParams &P = g.ip[g.blk_inst[blockIdx.x]];
  const double2 xi_i = g.xy[i], ui = u[i];
  const int len = g.len[i];
  double theta_sum = 0.0;
  for (int s = 0; s < len; s++) {
    const int j = g.nbr[(size_t)s * g.n_total + i];
    if (j < 0) continue;
    const double2 xj = g.xy[j], uj = u[j];
    const double xi_x = xj.x - xi_i.x, xi_y = xj.y - xi_i.y;
    const double xi_norm = sqrt(xi_x * xi_x + xi_y * xi_y);
    const double eta_x = uj.x - ui.x, eta_y = uj.y - ui.y;
    const double e = (eta_x * xi_x + eta_y * xi_y) / xi_norm;
    const double b = beta_dev(xi_norm, P);
    theta_sum += xi_norm * e * b * P.dx * P.dy;  // omega = 1 (:112-114)
  }
  const double mi = g.m[i];
  theta[i] = (mi > 0.0) ? (2.0 / mi) * theta_sum : 0.0;
}

// Inverse-distance-weighted theta at ABC nodes, src/main.cpp:765-790.  The
// neighbour lists and weights w = 1/(|r| + 1e-30) are built on the host in the
// reference's horizon order.  Runs after the dilatation pass (needs current
// theta); in the FP32-mixed form it also writes the nodes' force coefficients:
// (A', B') pairs on the neighbour-list path (ab32), the A' plane on the dense
// path (ap32, from the static B' plane bp32).
__global__ void __launch_bounds__(kNodeBlock)
    k_theta_idw(Abc ab, double *theta, float2 *ab32, const float2 *coef32, float *ap32, const float *bp32) {
  const int a = blockIdx.x * kAbcWarpsPerBlock + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (a >= ab.n_abc || !ab.writes[a]) return;
  const int off = ab.idw_off[a], len = ab.idw_len[a];
  double ta = 0.0, ws = 0.0;
  for (int e = lane; e < len; e += 32) {
    const double w = ab.idw_w[off + e];
    ta += w * theta[ab.idw_idx[off + e]];
    ws += w;
  }
  ta = warp_sum(ta);
  ws = warp_sum(ws);
  // every lane has read its neighbours before lane 0 writes (warp_sum syncs)
  if (lane == 0 && ws > 0.0) {
    theta[ab.node[a]] = ta / ws;
    if (ab32) write_ab32(ab32, coef32, ab.node[a], ta / ws, ab.ip[ab.inst[a]]);
    if (ap32) write_ap32(ap32, bp32, ab.node[a], ta / ws, ab.ip[ab.inst[a]]);
  }
}

// Force, src/main.cpp:821-874, with the corrector (:922-925) fused in.  ABC
// blocks run G_u / G_v; G_u writes to s_abc (merged by the next predictor) so
// that no thread of this launch sees a changed u^{n+1}.
__global__ void __launch_bounds__(kNodeBlock)
    k_force_csr(Geo g, Abc ab, StepPtrs p, const double *__restrict__ theta, int n_node_blocks,
                int abc_on, int *d_step) {
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
  const double m_i = g.m[i];
  double2 acc = make_double2(0.0, 0.0);
  if (m_i > 0.0) {
    const double2 xi_i = g.xy[i], ui = p.u_np1[i], ci = g.coef[i];
    const double th_i = theta[i];
    const int len = g.len[i];
    double F0 = 0.0, F1 = 0.0;
    for (int s = 0; s < len; s++) {
      const int j = g.nbr[(size_t)s * g.n_total + i];
      if (j < 0) continue;
      const double2 cj = g.coef[j];
      if (cj.y < 0.0) continue;  // m_j <= 0 (:852)
      const double2 xj = g.xy[j], uj = p.u_np1[j];
      const double xi_x = xj.x - xi_i.x, xi_y = xj.y - xi_i.y;
      const double xi_norm = sqrt(xi_x * xi_x + xi_y * xi_y);
      const double eta_x = uj.x - ui.x, eta_y = uj.y - ui.y;
      const double e = (eta_x * xi_x + eta_y * xi_y) / xi_norm;
      const double b = beta_dev(xi_norm, P);
      const double t_i = ci.x * th_i * xi_norm + ci.y * e;
      const double t_j = cj.x * theta[j] * xi_norm + cj.y * e;
      const double scale = (t_i + t_j) * b * P.dx * P.dy;
      F0 += scale * xi_x / xi_norm;
      F1 += scale * xi_y / xi_norm;
    }
    acc.x = F0 / P.rho;
    acc.y = F1 / P.rho;
  }
  p.a_np1[i] = acc;
  if (!(abc_on && (t & kActiveAbc))) {
    const double2 vh = p.vh[i];
    p.v_np1[i] = make_double2(vh.x + P.half_dt * acc.x, vh.y + P.half_dt * acc.y);
  }
}

// ---------------------------------------------------------------------------
__global__ void k_merge_abc(Abc ab, double2 *u, const double2 *s_abc) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= ab.n_abc || !ab.writes[a]) return;
  u[ab.node[a]] = s_abc[a];
}

// Diagnostics partial sums, src/main.cpp:986-1062: node blocks sum energy,
// momentum and maxima; ABC blocks sum the boundary norms of :1050-1062.
__global__ void __launch_bounds__(kNodeBlock)
    k_diag_csr(Geo g, Abc ab, const double2 *__restrict__ u, const double2 *__restrict__ v,
               const double2 *__restrict__ a, const double *__restrict__ theta,
               DiagPartial *partials, int n_node_blocks) {
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
  const int i = blockIdx.x * kNodeBlock + threadIdx.x;
  if (i < g.n_total && (g.type[i] & kExists)) {
    const InstParams &P = g.ip[g.blk_inst[blockIdx.x]];
    const int local = i - P.node_begin;
    const double2 xy = g.xy[i], un = u[i], vn = v[i], an = a[i];
    const double th = theta[i];
    const double r = sqrt(xy.x * xy.x + xy.y * xy.y);
    acc.add_maxima(un, vn, an, th, local);
    if (!(P.out_r > 0.0 && r > P.out_r)) {
      acc.Px = P.rho * vn.x * P.dx * P.dy;
      acc.Py = P.rho * vn.y * P.dx * P.dy;
      const double ek = 0.5 * P.rho * (vn.x * vn.x + vn.y * vn.y) * P.dx * P.dy;
      const double m_i = g.m[i];
      double W_i = 0.5 * P.kappa * th * th;
      const int len = g.len[i];
      for (int s = 0; s < len; s++) {
        const int j = g.nbr[(size_t)s * g.n_total + i];
        if (j < 0) continue;
        const double2 xj = g.xy[j], uj = u[j];
        const double xi_x = xj.x - xy.x, xi_y = xj.y - xy.y;
        const double xi_norm = sqrt(xi_x * xi_x + xi_y * xi_y);
        const double e = ((uj.x - un.x) * xi_x + (uj.y - un.y) * xi_y) / xi_norm;
        const double ed = e - th * xi_norm / 2.0;
        const double b = beta_dev(xi_norm, P);
        W_i += (P.c_mu4 / m_i) * ed * ed * b * P.dx * P.dy;
      }
      const double ep = W_i * P.dx * P.dy;
      acc.Ek = ek;
      acc.Ep = ep;
      acc.E = ek + ep;
    }
  }
  acc.block_reduce_store(partials + blockIdx.x);
}

// ---------------------------------------------------------------------------
void launch_predict_csr(const LaunchGeo &g, const StepPtrs &p, cudaStream_t st) {
  k_predict_csr<<<g.n_node_blocks, kNodeBlock, 0, st>>>(g.geo, p);
}

void launch_theta_csr(const LaunchGeo &g, const double2 *u, double *theta, const double *th_n,
                      const double *th_nm1, bool abc_override, cudaStream_t st) {
  const bool gth = abc_override && g.abcs_step != -1 && g.theta_method == 1 && g.abc.n_abc > 0;
  const int blocks = g.n_node_blocks + (gth ? g.n_abc_blocks : 0);
  k_theta_csr<<<blocks, kNodeBlock, 0, st>>>(g.geo, g.abc, u, theta, th_n, th_nm1, g.n_node_blocks,
                                              gth ? 1 : 0);
}

void launch_theta_idw(const LaunchGeo &g, double *theta, cudaStream_t st, float2 *ab32, const float2 *coef32,
                      float *ap32, const float *bp32) {
  if (g.abc.n_abc == 0) return;
  k_theta_idw<<<g.n_abc_blocks, kNodeBlock, 0, st>>>(g.abc, theta, ab32, coef32, ap32, bp32);
}

void launch_force_csr(const LaunchGeo &g, const StepPtrs &p, int *d_step, cudaStream_t st) {
  const bool abc_on = g.abcs_step != -1 && g.abc.n_abc > 0;
  const int blocks = g.n_node_blocks + (abc_on ? g.n_abc_blocks : 0);
  k_force_csr<<<blocks, kNodeBlock, 0, st>>>(g.geo, g.abc, p, p.th_np1, g.n_node_blocks,
                                              abc_on ? 1 : 0, d_step);
}

void launch_merge_abc(const LaunchGeo &g, double2 *u, const double2 *s_abc, cudaStream_t st) {
  if (g.abc.n_abc == 0 || g.abcs_step == -1) return;
  k_merge_abc<<<(g.abc.n_abc + 255) / 256, 256, 0, st>>>(g.abc, u, s_abc);
}

void launch_diag_csr(const LaunchGeo &g, const double2 *u, const double2 *v, const double2 *a,
                     const double *theta, DiagPartial *partials, DiagRecord *log, int *log_count,
                     int log_capacity, const int *d_step, cudaStream_t st) {
  const int abc_blocks = (g.abc.n_abc + kNodeBlock - 1) / kNodeBlock;
  k_diag_csr<<<g.n_node_blocks + abc_blocks, kNodeBlock, 0, st>>>(g.geo, g.abc, u, v, a, theta,
                                                                   partials, g.n_node_blocks);
  launch_diag_finish(g.geo.ip, g.n_inst, partials, g.n_node_blocks, log, log_count, log_capacity, d_step, st);
}

}  // namespace lps
