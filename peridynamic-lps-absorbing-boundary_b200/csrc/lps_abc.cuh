// lps_abc.cuh -- device helpers shared by the CSR and dense kernels: the
// volume-correction factor and the absorbing-boundary operator warps.
//
// Operator layout (packed on the host): the compacted cloud of ABC entry a
// occupies entries [cl_off, cl_off + cl_len); G_u and G_v are stored per
// entry component-major, 8 rows of cl_len doubles starting at 8 * cl_off:
//   rows 0-3: x output <- (x^n, y^n, x^{n-1}, y^{n-1}),  rows 4-7: y output,
// and G_theta as 2 rows (theta^n, theta^{n-1}) starting at 2 * cl_off, so the
// 32 lanes of a warp read 32 consecutive doubles per row.  A warp serves one
// ABC node and issues the loads of up to 64 cloud entries (two per lane)
// before it consumes any of them.
#pragma once
#include "lps_common.cuh"

namespace lps {

__device__ __forceinline__ double beta_dev(double xi, const InstParams &P) {
  // src/main.cpp:100-107
  if (xi <= P.beta_lo) return 1.0;
  if (xi <= P.beta_hi) return (P.beta_hi - xi) / P.dx;
  return 0.0;
}

// FP32-mixed form: the force pass's per-node coefficients (A', B') =
// ((lambda_PD / alpha) q theta, q) with q = m_ref / m_i (coef32.x), alpha =
// 8 mu / m_ref; the dense path measures bond lengths in lattice units, so its
// A' carries a factor dx.  Where m_i <= 0: (0, -1) on the CSR path (the force
// pass skips such neighbours, src/main.cpp:852), (0, 0) on the dense path
// (such a cell has no neighbours, so it is nobody's neighbour).  Written
// wherever theta is written.
__device__ __forceinline__ void write_ab32(float2 *ab32, const float2 *coef32, int node, double th,
                                           const InstParams &P) {
  const float2 co = coef32[node];
  const float l = P.dense ? (float)P.dx : 1.f;
  ab32[node] = co.y > 0.f ? make_float2((float)(th * P.f32_ab) * co.x * l, co.y)
                          : make_float2(0.f, P.dense ? 0.f : -1.f);
}

// The dense path's FP32-mixed form keeps A' and B' as separate planes; B' is
// static, so only A' (with its factor dx) is written wherever theta is.
__device__ __forceinline__ void write_ap32(float *ap32, const float *bp32, int node, double th, const InstParams &P) {
  const float q = bp32[node];
  ap32[node] = q > 0.f ? (float)(th * P.f32_ab) * q * (float)P.dx : 0.f;
}

// G_theta at one ABC node per warp, src/main.cpp:795-812 (and, in the
// FP32-mixed form, the node's force coefficients).
__device__ __forceinline__ void abc_theta_warp(const Abc &ab, int a, const double *__restrict__ th_n,
                                               const double *__restrict__ th_nm1, double *theta,
                                               float2 *ab32 = nullptr, const float2 *coef32 = nullptr) {
  const int lane = threadIdx.x & 31;
  if (a >= ab.n_abc || !ab.writes[a]) return;
  const int off = ab.cl_off[a], len = ab.cl_len[a];
  const double *__restrict__ w0 = ab.gth + 2 * (size_t)off;
  const double *__restrict__ w1 = w0 + len;
  double acc = 0.0;
  for (int e0 = 0; e0 < len; e0 += 64) {
    const int ea = e0 + lane, eb = e0 + 32 + lane;
    const bool va = ea < len, vb = eb < len;
    const int ka = va ? __ldg(ab.cl_idx + off + ea) : 0, kb = vb ? __ldg(ab.cl_idx + off + eb) : 0;
    const double wa0 = va ? __ldg(w0 + ea) : 0.0, wa1 = va ? __ldg(w1 + ea) : 0.0;
    const double wb0 = vb ? __ldg(w0 + eb) : 0.0, wb1 = vb ? __ldg(w1 + eb) : 0.0;
    const double ta0 = va ? th_n[ka] : 0.0, ta1 = va ? th_nm1[ka] : 0.0;
    const double tb0 = vb ? th_n[kb] : 0.0, tb1 = vb ? th_nm1[kb] : 0.0;
    acc += wa0 * ta0 + wa1 * ta1;
    acc += wb0 * tb0 + wb1 * tb1;
  }
  acc = warp_sum(acc);
  if (lane == 0) {
    theta[ab.node[a]] = acc;
    if (ab32) write_ab32(ab32, coef32, ab.node[a], acc, ab.ip[ab.inst[a]]);
  }
}

// One cloud entry's contribution to the x and y outputs of a 2-level operator.
__device__ __forceinline__ void g_entry(const double *__restrict__ g, int len, int e, double2 xn, double2 xm,
                                        double &ox, double &oy) {
  ox += __ldg(g + 0 * len + e) * xn.x + __ldg(g + 1 * len + e) * xn.y + __ldg(g + 2 * len + e) * xm.x +
        __ldg(g + 3 * len + e) * xm.y;
  oy += __ldg(g + 4 * len + e) * xn.x + __ldg(g + 5 * len + e) * xn.y + __ldg(g + 6 * len + e) * xm.x +
        __ldg(g + 7 * len + e) * xm.y;
}

// ABC displacement and velocity at one ABC node per warp,
// src/main.cpp:883-916 and :933-974.
__device__ __forceinline__ void abc_uv_warp(const Abc &ab, int a, const StepPtrs &p) {
  const int lane = threadIdx.x & 31;
  if (a >= ab.n_abc || !ab.writes[a]) return;
  const InstParams &P = ab.ip[ab.inst[a]];
  const int off = ab.cl_off[a], len = ab.cl_len[a];
  const double *__restrict__ gu = ab.gu + 8 * (size_t)off;
  const double *__restrict__ gv = ab.gv + 8 * (size_t)off;
  double ux = 0.0, uy = 0.0, vx = 0.0, vy = 0.0;
  const double2 z = make_double2(0.0, 0.0);
  for (int e0 = 0; e0 < len; e0 += 64) {
    const int ea = e0 + lane, eb = e0 + 32 + lane;
    const bool va = ea < len, vb = eb < len;
    const int ka = va ? __ldg(ab.cl_idx + off + ea) : 0, kb = vb ? __ldg(ab.cl_idx + off + eb) : 0;
    const double2 una = va ? p.u_n[ka] : z, uma = va ? p.u_nm1[ka] : z;
    const double2 unb = vb ? p.u_n[kb] : z, umb = vb ? p.u_nm1[kb] : z;
    if (va) g_entry(gu, len, ea, una, uma, ux, uy);
    if (vb) g_entry(gu, len, eb, unb, umb, ux, uy);
    if (!P.kinematic) {
      const double2 vna = va ? p.v_n[ka] : z, vma = va ? p.v_nm1[ka] : z;
      const double2 vnb = vb ? p.v_n[kb] : z, vmb = vb ? p.v_nm1[kb] : z;
      if (va) g_entry(gv, len, ea, vna, vma, vx, vy);
      if (vb) g_entry(gv, len, eb, vnb, vmb, vx, vy);
    }
  }
  ux = warp_sum(ux);
  uy = warp_sum(uy);
  if (!P.kinematic) {
    vx = warp_sum(vx);
    vy = warp_sum(vy);
  }
  if (lane == 0) {
    const int node = ab.node[a];
    p.s_abc[a] = make_double2(ux, uy);
    if (P.kinematic) {
      // v = (u^{n+1} - u^n) / dt, src/main.cpp:940-943
      const double2 un = p.u_n[node];
      p.v_np1[node] = make_double2((ux - un.x) / P.dt, (uy - un.y) / P.dt);
    } else {
      p.v_np1[node] = make_double2(vx, vy);
    }
  }
}

}  // namespace lps
