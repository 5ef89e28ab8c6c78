// lps_abc.cuh -- device helpers shared by the CSR and dense kernels: the
// volume-correction factor and the absorbing-boundary operator warps.
#pragma once
#include "lps_common.cuh"

namespace lps {

__device__ __forceinline__ double beta_dev(double xi, const InstParams &P) {
  // src/main.cpp:100-107
  if (xi <= P.beta_lo) return 1.0;
  if (xi <= P.beta_hi) return (P.beta_hi - xi) / P.dx;
  return 0.0;
}

// G_theta at one ABC node per warp, src/main.cpp:795-812.
__device__ __forceinline__ void abc_theta_warp(const Abc &ab, int a, const double *th_n,
                                               const double *th_nm1, double *theta) {
  const int lane = threadIdx.x & 31;
  if (a >= ab.n_abc || !ab.writes[a]) return;
  const int off = ab.cl_off[a], len = ab.cl_len[a];
  double acc = 0.0;
  for (int e = lane; e < len; e += 32) {
    const int k = ab.cl_idx[off + e];
    const double2 w = ab.gth[off + e];
    acc += w.x * th_n[k] + w.y * th_nm1[k];
  }
  acc = warp_sum(acc);
  if (lane == 0) theta[ab.node[a]] = acc;
}

// ABC displacement and velocity at one ABC node per warp,
// src/main.cpp:883-916 and :933-974.  G rows are stored per cloud entry as
// [gx(x^n), gx(y^n), gx(x^{n-1}), gx(y^{n-1}), gy(...) x4].
__device__ __forceinline__ void abc_uv_warp(const Abc &ab, int a, const StepPtrs &p) {
  const int lane = threadIdx.x & 31;
  if (a >= ab.n_abc || !ab.writes[a]) return;
  const InstParams &P = c_inst[ab.inst[a]];
  const int off = ab.cl_off[a], len = ab.cl_len[a];
  double ux = 0.0, uy = 0.0, vx = 0.0, vy = 0.0;
  for (int e = lane; e < len; e += 32) {
    const int k = ab.cl_idx[off + e];
    const double2 un = p.u_n[k], unm1 = p.u_nm1[k];
    const double *gu = ab.gu + (size_t)(off + e) * 8;
    ux += gu[0] * un.x + gu[1] * un.y + gu[2] * unm1.x + gu[3] * unm1.y;
    uy += gu[4] * un.x + gu[5] * un.y + gu[6] * unm1.x + gu[7] * unm1.y;
    if (!P.kinematic) {
      const double2 vn = p.v_n[k], vnm1 = p.v_nm1[k];
      const double *gv = ab.gv + (size_t)(off + e) * 8;
      vx += gv[0] * vn.x + gv[1] * vn.y + gv[2] * vnm1.x + gv[3] * vnm1.y;
      vy += gv[4] * vn.x + gv[5] * vn.y + gv[6] * vnm1.x + gv[7] * vnm1.y;
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
