// lps_kernels.cuh -- launch helpers of the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>

#include <functional>

#include "lps_device.cuh"

namespace lps {

// Called after each kernel launch with the kernel's name (per-kernel timing).
using Mark = std::function<void(const char *)>;

// Step geometry shared by every launch of a handle.
struct LaunchGeo {
  Geo geo;
  Abc abc;
  int n_node_blocks;   // blocks covering geo.n_total nodes
  int n_abc_blocks;    // blocks covering abc.n_abc (kAbcWarpsPerBlock each)
  int n_inst;
  int theta_method, abcs_step;
};

// CSR path, FP64: one time step is predictor | theta (+G_theta) | [IDW] |
// force + corrector (+G_u, G_v).
void launch_predict_csr(const LaunchGeo &g, const StepPtrs &p, cudaStream_t st);
void launch_theta_csr(const LaunchGeo &g, const double2 *u, double *theta, const double *th_n,
                      const double *th_nm1, bool abc_override, cudaStream_t st);
void launch_theta_idw(const LaunchGeo &g, double *theta, cudaStream_t st, float2 *ab32 = nullptr,
                      const float2 *coef32 = nullptr, float *ap32 = nullptr, const float *bp32 = nullptr);
void launch_force_csr(const LaunchGeo &g, const StepPtrs &p, int *d_step, cudaStream_t st);

// CSR path, FP32-mixed form (lps_kernels_csr32.cu): the predictor above also
// writes the FP32 copy p.u32_np1; dilatation and force run their bond
// arithmetic in FP32 from it, with the per-node force coefficients ab32
// ((lambda_PD / alpha) q theta, q) written beside theta.
void launch_theta_csr32(const LaunchGeo &g, const float2 *u32, double *theta, float2 *ab32, const float2 *coef32,
                        const double *th_n, const double *th_nm1, cudaStream_t st);
void launch_force_csr32(const LaunchGeo &g, const StepPtrs &p, const float2 *ab32, int *d_step, cudaStream_t st);

// Diagnostics: merge the pending ABC displacements into u, then the
// per-block partial sums and one record per instance.
void launch_merge_abc(const LaunchGeo &g, double2 *u, const double2 *s_abc, cudaStream_t st);
void launch_diag_csr(const LaunchGeo &g, const double2 *u, const double2 *v, const double2 *a,
                     const double *theta, DiagPartial *partials, DiagRecord *log, int *log_count,
                     int log_capacity, const int *d_step, cudaStream_t st);

}  // namespace lps
