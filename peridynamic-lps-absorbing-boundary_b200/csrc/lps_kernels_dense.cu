// lps_kernels_dense.cu -- masked dense-grid stencil path (sm_100a).
#include "lps_common.cuh"
#include "lps_dense.cuh"

namespace lps {

int DenseGeo::host_node_of_cell(int inst, int global_cell) const { return -1; }

bool dense_supported(const lps_problem *, int, const std::vector<InstanceSetup> &, const lps_options &) {
  return false;
}

int build_dense(DenseGeo &, LaunchGeo &, const lps_problem *, int, const std::vector<InstanceSetup> &,
                const lps_options &, std::vector<InstParams> &, std::vector<int> &, std::vector<int> &,
                std::vector<int> &, std::vector<int> &, int &, int &, std::string &err, DevAlloc) {
  err = "dense path not built";
  return LPS_ERR_UNSUPPORTED;
}

int enqueue_dense_step(const DenseGeo &, const LaunchGeo &, const StepPtrs &, int *, cudaStream_t, const Mark *) { return 0; }
void launch_theta_dense_init(const DenseGeo &, const LaunchGeo &, const double2 *, double *, cudaStream_t) {}
void launch_diag_dense(const DenseGeo &, const LaunchGeo &, const double2 *, const double2 *, const double2 *,
                       const double *, DiagPartial *, DiagRecord *, int *, int, const int *, cudaStream_t) {}

}  // namespace lps
