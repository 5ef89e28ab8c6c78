// lps_dense.cuh -- masked dense-grid path: layout and launch interface.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "lps_cuda.h"
#include "lps_kernels.cuh"
#include "lps_setup.h"

namespace lps {

// Host mirror of the dense layout (device pointers live in LaunchGeo).
struct DenseGeo {
  std::vector<std::vector<int>> host_cell_of_node;  // per instance: local node -> global cell
  std::vector<int> host_cells;                      // per instance: cell span (padded grid)
  std::vector<std::vector<int>> host_node_of_cell_v;// per instance: local cell -> node or -1
  int host_node_of_cell(int inst, int global_cell) const;
};

using DevAlloc = std::function<cudaError_t(void **, size_t)>;

// True when every instance's nodes sit exactly on a lattice with distinct
// cells and the stencil fits the kernels.
bool dense_supported(const lps_problem *probs, int n, const std::vector<InstanceSetup> &setup,
                     const lps_options &o);

int build_dense(DenseGeo &dg, LaunchGeo &lg, const lps_problem *probs, int n,
                const std::vector<InstanceSetup> &setup, const lps_options &o,
                std::vector<InstParams> &params, std::vector<int> &node_begin,
                std::vector<int> &node_count, std::vector<int> &abc_begin,
                std::vector<int> &abc_count, int &n_total, int &n_abc_total, std::string &err,
                DevAlloc alloc);

int enqueue_dense_step(const DenseGeo &dg, const LaunchGeo &lg, const StepPtrs &p, int *d_step,
                       cudaStream_t st, const Mark *mark);
void launch_theta_dense_init(const DenseGeo &dg, const LaunchGeo &lg, const double2 *u, double *theta,
                             cudaStream_t st);
void launch_diag_dense(const DenseGeo &dg, const LaunchGeo &lg, const double2 *u, const double2 *v,
                       const double2 *a, const double *theta, DiagPartial *partials, DiagRecord *log,
                       int *log_count, int log_capacity, const int *d_step, cudaStream_t st);

}  // namespace lps
