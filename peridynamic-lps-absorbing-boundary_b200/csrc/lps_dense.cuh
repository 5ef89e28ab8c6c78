// lps_dense.cuh -- masked dense-grid path: layout and launch interface.
//
// Every instance whose nodes sit exactly on a dx = dy lattice with
// delta = m dx (m in kDenseM) is stored as a padded 2-D grid of cells:
// row = x index, column = y index (so cell order follows the
// preprocessor's node order, x outer / y inner, preprocessor/main.cpp:851),
// column pitch a multiple of 8 cells (128-byte rows of double2), m cells of
// padding on every side plus the round-up to whole tiles.  Empty cells carry
// type 0.  The horizon of a cell is the fixed offset set
// {(a, b) != 0 : a^2 + b^2 <= m^2 + m} -- exactly the nodes the reference's
// search radius delta + dx/2 + 1e-5 (src/main.cpp:352) admits on such a
// lattice -- restricted to existing cells.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "lps_cuda.h"
#include "lps_kernels.cuh"
#include "lps_setup.h"

namespace lps {

constexpr int kTileRows = 16;   // owned cells per tile: 16 rows x 32 columns
constexpr int kTileCols = 32;
constexpr int kDenseM[] = {2, 3, 4, 5, 6, 8};

struct DenseTile {
  int base;   // global cell index of the tile's first owned cell
  int inst;   // instance id
  int full;   // 1: every neighbour of every owned node exists (no masking)
  int pad;
};

struct DenseGroup {
  int m;            // stencil ratio of the tiles in this group
  int tile_begin;   // first tile in the device tile list
  int n_tiles;
};

struct DenseGeo {
  const DenseTile *tiles = nullptr;            // device
  std::vector<DenseGroup> groups;
  std::vector<std::vector<int>> host_cell_of_node;  // per instance: local node -> global cell
  std::vector<int> host_cells;                      // per instance: cell span
  std::vector<int> host_cell_begin;                 // per instance: first cell
  std::vector<std::vector<int>> host_node_of_cell_v;// per instance: local cell -> node or -1
  int host_node_of_cell(int inst, int global_cell) const {
    const int c = global_cell - host_cell_begin[inst];
    if (c < 0 || c >= (int)host_node_of_cell_v[inst].size()) return -1;
    return host_node_of_cell_v[inst][c];
  }
};

bool dense_m_supported(int m);
// The compile-time offset list of stencil ratio m (host copy).
void dense_offsets(int m, std::vector<int> &a, std::vector<int> &b);
// Per-offset FP64 constants of ratio m for lattice spacing dx (= dy) and
// horizon delta, into __constant__ memory.
cudaError_t upload_dense_constants(int m, double dx, double dy, double delta, cudaStream_t st);

int enqueue_dense_step(const DenseGeo &dg, const LaunchGeo &lg, const StepPtrs &p, int *d_step,
                       cudaStream_t st, const Mark *mark);
void launch_theta_dense_init(const DenseGeo &dg, const LaunchGeo &lg, const double2 *u, double *theta,
                             cudaStream_t st);
void launch_diag_dense(const DenseGeo &dg, const LaunchGeo &lg, const double2 *u, const double2 *v,
                       const double2 *a, const double *theta, DiagPartial *partials, DiagRecord *log,
                       int *log_count, int log_capacity, const int *d_step, cudaStream_t st);
cudaError_t dense_prepare_kernels();

}  // namespace lps
