// lps_dense.cuh -- masked dense-grid path: layout and launch interface.
//
// Every instance whose nodes sit exactly on a dx = dy lattice with
// delta = m dx (m in kDenseM) is stored as a padded 2-D grid of cells:
// row = x index, column = y index (cell order follows the preprocessor's
// node order, x outer / y inner, preprocessor/main.cpp:851), m cells of
// padding on every side plus the round-up to whole tiles.  All instances of a
// batch share one column pitch (a multiple of 32 cells), so each state buffer
// is one 2-D tensor [rows][pitch] that one TMA descriptor covers; instance k
// owns a band of rows starting at a multiple of 8.  Empty cells carry type 0.
// The horizon of a cell is the fixed offset set
// {(a, b) != 0 : a^2 + b^2 <= m^2 + m} -- exactly the nodes the reference's
// search radius delta + dx/2 + 1e-5 (src/main.cpp:352) admits on such a
// lattice -- restricted to existing cells.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "lps_cuda.h"
#include "lps_kernels.cuh"
#include "lps_setup.h"

namespace lps {

constexpr int kTileRows = 16;   // owned cells per tile: 16 rows x 32 columns
constexpr int kTileCols = 32;
constexpr int kCellsPerThread = 2;                                // adjacent rows
constexpr int kTileThreads = kTileRows * kTileCols / kCellsPerThread;  // 256
constexpr int kDenseM[] = {2, 3, 4, 5, 6, 8};
constexpr int kUring = 4;       // displacement ring depth of the dense path

// tile flags
constexpr int kTileFull = 1;    // every neighbour of every owned node exists
constexpr int kTileDeep32 = 2;  // full, and B' = m_ref / m is 1.0f at every owned node and neighbour

// FP32-mixed form: per-cell buffers of the dense kernels.
struct Dense32 {
  float *ap32;            // force coefficient A' = dx q (lambda_PD / alpha) theta, written with theta; 0 at absent cells
  const float *bp32;      // force coefficient B' = q = m_ref / m_i (static); 0 at absent cells and where m_i <= 0
  const float2 *w32;      // W_i = sum over present offsets of beta (a, b)
  const float4 *ka32;     // Ka_i = sum over absent offsets of beta xi_hat xi_hat^T: (xx, xy, yy, 0)
};

struct DenseTile {
  int row;    // global row of the staged region's first row
  int col;    // column of the staged region's first column
  int inst;   // instance id
  int flags;
};

// TMA descriptors of one stencil ratio (box sizes depend on m).
struct DenseMaps {
  CUtensorMap u[kUring];  // displacement ring, double2 viewed as 2 x f64
  CUtensorMap th[3];      // theta ring
  CUtensorMap coef;       // (2(l-m)/m_i, 8 mu/m_i)
  CUtensorMap type;       // u8 node type
  CUtensorMap u32[2];     // FP32-mixed form: FP32 predicted displacements, by step parity
  CUtensorMap ap32, bp32; // FP32-mixed form: force coefficient planes A', B' (one float per cell)
};

struct DenseGroup {
  int m;            // stencil ratio of the tiles in this group
  int tile_begin;   // first tile in the device tile list
  int n_tiles;
  int grid_theta;   // persistent grid sizes
  int grid_force;
  int theta_rows;   // rows of a dilatation thread: 4 or 2
  int force_rows;   // rows of a force thread: 2, or 4 (FP32-mixed form)
  int max_theta_ctas, max_force_ctas;  // resident CTAs per SM at full occupancy
  int max_theta_ctas2;                 // the same for the two-row dilatation kernel
  int max_force_ctas4;                 // the same for the four-row FP32-mixed force kernel
  int *sched;       // device tile-scheduler counters (theta: [0..1], force: [2..3])
  DenseMaps maps;
};

struct DenseGeo {
  const DenseTile *tiles = nullptr;            // device
  std::vector<DenseGroup> groups;
  int pitch = 0;
  int total_rows = 0;
  int tile_priority = 0;                       // launch priority of the tile kernels
  bool fp32 = false;                           // FP32-mixed tile kernels
  Dense32 d32 = {};                            // their per-cell buffers
  cudaStream_t side = nullptr;                 // forked stream for the ABC kernels
  cudaEvent_t ev_fork[2] = {nullptr, nullptr}, ev_join[2] = {nullptr, nullptr};
  int *d_err = nullptr;                        // device wait-timeout flag
  int *sched = nullptr;                        // tile-scheduler counters, 4 per group
  int n_sched = 0;
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
// Encodes the TMA descriptors of group g over the given buffers (U32, ap32
// and bp32 only in the FP32-mixed form, else null).
int dense_encode_maps(DenseGroup &g, int pitch, int total_rows, double2 *const *U, double *const *TH,
                      const double2 *coef, const uint8_t *type, float2 *const *U32, const float *ap32,
                      const float *bp32, std::string &err);
// FP32-mixed form, host side: W_i and Ka_i of the existing cells in
// [first, first + count) of an m-stencil grid, and whether a tile whose first
// owned cell is first_owned is deep (kTileDeep32).
void dense32_static(int m, const std::vector<uint8_t> &type, int pitch, long first, long count,
                    std::vector<float2> &w32, std::vector<float4> &ka32);
bool dense32_tile_deep(int m, const std::vector<uint8_t> &type, const std::vector<float2> &coef32, int pitch,
                       long first_owned);
// Sets shared-memory limits and the persistent grid sizes of each group.
cudaError_t dense_prepare(DenseGeo &dg);
// Persistent grids of every group at the given rows per thread and resident
// CTAs per SM (each clamped to 1..the group's occupancy limit); force_rows 4
// only in the FP32-mixed form.
void dense_set_ctas(DenseGeo &dg, int theta_rows, int theta_ctas, int force_ctas, int force_rows = 2);

// FP32-mixed tile kernels (lps_kernels_dense32.cu): shared-memory limits,
// persistent grids and launches of one group.
cudaError_t dense32_prepare_group(DenseGroup &gr, int n_sm);
void launch_theta32_group(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                          int ring_u, bool skip_abc, cudaStream_t st);
void launch_force32_group(const DenseGroup &gr, const LaunchGeo &lg, const DenseGeo &dg, const StepPtrs &p,
                          int ring_u, int ring_th, bool abc_on, bool first, int *d_step, cudaStream_t st);
// One time step: theta tiles, [IDW], force tiles, ABC prediction; G_u/G_v
// runs beside both tile passes, the next step's G_theta beside the force tiles.
int enqueue_dense_step(const DenseGeo &dg, const LaunchGeo &lg, const StepPtrs &p, int *d_step,
                       cudaStream_t st, const Mark *mark, int ring_u);
// Reset helpers: predicted u^1 (and its FP32 copy u32_1 when not null) and
// vh for every cell from u^0, v^0.
void launch_dense_reset_predict(const LaunchGeo &lg, const double2 *u0, const double2 *v0, double2 *u1,
                                float2 *u32_1, double2 *vh, cudaStream_t st);
// G_theta of the first step (theta^1 at ABC nodes from theta^0, theta^-1); the
// dense step computes each later one a step ahead.
void launch_abc_theta_dense(const DenseGeo &dg, const LaunchGeo &lg, const double *th_n, const double *th_nm1,
                            double *th_np1, cudaStream_t st);
void launch_theta_dense_init(const DenseGeo &dg, const LaunchGeo &lg, const double2 *u, double *theta,
                             cudaStream_t st);
// Diagnostics of the level u = ring_u (its TMA descriptor) with v, a, theta.
void launch_diag_dense(const DenseGeo &dg, const LaunchGeo &lg, int ring_u, const double2 *u, const double2 *v,
                       const double2 *a, const double *theta, DiagPartial *partials, DiagRecord *log,
                       int *log_count, int log_capacity, const int *d_step, cudaStream_t st);

}  // namespace lps
