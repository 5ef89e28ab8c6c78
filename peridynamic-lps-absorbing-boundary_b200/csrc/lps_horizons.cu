// lps_horizons.cu -- the horizon (neighbour) search on the GPU.
//
// The reference finds each node's horizon with a k-d tree range query and
// sorts it by distance (src/main.cpp:352-356, kd_tree_interface.h:43-126);
// the host setup (lps_setup.cpp) does the same with a bucket grid and an
// (distance, index) order.  This is that search as one kernel, for large node
// sets: nodes are bucketed on the host (a counting sort, O(N)), then one warp
// per node scans the 3 x 3 buckets around its own, keeps the candidates within
// the search radius in shared memory and sorts them by (distance, index) with
// a bitonic sort.  Distances are formed without FMA contraction and with the
// correctly rounded square root, so every inclusion test and every order
// decision is the host's bit for bit (tests compare the two builds).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "lps_cuda.h"
#include "lps_setup.h"

namespace lps {

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kMaxRow = 256;   // shared-memory candidates per warp (longer rows: the host build)

// A candidate's sort key: (distance, node) in lexicographic order.
__device__ __forceinline__ bool key_less(double da, int ja, double db, int jb) {
  return da < db || (da == db && ja < jb);
}

__global__ void __launch_bounds__(32 * kWarpsPerBlock)
    k_horizons(int n, const double2 *__restrict__ xy, const long *__restrict__ cell, const int *__restrict__ start,
               const int *__restrict__ order, long gx, long gy, double r, int row_len, int *__restrict__ len,
               int *__restrict__ hz, int *__restrict__ overflow) {
  __shared__ double s_d[kWarpsPerBlock][kMaxRow];
  __shared__ int s_j[kWarpsPerBlock][kMaxRow];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kWarpsPerBlock + w;
  if (i >= n) return;  // whole warps leave together
  double *sd = s_d[w];
  int *sj = s_j[w];
  const double2 p = xy[i];
  const long cx = cell[i] % gx, cy = cell[i] / gx;
  int cnt = 0;  // candidates kept (warp-uniform)
  for (long by = max(0L, cy - 1); by <= min(gy - 1, cy + 1); by++)
    for (long bx = max(0L, cx - 1); bx <= min(gx - 1, cx + 1); bx++) {
      const long c = by * gx + bx;
      for (int q0 = start[c]; q0 < start[c + 1]; q0 += 32) {
        const int q = q0 + lane;
        double d = 0.0;
        int j = -1;
        bool keep = false;
        if (q < start[c + 1]) {
          j = order[q];
          const double2 o = xy[j];
          const double x = __dadd_rn(o.x, -p.x), y = __dadd_rn(o.y, -p.y);
          d = __dsqrt_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)));
          keep = d <= r;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        const int slot = cnt + __popc(mask & ((1u << lane) - 1u));
        if (keep && slot < kMaxRow) {
          sd[slot] = d;
          sj[slot] = j;
        }
        cnt += __popc(mask);
      }
    }
  __syncwarp();
  if (cnt > row_len) {
    if (lane == 0) atomicExch(overflow, 1);
    cnt = row_len;  // the host reports LPS_ERR_HORIZON; rows are cut as the host cuts them
  }
  // bitonic sort of the first P >= cnt entries (padding sorts last)
  int P = 1;
  while (P < cnt) P <<= 1;
  for (int k = cnt + lane; k < P; k += 32) {
    sd[k] = INFINITY;
    sj[k] = 0x7fffffff;
  }
  __syncwarp();
  for (int size = 2; size <= P; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = lane; t < P / 2; t += 32) {
        const int a = 2 * t - (t & (stride - 1)), b = a + stride;
        const bool up = (a & size) == 0;
        const double da = sd[a], db = sd[b];
        const int ja = sj[a], jb = sj[b];
        if (key_less(db, jb, da, ja) == up) {
          sd[a] = db;
          sj[a] = jb;
          sd[b] = da;
          sj[b] = ja;
        }
      }
      __syncwarp();
    }
  int *row = hz + (size_t)i * row_len;
  for (int k = lane; k < row_len; k += 32) row[k] = k < cnt ? sj[k] : -1;
  if (lane == 0) len[i] = cnt;
}

}  // namespace

// The horizons of build_horizons (lps_setup.cpp), computed on the current
// device.  Returns the longest row (before any cut), LPS_ERR_HORIZON if a row
// exceeds row_len, or LPS_ERR_CUDA.
int build_horizons_gpu(int n, const double *xy, double r, int row_len, std::vector<int> &len,
                       std::vector<int> &hz) {
  if (row_len > kMaxRow) return build_horizons(n, xy, r, row_len, len, hz);
  double xmin = xy[0], xmax = xy[0], ymin = xy[1], ymax = xy[1];
  for (int i = 1; i < n; i++) {
    xmin = std::min(xmin, xy[2 * i]); xmax = std::max(xmax, xy[2 * i]);
    ymin = std::min(ymin, xy[2 * i + 1]); ymax = std::max(ymax, xy[2 * i + 1]);
  }
  // the host build's buckets: side r, ascending node index inside a bucket
  const double cs = r > 0 ? r : 1.0;
  const long gx = (long)std::floor((xmax - xmin) / cs) + 1;
  const long gy = (long)std::floor((ymax - ymin) / cs) + 1;
  std::vector<int> start(gx * gy + 1, 0), order(n);
  std::vector<long> cell(n);
  for (int i = 0; i < n; i++) {
    const long cx = (long)std::floor((xy[2 * i] - xmin) / cs), cy = (long)std::floor((xy[2 * i + 1] - ymin) / cs);
    cell[i] = cy * gx + cx;
    start[cell[i] + 1]++;
  }
  for (long c = 0; c < gx * gy; c++) start[c + 1] += start[c];
  {
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int i = 0; i < n; i++) order[fill[cell[i]]++] = i;
  }
  double2 *d_xy = nullptr;
  long *d_cell = nullptr;
  int *d_start = nullptr, *d_order = nullptr, *d_len = nullptr, *d_hz = nullptr, *d_over = nullptr;
  int status = LPS_OK;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && status == LPS_OK) status = LPS_ERR_CUDA;
    return status == LPS_OK;
  };
  if (ok(cudaMalloc(&d_xy, sizeof(double2) * n)) && ok(cudaMalloc(&d_cell, sizeof(long) * n)) &&
      ok(cudaMalloc(&d_start, sizeof(int) * start.size())) && ok(cudaMalloc(&d_order, sizeof(int) * n)) &&
      ok(cudaMalloc(&d_len, sizeof(int) * n)) && ok(cudaMalloc(&d_hz, sizeof(int) * (size_t)n * row_len)) &&
      ok(cudaMalloc(&d_over, sizeof(int))) &&
      ok(cudaMemcpy(d_xy, xy, sizeof(double2) * n, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(d_cell, cell.data(), sizeof(long) * n, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(d_start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice)) &&
      ok(cudaMemset(d_over, 0, sizeof(int)))) {
    const int blocks = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
    k_horizons<<<blocks, 32 * kWarpsPerBlock>>>(n, d_xy, d_cell, d_start, d_order, gx, gy, r, row_len, d_len, d_hz,
                                                d_over);
    len.resize(n);
    hz.resize((size_t)n * row_len);
    int over = 0;
    if (ok(cudaGetLastError()) && ok(cudaMemcpy(len.data(), d_len, sizeof(int) * n, cudaMemcpyDeviceToHost)) &&
        ok(cudaMemcpy(hz.data(), d_hz, sizeof(int) * (size_t)n * row_len, cudaMemcpyDeviceToHost)) &&
        ok(cudaMemcpy(&over, d_over, sizeof(int), cudaMemcpyDeviceToHost)) && over)
      status = LPS_ERR_HORIZON;
  }
  cudaFree(d_xy);
  cudaFree(d_cell);
  cudaFree(d_start);
  cudaFree(d_order);
  cudaFree(d_len);
  cudaFree(d_hz);
  cudaFree(d_over);
  if (status != LPS_OK) return status;
  int longest = 0;
  for (int i = 0; i < n; i++) longest = std::max(longest, len[i]);
  return longest;
}

}  // namespace lps
