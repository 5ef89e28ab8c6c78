// lps_noalloc.cu -- state diagnostics that allocate nothing.
//
// Some callers cannot allocate device memory at the moment they need these
// numbers: a control loop that may not pay the implicit device-wide
// synchronisation of cudaMalloc/cudaFree between time steps, a host program
// whose GPU memory belongs to another allocator (a framework's caching pool)
// that this library must not grow or fragment, or code that runs while a
// stream capture is active.  lps_state_diag_noalloc serves them: it reduces a
// state the caller already holds in device memory to the kinetic energy,
// momentum and maxima of the reference's output step (src/main.cpp:992-1016)
// and writes them to a device buffer the caller passes.  Its only scratch --
// one partial-sum record per 256-node block -- is the file-scope device array
// below, so the call itself never allocates.
#include <cstdint>
#include <mutex>
#include <string>

#include "lps_common.cuh"
#include "lps_cuda.h"

namespace lps {
void set_create_error(const char *msg);  // lps_api.cu
}

namespace {

using lps::DiagAcc;
using lps::DiagPartial;

constexpr int kBlock = 256;
constexpr int kMaxBlocks = LPS_NOALLOC_MAX_NODES / kBlock;

// Per-block partial sums.  Every GPU that loads this library holds this array
// (kMaxBlocks x 112 bytes, about 0.46 MB) until the process exits; all calls
// on a device share it, and each call overwrites the slots it uses.
static __device__ __align__(256) DiagPartial g_partials[kMaxBlocks];

// Device addresses of g_partials, one per device, resolved with that device
// current (in host code the symbol name is only a host-side stand-in).  Each
// address is kept with the context it was resolved in: a context destroyed
// and recreated (cudaDeviceReset) reloads the module, so the address is
// resolved again in the new context.
constexpr int kMaxDevices = 64;
DiagPartial *g_addr[kMaxDevices] = {};
void *g_ctx[kMaxDevices] = {};
std::mutex g_addr_mu;

// The current driver context (cuCtxGetCurrent through the runtime's entry
// point table, so the library needs no link against libcuda).
void *current_context() {
  using Fn = int (*)(void **);
  static Fn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<Fn>(p);
  });
  void *ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

bool aligned(const void *p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

__global__ void __launch_bounds__(kBlock)
    k_state_partials(int n, const double2 *__restrict__ xy, const double2 *__restrict__ u,
                     const double2 *__restrict__ v, const double2 *__restrict__ a,
                     const double *__restrict__ theta, double rho, double dx, double dy, double out_r,
                     DiagPartial *part) {
  DiagAcc acc;
  acc.init();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i < n) {
    const double2 p = xy[i], un = u[i], vn = v[i], an = a[i];
    acc.add_maxima(un, vn, an, theta[i], i);
    const double r = sqrt(p.x * p.x + p.y * p.y);
    if (!(out_r > 0.0 && r > out_r)) {  // energy and momentum exclude the layer, :1007
      acc.Px = rho * vn.x * dx * dy;
      acc.Py = rho * vn.y * dx * dy;
      acc.Ek = 0.5 * rho * (vn.x * vn.x + vn.y * vn.y) * dx * dy;
      acc.E = acc.Ek;
    }
  }
  acc.block_reduce_store(part + blockIdx.x);
}

// One block folds the partials in block order and writes the results.
__global__ void __launch_bounds__(kBlock) k_state_finish(int nblocks, const DiagPartial *part, double *out) {
  const int per = (nblocks + kBlock - 1) / kBlock;
  DiagAcc acc;
  acc.init();
  for (int b = threadIdx.x * per; b < min(nblocks, (int)(threadIdx.x + 1) * per); b++) {
    DiagAcc r;
    r.from_partial(part + b);
    acc.combine(r);
  }
  __shared__ DiagPartial res;
  acc.block_reduce_store(&res);
  __syncthreads();
  if (threadIdx.x == 0) {
    out[0] = res.Ek;
    out[1] = res.Px;
    out[2] = res.Py;
    out[3] = res.max_u;
    out[4] = res.max_v;
    out[5] = res.max_a;
    out[6] = res.th_min;
    out[7] = res.th_max;
    out[8] = (double)res.iu;
    out[9] = (double)res.iv;
  }
}

}  // namespace

extern "C" int lps_state_diag_noalloc(int n_nodes, const double *xy, const double *u, const double *v,
                                      const double *a, const double *theta, double rho, double dx, double dy,
                                      double exclude_r, double *out, void *stream) {
  if (n_nodes <= 0 || n_nodes > LPS_NOALLOC_MAX_NODES) {
    lps::set_create_error("lps_state_diag_noalloc: n_nodes must be 1.." "1048576 (LPS_NOALLOC_MAX_NODES)");
    return LPS_ERR_INVALID_ARG;
  }
  if (!xy || !u || !v || !a || !theta || !out) {
    lps::set_create_error("lps_state_diag_noalloc: a device pointer is NULL");
    return LPS_ERR_INVALID_ARG;
  }
  // the kernel reads x/y pairs as 16-byte double2 loads
  if (!aligned(xy, 16) || !aligned(u, 16) || !aligned(v, 16) || !aligned(a, 16) || !aligned(theta, 8) ||
      !aligned(out, 8)) {
    lps::set_create_error("lps_state_diag_noalloc: xy, u, v, a must be 16-byte aligned, theta and out 8-byte");
    return LPS_ERR_INVALID_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    lps::set_create_error("lps_state_diag_noalloc: no current CUDA device");
    return LPS_ERR_NO_DEVICE;
  }
  {
    // an error the caller left pending is the caller's: report it, keep it
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
      lps::set_create_error((std::string("lps_state_diag_noalloc: a CUDA error was pending before the call: ") +
                             cudaGetErrorString(pending)).c_str());
      return LPS_ERR_CUDA;
    }
  }
  DiagPartial *part = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_addr_mu);
    void *ctx = current_context();
    if (!g_addr[dev] || g_ctx[dev] != ctx) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
      if (e != cudaSuccess || !p) {
        lps::set_create_error((std::string("lps_state_diag_noalloc: cudaGetSymbolAddress failed: ") +
                               cudaGetErrorString(e)).c_str());
        return LPS_ERR_CUDA;
      }
      g_addr[dev] = static_cast<DiagPartial *>(p);
      g_ctx[dev] = ctx;
    }
    part = g_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nblocks = (n_nodes + kBlock - 1) / kBlock;
  k_state_partials<<<nblocks, kBlock, 0, st>>>(n_nodes, reinterpret_cast<const double2 *>(xy),
                                               reinterpret_cast<const double2 *>(u),
                                               reinterpret_cast<const double2 *>(v),
                                               reinterpret_cast<const double2 *>(a), theta, rho, dx, dy, exclude_r,
                                               part);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_state_finish<<<1, kBlock, 0, st>>>(nblocks, part, out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    lps::set_create_error((std::string("lps_state_diag_noalloc: kernel launch failed: ") + cudaGetErrorString(e))
                              .c_str());
    return LPS_ERR_CUDA;
  }
  return LPS_OK;
}
