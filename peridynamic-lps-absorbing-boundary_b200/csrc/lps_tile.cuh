// lps_tile.cuh -- pieces shared by the FP64 and FP32-mixed dense tile kernels:
// the compile-time stencil, the staged-region geometry, the TMA / mbarrier
// primitives (inline PTX) and the dynamic tile scheduler.
#pragma once
#include <cuda.h>
#include <algorithm>
#include <cstdint>
#include <type_traits>
#include <utility>

#include "lps_dense.cuh"

namespace lps {

// Calls FN<m>(...) for a supported stencil ratio m.
#define LPS_DISPATCH_M(m, FN, ...)      \
  switch (m) {                          \
    case 2: FN<2>(__VA_ARGS__); break;  \
    case 3: FN<3>(__VA_ARGS__); break;  \
    case 4: FN<4>(__VA_ARGS__); break;  \
    case 5: FN<5>(__VA_ARGS__); break;  \
    case 6: FN<6>(__VA_ARGS__); break;  \
    case 8: FN<8>(__VA_ARGS__); break;  \
    default: break;                     \
  }


// ---------------------------------------------------------------------------
// compile-time stencils: {(a, b) != 0 : a^2 + b^2 <= M^2 + M}, enumerated
// a-major from (-M, -M); offset j and N-1-j are negatives of each other.
__host__ __device__ constexpr int sten_count(int M) {
  int n = 0;
  for (int a = -M; a <= M; a++)
    for (int b = -M; b <= M; b++)
      if ((a != 0 || b != 0) && a * a + b * b <= M * M + M) n++;
  return n;
}
__host__ __device__ constexpr int sten_index(int M, int a0, int b0) {
  int n = 0;
  for (int a = -M; a <= M; a++)
    for (int b = -M; b <= M; b++)
      if ((a != 0 || b != 0) && a * a + b * b <= M * M + M) {
        if (a == a0 && b == b0) return n;
        n++;
      }
  return -1;
}
// largest |a| with a^2 + b^2 <= M^2 + M
__host__ __device__ constexpr int amax(int M, int b) {
  int A = 0;
  while ((A + 1) * (A + 1) + b * b <= M * M + M) A++;
  return A;
}

// Compile-time loop: f(std::integral_constant<int, I>) for I in [I0, N), so
// that stencil offsets, table indices and per-offset constants inside f are
// constant expressions (not values the optimiser may or may not fold).
template <int I0, class F, int... Is>
__device__ __forceinline__ void static_for_seq(F &&f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, I0 + Is>{}), ...);  // in order, no recursion depth
}
template <int I0, int N, class F>
__device__ __forceinline__ void static_for(F &&f) {
  if constexpr (N > I0) static_for_seq<I0>(f, std::make_integer_sequence<int, N - I0>{});
}

// Visits the offset pairs (a, b) / (-a, -b) of ratio M column by column,
// b = 0..M, a = -amax..amax (b = 0: a > 0), as
// pair(std::integral_constant<int, a>, std::integral_constant<int, b>); calls
// col_end(std::integral_constant<int, b>) after each column.
template <int M, class P, class E>
__device__ __forceinline__ void for_each_pair(P &&pair, E &&col_end) {
  static_for<0, M + 1>([&](auto bc) {
    constexpr int b = decltype(bc)::value;
    constexpr int A = amax(M, b);
    static_for<0, 2 * A + 1>([&](auto ic) {
      constexpr int a = decltype(ic)::value - A;
      if constexpr (b != 0 || a > 0) pair(std::integral_constant<int, a>{}, bc);
    });
    col_end(bc);
  });
}

template <int M>
struct Sten {
  static constexpr int N = sten_count(M);
  int a[N], b[N];
};

template <int M>
__host__ __device__ constexpr Sten<M> make_sten() {
  Sten<M> s{};
  int n = 0;
  for (int a = -M; a <= M; a++)
    for (int b = -M; b <= M; b++)
      if ((a != 0 || b != 0) && a * a + b * b <= M * M + M) {
        s.a[n] = a;
        s.b[n] = b;
        n++;
      }
  return s;
}

// ---------------------------------------------------------------------------
// staged region geometry; UB / CB: bytes per cell of the staged displacement
// and coefficient pairs (16: FP64 form, 8: FP32-mixed form)
template <int M, int UB = 16, int CB = 16>
struct Region {
  static constexpr int RR = kTileRows + 2 * M;   // staged rows
  static constexpr int RC = kTileCols + 2 * M;   // staged columns (pair boxes)
  static constexpr int RT = 48;                  // staged columns of the u8 box (x16 bytes)
  static constexpr int CELLS = RR * RC;
  static_assert(RC <= RT, "type box narrower than the region");
  static constexpr int U_BYTES = CELLS * UB;
  static constexpr int TH_BYTES = CELLS * 8;
  static constexpr int CO_BYTES = CELLS * CB;
  static constexpr int TY_BYTES = RR * RT;
  static constexpr int align128(int x) { return (x + 127) / 128 * 128; }
  // every TMA destination starts on a 128-byte boundary
  // theta stage: u | type
  static constexpr int T_TY = align128(U_BYTES);
  static constexpr int THETA_STAGE = align128(T_TY + TY_BYTES);
  static constexpr int THETA_TX = U_BYTES + TY_BYTES;
  // force stage: u | th | coef | type
  static constexpr int F_TH = align128(U_BYTES);
  static constexpr int F_CO = align128(F_TH + TH_BYTES);
  static constexpr int F_TY = align128(F_CO + CO_BYTES);
  static constexpr int FORCE_STAGE = align128(F_TY + TY_BYTES);
  static constexpr int FORCE_TX = U_BYTES + TH_BYTES + CO_BYTES + TY_BYTES;
  static constexpr int THETA_SMEM = 2 * THETA_STAGE + 64;
  static constexpr int FORCE_SMEM = 2 * FORCE_STAGE + 64;
};

template <int M>
__device__ __forceinline__ int QI(int r, int c) {
  return (r + M) * Region<M>::RC + (c + M);
}

// ---- TMA / mbarrier primitives (inline PTX) --------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait on a transaction barrier: gives up after ~2 s (clock64) or
// 2^26 polls, whichever comes first, and raises the error flag.
constexpr int kErrWaitTimeout = 1;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *err) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  for (int it = 0; it < (1 << 26); it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > 4000000000LL) break;
  }
  atomicExch(err, kErrWaitTimeout);
  return false;
}

// After a timed-out wait in iteration `it` of a double-buffered tile loop:
// waits (bounded) for the copies still in flight into this CTA's two stages --
// the one the loop gave up on and, if it was issued, the next one -- so that no
// bulk copy lands in shared memory after the CTA has left.  Thread 0 (the
// thread that issued the copies) calls it.
__device__ __forceinline__ void drain_stages(uint64_t *bar, int it, bool next_issued, int *err) {
  const int stage = it & 1;
  mbar_wait_bounded(&bar[stage], (it >> 1) & 1, err);
  if (next_issued) mbar_wait_bounded(&bar[stage ^ 1], ((it + 1) >> 1) & 1, err);
}

// Dynamic tile scheduler of the persistent tile kernels: a CTA takes its next
// tile from a counter, so a CTA that becomes resident late (its SM still runs
// blocks of the concurrent absorbing-boundary kernel) takes fewer tiles instead
// of stretching the launch.  sched[0] is the next tile, sched[1] counts
// finished CTAs; the last CTA to finish rewinds both for the next launch.
__device__ __forceinline__ int sched_next(int *sched) { return atomicAdd(sched, 1); }

__device__ __forceinline__ void sched_finish(int *sched) {
  __threadfence();
  if (atomicAdd(sched + 1, 1) == (int)gridDim.x - 1) {
    sched[0] = 0;
    sched[1] = 0;
  }
}

}  // namespace lps
