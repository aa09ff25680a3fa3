// Device helpers of the TMA-staged kernels: mbarriers with bounded waits, 3-D tensor loads,
// closure classes.
#pragma once

#include <stdint.h>

#include <type_traits>
#include <utility>

#include <cuda.h>

namespace lee {
namespace {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(n) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ unsigned mbar_try(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok;
}

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// The default limit of a bounded wait: one second of %globaltimer.
constexpr unsigned long long kWaitNs = 1000000000ull;

// Wait for the phase of the given parity; false once `limit_ns` nanoseconds have passed. A limit
// of 0 gives up at once, without looking: it drives the failure path in tests, whether or not the
// copy has landed. The drains that follow a failed wait always use the default limit, so a CTA
// never exits with a copy in flight.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity, unsigned long long limit_ns = kWaitNs) {
  if (limit_ns == 0) return false;
  if (mbar_try(b, parity)) return true;
  const unsigned long long t0 = gtimer();
  for (unsigned it = 1;; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 63u) == 0u && gtimer() - t0 > limit_ns) return false;
  }
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

template <int N, typename F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
// f(integral_constant<0>) ... f(integral_constant<N-1>), in order
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl<N>(f, std::make_integer_sequence<int, N>{});
}

// Closure class of a position along a line with nb closure rows at each end:
// 0 interior, 1 + p for the left rows, 1 + nb + (n - 1 - p) for the right rows.
__device__ __forceinline__ int cls_of(int pos, int n, int nb) {
  return pos < nb ? 1 + pos : (pos > n - 1 - nb ? 1 + nb + (n - 1 - pos) : 0);
}

// The same classes from a closure code (closure_codes on the host: 0 interior, 1 + r the left
// row r, -(1 + r) the mirrored right row r, kCodeZero a zero value), the zero class 1 + 2 nb.
__device__ __forceinline__ int cls_of_code(int code, int nb) {
  if (code == kCodeZero) return 1 + 2 * nb;
  return code >= 0 ? code : 1 + nb + (-code - 1);
}

}  // namespace
}  // namespace lee
