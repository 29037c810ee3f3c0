// Shared device helpers for the redrock-b200 kernels (sm_100a only).
//
// Error words, bounded mbarrier waits and 1-D bulk (TMA) copies.  Every
// spin-wait in this library is bounded: after RR_SPIN_LIMIT polls the
// waiting thread records RR_ETIMEOUT in a device status word and the kernel
// returns instead of hanging.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/redrock_b200.h"

#ifndef RR_SPIN_LIMIT
#define RR_SPIN_LIMIT (1u << 26)
#endif

namespace rr {

// "exactly nine nines": redrock's HUGE_CHI2 (zscan.py:18)
constexpr double kHugeChi2 = 9999999.0;

// resolution half-bandwidth handled by the band kernels: offsets -5..5
constexpr int kHalfBand = 5;
constexpr int kBand = 2 * kHalfBand + 1;

__device__ __forceinline__ void set_status(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// ---------------------------------------------------------------------------
// mbarrier + bulk copy (cp.async.bulk, the 1-D form of the TMA engine)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// Bounded wait on phase `parity`.  Returns true when the phase completed,
// false (after recording RR_ETIMEOUT) when the poll limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status) {
  uint32_t addr = smem_u32(bar);
  for (uint32_t it = 0; it < RR_SPIN_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  set_status(status, RR_ETIMEOUT);
  return false;
}

// Global -> shared bulk copy completing on `bar`.  dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// IEEE-rounded double arithmetic that the compiler may not contract into
// FMAs: used where results must reproduce a reference's operation order
// bit for bit.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

}  // namespace rr

#define RR_CUDA_TRY(expr)                           \
  do {                                              \
    cudaError_t _e = (expr);                        \
    if (_e != cudaSuccess) return RR_ECUDA;         \
  } while (0)

#define RR_CHECK_LAUNCH()                           \
  do {                                              \
    cudaError_t _e = cudaGetLastError();            \
    if (_e != cudaSuccess) return RR_ECUDA;         \
  } while (0)
