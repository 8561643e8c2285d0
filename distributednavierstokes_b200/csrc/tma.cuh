// tma.cuh -- bulk asynchronous copies (TMA) and mbarrier helpers, sm_90+.
//
// A persistent CTA prefetches the next tile of lines with one
// cp.async.bulk (global -> shared, completion counted on an mbarrier)
// while it transforms the current one.  No multicast is used anywhere.
// Every wait is bounded: after a caller-given number of polls the kernel
// records an error code in a global word and returns; DNSB_WAIT_LIMIT is the
// default limit and the one used to drain copies still in flight.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dnsb {

constexpr unsigned DNSB_WAIT_LIMIT = 1u << 26;
enum DevErr { DEVERR_NONE = 0, DEVERR_TMA_TIMEOUT = 1 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order earlier generic-proxy accesses of shared memory before later
// async-proxy (bulk copy) writes to it
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// 1D bulk copy global -> shared; bytes, src and dst multiples of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// expected transaction bytes of the current phase, without an arrival
__device__ __forceinline__ void mbar_expect_tx_only(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 3-D tiled tensor copy global -> shared (box of the tensor map at
// coordinates {c0, c1, c2}; out-of-range elements read as zero)
__device__ __forceinline__ void tma_load3(void *dst, const void *map, int c0, int c1, int c2,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
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

// bounded wait of the calling thread: at most `limit` polls (0: none);
// returns false when they ran out
__device__ __forceinline__ bool mbar_wait_n(uint64_t *bar, uint32_t parity, unsigned limit) {
  for (unsigned it = 0; it < limit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Per-thread asynchronous 16-byte copy global -> shared (bypasses L1); the
// copies of a thread form groups (commit) that are waited for in order.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// waits until at most N of this thread's groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

}  // namespace dnsb
