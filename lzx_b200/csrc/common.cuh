// common.cuh -- shared device helpers for the lattice_cuda library (sm_100a).
//
// TMA bulk copies (cp.async.bulk, no multicast), mbarrier waits with an
// iteration bound, and the library-wide error flag.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lattice_cuda.h"

#define LC_HD __host__ __device__ __forceinline__
#define LC_D __device__ __forceinline__

// Spin bound for every wait on an mbarrier: about 2^26 polls (well above any
// legitimate TMA latency, far below a watchdog).  On expiry the kernel records
// LC_DEVERR_TIMEOUT in the plan's device error word and returns.
constexpr uint32_t kSpinLimit = 1u << 26;

// LC_DEVERR_POISONED: after a timeout, a bulk copy of the timed-out kernel
// did not land within a second bounded wait either, so it may still write
// into shared memory that a later CTA owns; the word stays set (sticky).
enum : uint32_t {
  LC_DEVERR_NONE = 0,
  LC_DEVERR_TIMEOUT = 1,
  LC_DEVERR_POISONED = 2,
};

namespace lc {

LC_D uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

LC_D void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

LC_D void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

LC_D void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

LC_D void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Returns true once the phase with the given parity has completed, false if
// the spin bound expired first.
LC_D bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint32_t addr = smem_u32(bar);
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
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
  return false;
}

// 1-D bulk copy global -> shared, completion signalled on an mbarrier.
// dst, src 16-byte aligned; bytes a multiple of 16.
LC_D void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// 1-D bulk copy shared -> global (bulk-group completion).
LC_D void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_u32(src)), "r"(bytes)
               : "memory");
}

LC_D void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Wait until at most N committed bulk groups still read shared memory.
template <int N>
LC_D void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

template <int N>
LC_D void bulk_wait() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}

// Make generic-proxy writes to shared memory visible to the async (TMA) proxy.
LC_D void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

LC_D void record_error(uint32_t* err, uint32_t code) {
  if (err) atomicCAS(err, 0u, code);
}

LC_D void record_poisoned(uint32_t* err) {
  if (err) atomicMax(err, (uint32_t)LC_DEVERR_POISONED);
}

}  // namespace lc
