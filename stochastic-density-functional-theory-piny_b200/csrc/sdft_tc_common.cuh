// sdft_tc_common.cuh -- device helpers shared by the tcgen05 GEMM kernels:
// mbarriers with bounded waits, TMA tile loads, shared-memory matrix
// descriptors, MMA commit and TMEM loads (inline PTX, sm_100a).
//
// Every wait on an mbarrier gives up after kWaitLimit polls, sets the
// device error word (read by the host as SDFT_ERR_TIMEOUT) and lets the
// kernel run to its end; no kernel here can spin forever.  No TMA load
// uses cluster multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace sdft {

constexpr long long kWaitLimit = 1ll << 22;  // bounded spin on mbarriers

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count));
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, int *err, long long limit = kWaitLimit) {
  for (long long i = 0; i < limit; i++)
    if (mbar_try(a, parity)) return true;
  atomicExch(err, 1);
  return false;
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *tm, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(tm), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *tm, int x, int y, int z,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(dst), "l"(tm), "r"(x), "r"(y), "r"(z), "r"(mbar)
      : "memory");
}

// tcgen05 shared-memory matrix descriptor for a K-major operand whose rows
// are one swizzle span wide: start address, leading byte offset field 1
// (unused for swizzled K-major tiles), stride byte offset = distance
// between 8-row groups, descriptor version 1, swizzle mode
// (2 = 128 B, 4 = 64 B).
template <int SWZ_BYTES>
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  static_assert(SWZ_BYTES == 128 || SWZ_BYTES == 64, "swizzle span");
  constexpr uint64_t mode = (SWZ_BYTES == 128) ? 2ull : 4ull;
  constexpr uint64_t sbo = (uint64_t)(8 * SWZ_BYTES) >> 4;
  return (uint64_t)((saddr >> 4) & 0x3FFF) | (1ull << 16) | (sbo << 32) | (1ull << 46) | (mode << 61);
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t ta, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(ta));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace sdft
