// Shared helpers of the hand-written tcgen05 GEMMs (sm_100a): mbarriers with
// bounded waits, the 128B-swizzled K-major UMMA shared-memory descriptor and
// its element offsets, and the MMA commit.  Every operand tile is 128 rows x
// 128 bytes (32 TF32 or 64 BF16 per row) stored in the SW128 layout.
#pragma once
#include "ctx.cuh"

namespace ipeps {
namespace {

constexpr long long WAIT_LIMIT = 1LL << 22;  // bounded mbarrier waits (then the status word records it)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// bounded wait for the phase with the given parity; false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// SW128 K-major UMMA shared-memory descriptor (LBO = 16 B, SBO = 1024 B,
// descriptor version 1, layout type 2 = 128B swizzle)
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
  return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t(1) << 16) | (uint64_t(1024 >> 4) << 32) |
         (uint64_t(1) << 46) | (uint64_t(2) << 61);
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// byte offset of 16-byte chunk `chunk` of row r in a 128-row K-major SW128 tile
__device__ __forceinline__ uint32_t sw128(int r, int chunk) {
  return uint32_t((r >> 3) * 1024 + (r & 7) * 128 + ((chunk ^ (r & 7)) << 4));
}

}  // namespace
}  // namespace ipeps
