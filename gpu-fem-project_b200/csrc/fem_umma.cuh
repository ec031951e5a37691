// Blackwell fifth-generation tensor-core primitives (tcgen05) used by the element
// kernel's BF16x6 stiffness stage at order 4 (kU, FEM_PRECISION_MIXED): TMEM
// allocation, the kind::f16 MMA with BF16 operands in shared memory and an FP32
// accumulator in tensor memory, its commit to an mbarrier, and the TMEM loads of
// the epilogue.  Operand tiles are K-major without swizzle: a 64-row x 16-column
// BF16 tile is eight 8-row core matrices of 2 x 16 bytes; element (r, k) sits at
//   (r / 8) * 256 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// bytes from the tile start, i.e. leading-dimension (K) byte offset 128 and
// stride-dimension (8-row group) byte offset 256.  For M = 64 (one CTA) the
// accumulator row m lies in TMEM lane (m % 16) + 32 (m / 16) and column n in
// column n of the allocation: warp w reads rows 16 w .. 16 w + 15 through its
// lanes 0-15.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace fem {
namespace dev {
namespace umma {

constexpr int kTileBytes = 2048;  // one 64 x 16 BF16 operand tile
constexpr uint32_t kLBO = 128, kSBO = 256;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) inside a 64 x 16 tile; k % 8 == 0 gives the start
// of a 16-byte row of eight K-consecutive values.
__host__ __device__ constexpr int tile_offset(int r, int k) {
  return (r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// Shared-memory matrix descriptor: start address, leading and stride byte offsets
// (16-byte units), descriptor version 1 (Blackwell), no swizzle, base offset 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((kLBO >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((kSBO >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 64, M = 64.
constexpr uint32_t kIdescBF16_M64N64 = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((64u >> 4) << 24);

// One warp allocates `ncols` TMEM columns and writes their base address to `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy stores to shared memory visible to the tensor core's (async-proxy) reads
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (+)= A B^T, cta_group::1, kind::f16; accumulate == 0 overwrites D.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrives once on the mbarrier when every MMA this thread issued before has completed.
__device__ __forceinline__ void commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the mbarrier phase `parity` to complete: true when it did,
// false when `limit` polls passed first.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t it = 0; it < limit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive FP32 columns of this warp's 32 TMEM lanes (one lane per thread).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

}  // namespace umma
}  // namespace dev
}  // namespace fem
