// umma.cuh -- thin sm_100a tensor-core helpers (tcgen05 + TMEM + mbarrier)
// used by the MLP radiance cache.
//
// Operand tiles live in shared memory in the canonical no-swizzle layout:
// 8 x 16-byte "core matrices" (8 rows, 8 bf16 each).  For a matrix of R rows
// and C bf16 columns stored "row-contiguous in 16-byte chunks", element
// (r, c) is at byte
//     ((r / 8) * (C / 8) + c / 8) * 128 + (r % 8) * 16 + (c % 8) * 2.
// Read K-major (rows = M or N, columns = K) the core matrix stride along M/N
// (SBO) is 16*C bytes and along K (LBO) 128 bytes.  The same bytes read
// MN-major (columns = M or N, rows = K) have MN-group stride 128 bytes and
// K-group stride 16*C bytes -- which lets a weight-gradient GEMM consume the
// forward activations without a transpose.
#pragma once
#include <cstdint>

#define UMMA_DI __device__ __forceinline__

namespace vrt {
namespace umma {

UMMA_DI uint32_t canon_off(int r, int c, int C) {
  return (uint32_t)((((r >> 3) * (C >> 3) + (c >> 3)) << 7) + ((r & 7) << 4) + ((c & 7) << 1));
}

UMMA_DI uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (no swizzle).  lbo/sbo in bytes.
UMMA_DI uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version for sm_100
  return d;                 // base offset 0, legacy LBO mode, layout SWIZZLE_NONE
}

// Descriptor of a row-chunked matrix with C columns read K-major (K = columns).
UMMA_DI uint64_t desc_kmajor(uint32_t saddr, int C) { return smem_desc(saddr, 128u, 16u * (uint32_t)C); }
// The same matrix read MN-major (MN = columns, K = rows).
UMMA_DI uint64_t desc_mnmajor(uint32_t saddr, int C) { return smem_desc(saddr, 16u * (uint32_t)C, 128u); }

// Instruction descriptor of kind::f16 with BF16 A/B, FP32 D.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]; issued by one thread.
UMMA_DI void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// Arrive on `mbar` once all previously issued MMAs of this thread completed.
UMMA_DI void commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

UMMA_DI void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for phase `parity` of `mbar`; false when the bound ran out.
UMMA_DI bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t max_iter) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t i = 0; i < max_iter; i++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Generic-proxy shared-memory writes -> visible to the tensor core (async proxy).
UMMA_DI void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
UMMA_DI void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
UMMA_DI void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation by one full warp; the base address is written to *dst_smem.
UMMA_DI void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
UMMA_DI void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane (warp w reads lanes
// 32w..32w+31; taddr must already include the warp's lane offset).
UMMA_DI void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Raw 16-column load without the wait.  The registers are valid only after
// tmem_wait_dep() on the same array, which also orders every later use of
// them after the wait (the wait takes them as read-write operands).
UMMA_DI void tmem_ld16_raw(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
UMMA_DI void tmem_wait_dep(uint32_t* r) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15])
               :
               : "memory");
}

}  // namespace umma
}  // namespace vrt
