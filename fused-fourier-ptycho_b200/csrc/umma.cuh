// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a: shared-memory
// operand descriptors, the BF16 x BF16 -> FP32 instruction descriptor, the MMA, its
// completion on an mbarrier, tensor-memory (TMEM) allocation and the loads of the
// accumulator.  One CTA (cta_group::1), operands K-major in shared memory with the
// 128-byte swizzle.
//
// Operand tile layout (K-major, 128-byte swizzle): a tile of R rows by 64 BF16 along K
// is R rows of 128 bytes; the 16-byte chunk c of row r sits at
//     r * 128 + ((c ^ (r & 7)) * 16)
// from a 1024-byte aligned base, so eight rows form one 1024-byte swizzle atom.  An MMA
// consumes K = 16 (32 bytes of each row); the k-th of the four K steps of a tile starts
// 32 k bytes into the rows (the hardware applies the swizzle to the addresses it forms).
#pragma once

#include <cstdint>

namespace fpm {
namespace umma {

__device__ __forceinline__ uint32_t saddr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Descriptor of a K-major, 128-byte swizzled operand tile starting at shared address a
// (1024-byte aligned, or 32 k bytes past such an address for the k-th K step):
// start address >> 4 in bits [0, 14), leading byte offset 1 (unused with a swizzle) in
// [16, 30), stride byte offset 1024 >> 4 (between 8-row groups) in [32, 46), descriptor
// version 1 in [46, 48), base offset 0, layout type 2 (128-byte swizzle) in [61, 64).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t a) {
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 accumulation, both
// operands K-major, dense, no negation: D format (1 = F32) in bits [4, 6), A and B
// formats (1 = BF16) in [7, 10) and [10, 13), N >> 3 in [17, 23), M >> 4 in [24, 29).
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A B^T for one K step; accumulate = 0 overwrites D.  Issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// The mbarrier at bar completes one arrival once every MMA this thread issued before is
// done (its shared-memory operands may then be overwritten, its TMEM result read).
__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     saddr(bar))
                 : "memory");
}

// ordering of tcgen05 operations against thread barriers
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Allocates ncols TMEM columns (a power of two >= 32) for the CTA and writes their base
// address to *slot (shared memory).  Executed by one whole warp.
__device__ __forceinline__ void alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Frees what alloc took (one whole warp, after every use of the columns).
__device__ __forceinline__ void dealloc(uint32_t tmem, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols)
                 : "memory");
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (the warp reads lanes
// 32 (warp % 4) .. +31 at column offset col of the address).
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// TMEM columns to allocate for an accumulator of n FP32 columns
__host__ __device__ constexpr uint32_t tmem_cols(int n) {
    return n <= 32 ? 32u : n <= 64 ? 64u : n <= 128 ? 128u : n <= 256 ? 256u : 512u;
}

}  // namespace umma
}  // namespace fpm
