// umma.cuh -- fifth-generation tensor-core (tcgen05) helpers for sm_100a
// (internal header): tensor-memory allocation, shared-memory matrix
// descriptors, BF16 MMA with FP32 accumulation in tensor memory, commit to an
// mbarrier, and tensor-memory loads for the epilogue.
//
// Operand images.  Every operand lives in shared memory as a K-major "image"
// in the 128-byte swizzled layout: K is split into atoms of 64 BF16 values
// (128 bytes); within an atom, row r occupies bytes [128 r, 128 r + 128), and
// its 16-byte chunk c is stored at chunk c ^ (r & 7).  Atoms of an image with
// R rows are R * 128 bytes apart.  An image starts on a 1024-byte boundary so
// that the swizzle phase, which the hardware takes from address bits [7, 10),
// matches r & 7.  The same layout is kept in global memory for images that a
// kernel copies in with one bulk copy.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "mbar.cuh"

namespace alebgk {

// Byte offset of element (r, k) in a K-major swizzled image of `rows` rows.
__host__ __device__ __forceinline__ uint32_t swzOffset(int r, int k, int rows)
{
    return (uint32_t)((k >> 6) * rows * 128 + r * 128 + ((((k & 63) >> 3) ^ (r & 7)) << 4) +
                      (k & 7) * 2);
}

// Bytes of an image with `rows` rows and K columns (K a multiple of 16).
__host__ __device__ __forceinline__ uint32_t swzBytes(int rows, int K)
{
    return (uint32_t)(((K + 63) >> 6) * rows * 128);
}

// Shared-memory matrix descriptor of the K-step `kk` (16 BF16 values) of a
// K-major 128-byte-swizzled image at shared address `base` with `rows` rows:
//   start address >> 4 in bits [0,14); leading byte offset 16 B (unused by
//   swizzled K-major layouts) in [16,30); stride byte offset 1024 B between
//   8-row groups in [32,46); descriptor version 1 in [46,48); swizzle mode
//   128 B (2) in [61,64).
__device__ __forceinline__ uint64_t ummaDesc(uint32_t base, int rows, int kk)
{
    const uint32_t addr = base + (uint32_t)((kk >> 2) * rows * 128 + (kk & 3) * 32);
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator, both
// operands K-major, M x N tile.
__host__ __device__ constexpr uint32_t ummaIdescBf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K-step; issued by a single thread.
__device__ __forceinline__ void ummaBf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc,
                                         uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrives once on `bar` when every MMA this thread issued before has completed.
__device__ __forceinline__ void ummaCommit(uint64_t *bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smemAddr(bar))
        : "memory");
}

__device__ __forceinline__ void tmemFenceBefore()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmemFenceAfter()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Allocates `ncols` tensor-memory columns (a power of two >= 32); the whole
// warp executes it and the base address lands in *slot.
__device__ __forceinline__ void tmemAlloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smemAddr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmemDealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
                 "r"(ncols)
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's lane.  The warp reads lanes
// [32 (warp % 4), +32); `taddr` carries that lane base in bits [16, 32).
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Round-to-nearest-even FP32 -> BF16 of a pair, packed low | high << 16.
__device__ __forceinline__ uint32_t packBf16(float lo, float hi)
{
    uint32_t out;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(out) : "f"(hi), "f"(lo));
    return out;
}

__device__ __forceinline__ float bf16Lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16Hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

}  // namespace alebgk
