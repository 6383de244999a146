// nn_tc.cuh -- 5th-generation tensor-core primitives (tcgen05 + TMEM) for the surrogate's
// dense layers on sm_100a: shared-memory matrix descriptors, the BF16 instruction
// descriptor, TMEM allocation, MMA issue/commit, bounded mbarrier waits and TMEM loads.
//
// Shared-memory tile format used by every operand ("row tile"): a row-major source block of
// R rows x F features (bf16) is stored as 16-byte chunks of 8 features,
//     byte offset(row, f) = (f / 8) * (R * 16) + row * 16 + (f % 8) * 2,
// i.e. feature chunk c of all R rows is one contiguous R*16-byte run.  The same image is a
// canonical no-swizzle UMMA operand in both majors:
//   K-major  (rows = M or N, features = K): LBO = R*16 (next 8-wide K chunk), SBO = 128
//            (next 8-row group); K step s of 16 starts at + s * 2 * R * 16.
//   MN-major (rows = K, features = M or N): LBO = 128 (next 8-row K group), SBO = R*16
//            (next 8-wide M/N chunk); K step s of 16 starts at + s * 256.
// Threads that write consecutive rows of one chunk write consecutive 16-byte words, so the
// staging stores are free of bank conflicts.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace b200dem {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, no swizzle, version 1 (sm_100).  Fields (bits): start
// address >> 4 [0,14), leading byte offset >> 4 [16,30), stride byte offset >> 4 [32,46),
// version [46,48), base offset [49,52), LBO mode [52], layout type [61,64) (0 = none).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of tcgen05.mma.kind::f16 with BF16 A and B and an F32
// accumulator: D format [4,6) = 1, A format [7,10) = 1, B format [10,13) = 1, A major [15],
// B major [16] (0 = K-major, 1 = MN-major), N >> 3 [17,23), M >> 4 [24,29).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Row-tile descriptors (see the file comment).  R = rows of the staged block.
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t base, int R, int kstep) {
    return sdesc(base + (uint32_t)(kstep * 2 * R * 16), (uint32_t)(R * 16), 128u);
}
__device__ __forceinline__ uint64_t mnmajor_desc(uint32_t base, int R, int kstep) {
    return sdesc(base + (uint32_t)(kstep * 256), 128u, (uint32_t)(R * 16));
}

// Descriptor of a K-major operand block in the 128-byte swizzle layout that a tiled tensor copy
// with CU_TENSOR_MAP_SWIZZLE_128B writes: rows of 128 bytes (64 BF16 features), the 16-byte
// chunks of row r at chunk position c ^ (r % 8), 8-row groups 1,024 bytes apart (SBO); the block
// starts on a 1,024-byte boundary.  Layout type [61,64) = 2 (128-byte swizzle); the leading byte
// offset is not used by this layout (16 bytes).  The K step s (16 features, 32 bytes) inside the
// 128-byte row starts at + 32 s: the swizzle is applied to the address bits, so the same rows
// are read.
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// ---- TMEM allocation (one full warp; power-of-two column count >= 32) ----
__device__ __forceinline__ void tmem_alloc(uint32_t *smem_dst, int ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_dst)),
                 "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// ---- MMA: D[tmem] (+)= A[smem] * B[smem]; issued by one thread ----
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;   // no output lane disabled
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
}

// The same with A in tensor memory (rows = TMEM lanes, two BF16 features per 32-bit column,
// the lower-indexed feature in the low half).
__device__ __forceinline__ void mma_bf16_tmem_a(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                                uint32_t accumulate) {
    const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
}

// Arrive once on the mbarrier when every MMA issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity.  Returns false after `limit` polls
// (each try_wait itself suspends for a bounded, implementation-defined time).
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, int limit = 1 << 22) {
    for (int k = 0; k < limit; ++k)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

// ---- TMEM -> registers: this warp's 32 lanes, 16 consecutive 32-bit columns ----
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 consecutive 32-bit columns of this warp's lanes; no wait (issue several, then one wait).
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t r[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

// Registers -> this warp's 32 lanes, 16 consecutive 32-bit columns; tmem_wait_st before the
// values are read by an MMA (then the tcgen05 fences around the thread barrier).
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t r[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// ---- tiled tensor copies (TMA), global -> shared, completing on an mbarrier ----
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
                 : "memory");
}
// Box at element coordinates (x, y) of a 2-D tensor map (a kernel parameter) into dst; x times
// the element size is a multiple of 16 bytes.  No multicast.
__device__ __forceinline__ void tma_load_2d(void *dst, const void *tmap, int x, int y, uint64_t *mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(mbar))
        : "memory");
}

// TMEM address of (lane = 32 * (warp % 4), column col) for this warp's quarter.
__device__ __forceinline__ uint32_t tmem_warp_addr(uint32_t base, int col) {
    const uint32_t q = (threadIdx.x >> 5) & 3u;
    return base + ((q * 32u) << 16) + (uint32_t)col;
}

// ---- staging: 16-byte chunk (row, chunk c) of a row tile with R rows ----
__device__ __forceinline__ uint32_t tile_off(int R, int row, int c) { return (uint32_t)(c * R * 16 + row * 16); }

__device__ __forceinline__ uint4 pack8(const float v[8]) {
    uint4 u;
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 c = __floats2bfloat162_rn(v[4], v[5]), d = __floats2bfloat162_rn(v[6], v[7]);
    u.x = *reinterpret_cast<uint32_t *>(&a);
    u.y = *reinterpret_cast<uint32_t *>(&b);
    u.z = *reinterpret_cast<uint32_t *>(&c);
    u.w = *reinterpret_cast<uint32_t *>(&d);
    return u;
}
__device__ __forceinline__ void unpack8(uint4 u, float v[8]) {
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
    for (int k = 0; k < 4; ++k) {
        __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162 *>(&w[k]);
        const float2 f = __bfloat1622float2(h);
        v[2 * k] = f.x;
        v[2 * k + 1] = f.y;
    }
}

}  // namespace tc
}  // namespace b200dem
