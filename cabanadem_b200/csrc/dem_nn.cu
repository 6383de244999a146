// dem_nn.cu -- dense layers of the learned surrogate on the 5th-generation tensor cores.
//
// Every dense block of the message-passing network is a two-layer perceptron over rows
// (edges or particles):  y = W2 relu(W1 x + b1) + b2 (+ residual), hidden width 128,
// BF16 operands, FP32 accumulation in TMEM.  Three kernels cover training and inference:
//
//   k_mlp_fwd    gather the input row tile (up to three sources, e.g. [e_ij, h_i, h_j]),
//                GEMM1 -> bias + ReLU -> GEMM2 -> bias (+ residual); the hidden tile never
//                leaves shared memory/TMEM (saved to HBM only when training).
//   k_mlp_bwd    dH = dY W2^T, dZ = dH * [h > 0], dX = dZ W1^T (input gradient, split into
//                128-wide N chunks).
//   k_mlp_wgrad  dW1^T = dZ^T X, dW2^T = dY^T H (or dW2 = H^T dY for a 16-wide output) and
//                the bias sums, accumulated in TMEM over each CTA's row tiles; per-CTA
//                partials are then summed in a fixed order (k_wgrad_reduce), so the
//                gradients are deterministic.
//
// One CTA of 128 threads per SM (persistent over row tiles): thread t owns tile row t, which
// is TMEM lane t of the M = 128 accumulators.  One elected thread issues tcgen05.mma and
// commits to an mbarrier; every wait is bounded and a timeout raises the context's error
// word instead of hanging.
#include <cuda_bf16.h>
#include <cstdint>

#include "b200dem.h"
#include "dem_internal.cuh"
#include "nn_tc.cuh"

namespace b200dem {
namespace {

using bf16 = __nv_bfloat16;
constexpr int kRows = 128;      // rows per tile (= MMA M)
constexpr int kHidden = 128;    // hidden width
constexpr int kThreads = 128;

struct RowSrc {
    const bf16 *p;
    const int *idx;
    int width;   // features taken from this source (multiple of 8)
};

struct MlpW {
    const bf16 *w1t, *w1, *w2t, *w2;
    const float *b1, *b2;
};

// 16-byte chunk `kc` (features 8kc..8kc+7) of input row `grow` of the concatenated sources.
__device__ __forceinline__ uint4 src_chunk(const RowSrc *src, int nsrc, long grow, int kc) {
    int f = kc * 8;
    for (int s = 0; s < nsrc; ++s) {
        const int w = src[s].width;
        if (f < w) {
            const long r = src[s].idx ? (long)src[s].idx[grow] : grow;
            return *reinterpret_cast<const uint4 *>(src[s].p + r * w + f);
        }
        f -= w;
    }
    return make_uint4(0, 0, 0, 0);
}

// Stage rows [row0, row0 + kRows) (zero past `rows`) of the concatenated sources, C chunks
// per row, into a row tile of 128 rows.  Eight consecutive threads take eight consecutive
// rows of one chunk (bank-conflict-free 128-byte runs in shared memory).
__device__ __forceinline__ void stage_gather(unsigned char *tile, const RowSrc *src, int nsrc, int C, long row0,
                                             long rows) {
    const int G = C < 4 ? C : 4;
    for (int q = threadIdx.x; q < kRows * C; q += blockDim.x) {
        const int i = q & 7;
        const int g = (q >> 3) % G;
        const int rest = (q >> 3) / G;
        const int row = (rest % (kRows / 8)) * 8 + i;
        const int kc = (rest / (kRows / 8)) * G + g;
        const long grow = row0 + row;
        const uint4 v = grow < rows ? src_chunk(src, nsrc, grow, kc) : make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4 *>(tile + tc::tile_off(kRows, row, kc)) = v;
    }
}

// Stage a dense row-major block [R rows][F features] (row stride F) into a row tile of R rows.
__device__ __forceinline__ void stage_dense(unsigned char *tile, const bf16 *g, int R, int F, long row0, long rows) {
    const int C = F / 8;
    for (int q = threadIdx.x; q < R * C; q += blockDim.x) {
        const int row = q % R, kc = q / R;
        const long grow = row0 + row;
        const uint4 v = grow < rows ? *reinterpret_cast<const uint4 *>(g + grow * F + kc * 8) : make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4 *>(tile + tc::tile_off(R, row, kc)) = v;
    }
}

// Thread t reads 16 accumulator columns [col, col + 16) of its TMEM lane.
__device__ __forceinline__ void acc16(uint32_t tm, int col, float v[16]) {
    tc::tmem_ld16(tc::tmem_warp_addr(tm, col), v);
    tc::tmem_wait_ld();
}

// Shared-memory prologue of every kernel: mbarrier, TMEM allocation (warp 0).
__device__ __forceinline__ uint32_t tc_setup(uint64_t *mbar, uint32_t *tslot, int ncols) {
    if (threadIdx.x == 0) tc::mbar_init(mbar, 1);
    if (threadIdx.x < 32) {
        tc::tmem_alloc(tslot, ncols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    return *tslot;
}

__device__ __forceinline__ void tc_teardown(uint32_t tm, int ncols, bool ok, int *err) {
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tm, ncols);
    }
    if (!ok && threadIdx.x == 0 && err) atomicOr(err, DEM_ERR_TIMEOUT);
}

// All threads wait for the MMA batch committed last; uniform result across the block.
__device__ __forceinline__ bool mma_wait(uint64_t *mbar, uint32_t &phase) {
    const bool ok = tc::mbar_wait(mbar, phase);
    phase ^= 1u;
    const bool all = __syncthreads_and(ok) != 0;
    tc::fence_after_sync();
    return all;
}

// ------------------------------------------------------------------------------------
// forward
// ------------------------------------------------------------------------------------
struct FwdArgs {
    long rows;
    RowSrc src[3];
    int nsrc;
    MlpW w;
    const bf16 *resid;   // [rows][NOUT] or null
    bf16 *out;           // [rows][NOUT] or null
    float *out_f32;      // [rows][NOUT] or null
    bf16 *h1;            // [rows][128] or null
    int *err;
};

template <int KIN, int NOUT>
constexpr size_t fwd_smem() {
    return (size_t)kHidden * KIN * 2 + (size_t)NOUT * kHidden * 2 + (size_t)kRows * (KIN > kHidden ? KIN : kHidden) * 2 + 64;
}

template <int KIN, int NOUT>
__global__ void __launch_bounds__(kThreads, 1) k_mlp_fwd(FwdArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr int KA = KIN > kHidden ? KIN : kHidden;
    unsigned char *sW1 = smem;                                // W1^T: 128 rows x KIN
    unsigned char *sW2 = sW1 + (size_t)kHidden * KIN * 2;     // W2^T: NOUT rows x 128
    unsigned char *sA = sW2 + (size_t)NOUT * kHidden * 2;     // input tile, then hidden tile
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sA + (size_t)kRows * KA * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int t = threadIdx.x;

    stage_dense(sW1, a.w.w1t, kHidden, KIN, 0, kHidden);
    stage_dense(sW2, a.w.w2t, NOUT, kHidden, 0, NOUT);
    const uint32_t tm = tc_setup(mbar, tslot, 128);
    const uint32_t aW1 = tc::smem_u32(sW1), aW2 = tc::smem_u32(sW2), aA = tc::smem_u32(sA);
    constexpr uint32_t id1 = tc::idesc_bf16(kRows, kHidden, false, false);
    constexpr uint32_t id2 = tc::idesc_bf16(kRows, NOUT, false, false);
    uint32_t phase = 0;
    bool ok = true;
    const long ntiles = (a.rows + kRows - 1) / kRows;
    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long row0 = tile * kRows;
        const long grow = row0 + t;
        stage_gather(sA, a.src, a.nsrc, KIN / 8, row0, a.rows);
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (t == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < KIN / 16; ++ks)
                tc::mma_bf16(tm, tc::kmajor_desc(aA, kRows, ks), tc::kmajor_desc(aW1, kHidden, ks), id1, ks > 0);
            tc::mma_commit(mbar);
        }
        ok = mma_wait(mbar, phase);
        if (!ok) break;
        // hidden = relu(acc + b1) -> bf16 tile (A operand of GEMM2), optionally saved
        for (int c = 0; c < kHidden / 16; ++c) {
            float v[16];
            acc16(tm, c * 16, v);
            for (int k = 0; k < 16; ++k) v[k] = fmaxf(v[k] + a.w.b1[c * 16 + k], 0.f);
            const uint4 lo = tc::pack8(v), hi = tc::pack8(v + 8);
            *reinterpret_cast<uint4 *>(sA + tc::tile_off(kRows, t, 2 * c)) = lo;
            *reinterpret_cast<uint4 *>(sA + tc::tile_off(kRows, t, 2 * c + 1)) = hi;
            if (a.h1 && grow < a.rows) {
                uint4 *dst = reinterpret_cast<uint4 *>(a.h1 + grow * kHidden + c * 16);
                dst[0] = lo;
                dst[1] = hi;
            }
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (t == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < kHidden / 16; ++ks)
                tc::mma_bf16(tm, tc::kmajor_desc(aA, kRows, ks), tc::kmajor_desc(aW2, NOUT, ks), id2, ks > 0);
            tc::mma_commit(mbar);
        }
        ok = mma_wait(mbar, phase);
        if (!ok) break;
        for (int c = 0; c < NOUT / 16; ++c) {
            float v[16];
            acc16(tm, c * 16, v);
            if (grow < a.rows) {
                for (int k = 0; k < 16; ++k) v[k] += a.w.b2[c * 16 + k];
                if (a.resid) {
                    float r[8];
                    const uint4 *src = reinterpret_cast<const uint4 *>(a.resid + grow * NOUT + c * 16);
                    tc::unpack8(src[0], r);
                    for (int k = 0; k < 8; ++k) v[k] += r[k];
                    tc::unpack8(src[1], r);
                    for (int k = 0; k < 8; ++k) v[8 + k] += r[k];
                }
                if (a.out) {
                    uint4 *dst = reinterpret_cast<uint4 *>(a.out + grow * NOUT + c * 16);
                    dst[0] = tc::pack8(v);
                    dst[1] = tc::pack8(v + 8);
                }
                if (a.out_f32) {
                    float4 *dst = reinterpret_cast<float4 *>(a.out_f32 + grow * NOUT + c * 16);
                    for (int k = 0; k < 4; ++k) dst[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();   // TMEM and the A tile are reused by the next tile
    }
    tc_teardown(tm, 128, ok, a.err);
}

// ------------------------------------------------------------------------------------
// backward: input gradient
// ------------------------------------------------------------------------------------
struct BwdArgs {
    long rows;
    MlpW w;
    const bf16 *dy;   // [rows][NOUT]
    const bf16 *h1;   // [rows][128]
    bf16 *dz1;        // [rows][128]
    float *dx;        // [rows][KIN] or null
    int *err;
};

template <int KIN, int NOUT>
constexpr size_t bwd_smem() {
    return (size_t)kHidden * NOUT * 2 + (size_t)KIN * kHidden * 2 + (size_t)kRows * NOUT * 2 + (size_t)kRows * kHidden * 2 + 64;
}

template <int KIN, int NOUT>
__global__ void __launch_bounds__(kThreads, 1) k_mlp_bwd(BwdArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *sW2 = smem;                                  // W2: 128 rows (in) x NOUT
    unsigned char *sW1 = sW2 + (size_t)kHidden * NOUT * 2;      // W1: KIN rows (in) x 128
    unsigned char *sY = sW1 + (size_t)KIN * kHidden * 2;        // dY tile: 128 x NOUT
    unsigned char *sZ = sY + (size_t)kRows * NOUT * 2;          // dZ tile: 128 x 128
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sZ + (size_t)kRows * kHidden * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int t = threadIdx.x;
    const bool want_dx = a.dx != nullptr;

    stage_dense(sW2, a.w.w2, kHidden, NOUT, 0, kHidden);
    if (want_dx) stage_dense(sW1, a.w.w1, KIN, kHidden, 0, KIN);
    const uint32_t tm = tc_setup(mbar, tslot, 512);
    const uint32_t aW1 = tc::smem_u32(sW1), aW2 = tc::smem_u32(sW2), aY = tc::smem_u32(sY), aZ = tc::smem_u32(sZ);
    constexpr uint32_t id1 = tc::idesc_bf16(kRows, kHidden, false, false);
    constexpr int NX = KIN < 128 ? KIN : 128;   // N of one input-gradient chunk
    constexpr uint32_t idx = tc::idesc_bf16(kRows, NX, false, false);
    uint32_t phase = 0;
    bool ok = true;
    const long ntiles = (a.rows + kRows - 1) / kRows;
    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long row0 = tile * kRows;
        const long grow = row0 + t;
        stage_dense(sY, a.dy, kRows, NOUT, row0, a.rows);
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (t == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < NOUT / 16; ++ks)
                tc::mma_bf16(tm, tc::kmajor_desc(aY, kRows, ks), tc::kmajor_desc(aW2, kHidden, ks), id1, ks > 0);
            tc::mma_commit(mbar);
        }
        ok = mma_wait(mbar, phase);
        if (!ok) break;
        for (int c = 0; c < kHidden / 16; ++c) {
            float v[16], h[8];
            acc16(tm, c * 16, v);
            if (grow < a.rows) {
                const uint4 *hs = reinterpret_cast<const uint4 *>(a.h1 + grow * kHidden + c * 16);
                tc::unpack8(hs[0], h);
                for (int k = 0; k < 8; ++k) v[k] = h[k] > 0.f ? v[k] : 0.f;
                tc::unpack8(hs[1], h);
                for (int k = 0; k < 8; ++k) v[8 + k] = h[k] > 0.f ? v[8 + k] : 0.f;
            } else {
                for (int k = 0; k < 16; ++k) v[k] = 0.f;
            }
            const uint4 lo = tc::pack8(v), hi = tc::pack8(v + 8);
            *reinterpret_cast<uint4 *>(sZ + tc::tile_off(kRows, t, 2 * c)) = lo;
            *reinterpret_cast<uint4 *>(sZ + tc::tile_off(kRows, t, 2 * c + 1)) = hi;
            if (grow < a.rows) {
                uint4 *dst = reinterpret_cast<uint4 *>(a.dz1 + grow * kHidden + c * 16);
                dst[0] = lo;
                dst[1] = hi;
            }
        }
        if (want_dx) {
            tc::fence_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            if (t == 0) {
                tc::fence_after_sync();
                for (int j = 0; j < KIN / NX; ++j)   // N chunk j: input features [j*NX, j*NX + NX)
                    for (int ks = 0; ks < kHidden / 16; ++ks)
                        tc::mma_bf16(tm + kHidden + j * NX, tc::kmajor_desc(aZ, kRows, ks),
                                     tc::kmajor_desc(aW1 + (uint32_t)(j * NX * 16), KIN, ks), idx, ks > 0);
                tc::mma_commit(mbar);
            }
            ok = mma_wait(mbar, phase);
            if (!ok) break;
            for (int c = 0; c < KIN / 16; ++c) {
                float v[16];
                acc16(tm, kHidden + c * 16, v);
                if (grow < a.rows) {
                    float4 *dst = reinterpret_cast<float4 *>(a.dx + grow * KIN + c * 16);
                    for (int k = 0; k < 4; ++k) dst[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
    }
    tc_teardown(tm, 512, ok, a.err);
}

// ------------------------------------------------------------------------------------
// backward: weight and bias gradients (per-CTA partials)
// ------------------------------------------------------------------------------------
struct WgradArgs {
    long rows;
    RowSrc src[3];
    int nsrc;
    const bf16 *dz1;   // [rows][128]
    const bf16 *h1;    // [rows][128]
    const bf16 *dy;    // [rows][NOUT]
    float *part;       // [gridDim.x][128][KIN + NW2 + 2]: dW1^T | dW2 block | db1 | db2
    int *err;
};

template <int NOUT>
__host__ __device__ constexpr int wgrad_w2_cols() { return NOUT == kHidden ? kHidden : NOUT; }
template <int KIN, int NOUT>
__host__ __device__ constexpr int wgrad_cols() { return KIN + wgrad_w2_cols<NOUT>() + 2; }
template <int KIN, int NOUT>
__host__ __device__ constexpr int wgrad_tmem_cols() {
    return (KIN + wgrad_w2_cols<NOUT>()) <= 256 ? 256 : 512;
}
template <int KIN, int NOUT>
constexpr size_t wgrad_smem() {
    return (size_t)kRows * kHidden * 2 * 2 + (size_t)kRows * KIN * 2 + (size_t)kRows * NOUT * 2 + 64;
}

template <int KIN, int NOUT>
__global__ void __launch_bounds__(kThreads, 1) k_mlp_wgrad(WgradArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *sZ = smem;                                   // dZ tile: 128 rows x 128
    unsigned char *sH = sZ + (size_t)kRows * kHidden * 2;       // H tile: 128 x 128
    unsigned char *sX = sH + (size_t)kRows * kHidden * 2;       // X tile: 128 x KIN
    unsigned char *sY = sX + (size_t)kRows * KIN * 2;           // dY tile: 128 x NOUT
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sY + (size_t)kRows * NOUT * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int t = threadIdx.x;
    constexpr int TC = wgrad_tmem_cols<KIN, NOUT>();
    const uint32_t tm = tc_setup(mbar, tslot, TC);
    const uint32_t aZ = tc::smem_u32(sZ), aH = tc::smem_u32(sH), aX = tc::smem_u32(sX), aY = tc::smem_u32(sY);
    constexpr int NX = KIN < 128 ? KIN : 128;
    constexpr uint32_t idx = tc::idesc_bf16(kRows, NX, true, true);
    constexpr uint32_t id2 = tc::idesc_bf16(kRows, NOUT == kHidden ? kHidden : NOUT, true, true);
    uint32_t phase = 0;
    bool ok = true;
    float db1 = 0.f, db2 = 0.f;   // thread t: bias sums of hidden unit t and output t
    bool first = true;
    const long ntiles = (a.rows + kRows - 1) / kRows;
    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long row0 = tile * kRows;
        stage_dense(sZ, a.dz1, kRows, kHidden, row0, a.rows);
        stage_dense(sH, a.h1, kRows, kHidden, row0, a.rows);
        stage_gather(sX, a.src, a.nsrc, KIN / 8, row0, a.rows);
        stage_dense(sY, a.dy, kRows, NOUT, row0, a.rows);
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (t == 0) {
            tc::fence_after_sync();
            for (int j = 0; j < KIN / NX; ++j)   // dW1^T[:, j*NX .. ] += dZ^T X_j
                for (int ks = 0; ks < kRows / 16; ++ks)
                    tc::mma_bf16(tm + j * NX, tc::mnmajor_desc(aZ, kRows, ks),
                                 tc::mnmajor_desc(aX + (uint32_t)(j * (NX / 8) * kRows * 16), kRows, ks), idx,
                                 (!first || ks > 0) ? 1u : 0u);
            for (int ks = 0; ks < kRows / 16; ++ks) {
                if (NOUT == kHidden)   // dW2^T += dY^T H
                    tc::mma_bf16(tm + KIN, tc::mnmajor_desc(aY, kRows, ks), tc::mnmajor_desc(aH, kRows, ks), id2,
                                 (!first || ks > 0) ? 1u : 0u);
                else                   // dW2 += H^T dY (M = 128 hidden, N = NOUT)
                    tc::mma_bf16(tm + KIN, tc::mnmajor_desc(aH, kRows, ks), tc::mnmajor_desc(aY, kRows, ks), id2,
                                 (!first || ks > 0) ? 1u : 0u);
            }
            tc::mma_commit(mbar);
        }
        // bias sums from the staged tiles while the tensor core runs (fixed row order)
        for (int r = 0; r < kRows; ++r) {
            db1 += __bfloat162float(*reinterpret_cast<const bf16 *>(sZ + tc::tile_off(kRows, r, t >> 3) + (t & 7) * 2));
            if (t < NOUT)
                db2 += __bfloat162float(*reinterpret_cast<const bf16 *>(sY + tc::tile_off(kRows, r, t >> 3) + (t & 7) * 2));
        }
        ok = mma_wait(mbar, phase);
        first = false;
        tc::fence_before_sync();
        __syncthreads();
    }
    constexpr int NC = wgrad_cols<KIN, NOUT>();
    float *dst = a.part + ((long)blockIdx.x * kRows + t) * NC;
    if (ok && !first) {
        tc::fence_after_sync();
        for (int c = 0; c < (KIN + wgrad_w2_cols<NOUT>()) / 16; ++c) {
            float v[16];
            acc16(tm, c * 16, v);
            for (int k = 0; k < 16; ++k) dst[c * 16 + k] = v[k];
        }
    } else {
        for (int c = 0; c < NC - 2; ++c) dst[c] = 0.f;
    }
    dst[NC - 2] = db1;
    dst[NC - 1] = t < NOUT ? db2 : 0.f;
    tc_teardown(tm, TC, ok, a.err);
}

// Sum the per-CTA partials in block order and add them to the gradient buffers:
// g_w1t [128][KIN], g_b1 [128], g_w2t [NOUT][128], g_b2 [NOUT].
__global__ void k_wgrad_reduce(const float *part, int nblocks, int kin, int nout, float *g_w1t, float *g_b1,
                               float *g_w2t, float *g_b2) {
    const int nw2 = nout == kHidden ? kHidden : nout;
    const int nc = kin + nw2 + 2;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kRows * nc; e += gridDim.x * blockDim.x) {
        const int r = e / nc, c = e % nc;
        float s = 0.f;
        for (int b = 0; b < nblocks; ++b) s += part[((long)b * kRows + r) * nc + c];
        if (c < kin) g_w1t[r * kin + c] += s;
        else if (c < kin + nw2) {
            const int cc = c - kin;
            if (nout == kHidden) g_w2t[r * kHidden + cc] += s;   // row r = output unit
            else g_w2t[cc * kHidden + r] += s;                   // row r = hidden unit
        } else if (c == kin + nw2) g_b1[r] += s;
        else if (r < nout) g_b2[r] += s;
    }
}

// Dynamic shared memory is raised so that the CTAs one SM can hold never ask for more TMEM
// columns than its 512 (an allocation that cannot be met would wait for another CTA).
// 228 KB of shared memory per SM: > 114 KB leaves one CTA, > 76 KB two, > 57 KB three.
template <typename K, typename A>
int launch_tc(K kernel, size_t smem, int tmem_cols, long rows, A args, cudaStream_t s, int max_blocks = 148) {
    if (rows <= 0) return DEM_OK;
    const size_t floor_bytes = tmem_cols >= 512 ? 116 * 1024 : (tmem_cols >= 256 ? 80 * 1024 : 0);
    if (smem < floor_bytes) smem = floor_bytes;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return DEM_ERR_CUDA;
    const long ntiles = (rows + kRows - 1) / kRows;
    const int grid = (int)(ntiles < max_blocks ? ntiles : max_blocks);
    kernel<<<grid, kThreads, smem, s>>>(args);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

}  // namespace

// ---- dispatch over the (KIN, NOUT) shapes the surrogate uses ----
#define B200_NN_SHAPES(X) X(16, 128) X(128, 128) X(256, 128) X(384, 128) X(128, 16)

int nn_mlp_forward(const dem_nn_mlp &m, long rows, const dem_nn_rows *src, int nsrc, const void *resid, void *out,
                   float *out_f32, void *h1, int *err, cudaStream_t s) {
    FwdArgs a{};
    a.rows = rows;
    a.nsrc = nsrc;
    int kin = 0;
    for (int k = 0; k < nsrc && k < 3; ++k) {
        a.src[k] = RowSrc{(const bf16 *)src[k].data, src[k].index, src[k].width};
        kin += src[k].width;
    }
    if (kin != m.kin) return DEM_ERR_INVALID;
    a.w = MlpW{(const bf16 *)m.w1t, (const bf16 *)m.w1, (const bf16 *)m.w2t, (const bf16 *)m.w2, m.b1, m.b2};
    a.resid = (const bf16 *)resid;
    a.out = (bf16 *)out;
    a.out_f32 = out_f32;
    a.h1 = (bf16 *)h1;
    a.err = err;
#define X(KI, NO) \
    if (m.kin == KI && m.nout == NO) return launch_tc(k_mlp_fwd<KI, NO>, fwd_smem<KI, NO>(), 128, rows, a, s);
    B200_NN_SHAPES(X)
#undef X
    return DEM_ERR_UNSUPPORTED;
}

int nn_mlp_backward(const dem_nn_mlp &m, long rows, const dem_nn_rows *src, int nsrc, const void *dy, const void *h1,
                    void *dz1, float *dx, float *g_w1t, float *g_b1, float *g_w2t, float *g_b2, float *part,
                    int *err, cudaStream_t s) {
    BwdArgs b{};
    b.rows = rows;
    b.w = MlpW{(const bf16 *)m.w1t, (const bf16 *)m.w1, (const bf16 *)m.w2t, (const bf16 *)m.w2, m.b1, m.b2};
    b.dy = (const bf16 *)dy;
    b.h1 = (const bf16 *)h1;
    b.dz1 = (bf16 *)dz1;
    b.dx = dx;
    b.err = err;
    WgradArgs g{};
    g.rows = rows;
    g.nsrc = nsrc;
    int kin = 0;
    for (int k = 0; k < nsrc && k < 3; ++k) {
        g.src[k] = RowSrc{(const bf16 *)src[k].data, src[k].index, src[k].width};
        kin += src[k].width;
    }
    if (kin != m.kin) return DEM_ERR_INVALID;
    g.dz1 = (const bf16 *)dz1;
    g.h1 = (const bf16 *)h1;
    g.dy = (const bf16 *)dy;
    g.part = part;
    g.err = err;
    const long ntiles = (rows + kRows - 1) / kRows;
    const int nblocks = (int)(ntiles < 148 ? ntiles : 148);
    int st = DEM_ERR_UNSUPPORTED;
#define X(KI, NO)                                                                             \
    if (m.kin == KI && m.nout == NO) {                                                        \
        st = launch_tc(k_mlp_bwd<KI, NO>, bwd_smem<KI, NO>(), 512, rows, b, s);                    \
        if (st == DEM_OK) st = launch_tc(k_mlp_wgrad<KI, NO>, wgrad_smem<KI, NO>(), wgrad_tmem_cols<KI, NO>(), rows, g, s); \
    }
    B200_NN_SHAPES(X)
#undef X
    if (st != DEM_OK || rows <= 0) return st;
    k_wgrad_reduce<<<64, 256, 0, s>>>(part, nblocks, m.kin, m.nout, g_w1t, g_b1, g_w2t, g_b2);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

// Scratch floats the per-CTA weight-gradient partials of one backward call need.
long nn_wgrad_scratch(int kin, int nout) {
    const int nw2 = nout == kHidden ? kHidden : nout;
    return 148L * kRows * (kin + nw2 + 2);
}

}  // namespace b200dem
