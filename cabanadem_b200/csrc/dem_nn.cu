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
#include <cuda.h>   // CUtensorMap (encoded on the host through the driver entry point)
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
constexpr int kFwdThreads = 256;   // forward kernels: warps w and w + 4 split a TMEM lane quarter's columns

struct RowSrc {
    const bf16 *p;
    const int *idx;
    int width;   // features taken from this source (multiple of 8)
};

struct MlpW {
    const bf16 *w1t, *w1, *w2t, *w2;
    const float *b1, *b2;
};

// ---- asynchronous staging (cp.async: every chunk copy of a tile in flight at once) ----
__device__ __forceinline__ void cp16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc::smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Row indices of the tile's rows for the gathered sources: s_idx[s][row] (one round trip).
__device__ __forceinline__ void load_row_index(int *s_idx, const RowSrc *src, int nsrc, long row0, long rows) {
    const int t = threadIdx.x;
    if (t < kRows) {
        const long grow = row0 + t;
        for (int s = 0; s < nsrc; ++s)
            s_idx[s * kRows + t] = src[s].idx ? (grow < rows ? src[s].idx[grow] : 0) : (int)(grow < rows ? grow : 0);
    }
}

// Queue the copies of rows [row0, row0 + kRows) of the concatenated sources (C chunks of 8
// features per row) into a row tile of 128 rows; rows past `rows` are zero-filled.  Eight
// consecutive threads take eight consecutive rows of one chunk (conflict-free 128-byte runs
// in shared memory).  s_idx must hold the tile's row indices (load_row_index + barrier).
__device__ __forceinline__ void stage_gather(unsigned char *tile, const RowSrc *src, int nsrc, int C, long row0,
                                             long rows, const int *s_idx) {
    const int G = C < 4 ? C : 4;
    for (int q = threadIdx.x; q < kRows * C; q += blockDim.x) {
        const int i = q & 7;
        const int g = (q >> 3) % G;
        const int rest = (q >> 3) / G;
        const int row = (rest % (kRows / 8)) * 8 + i;
        const int kc = (rest / (kRows / 8)) * G + g;
        unsigned char *dst = tile + tc::tile_off(kRows, row, kc);
        if (row0 + row < rows) {
            int f = kc * 8, s = 0;
            while (s < nsrc - 1 && f >= src[s].width) {
                f -= src[s].width;
                ++s;
            }
            cp16(dst, src[s].p + (long)s_idx[s * kRows + row] * src[s].width + f);
        } else {
            *reinterpret_cast<uint4 *>(dst) = make_uint4(0, 0, 0, 0);
        }
    }
}

// Queue the copies of a dense row-major block [R rows][F features] (row stride F) into a row
// tile of R rows; rows past `rows` are zero-filled.
__device__ __forceinline__ void stage_dense(unsigned char *tile, const bf16 *g, int R, int F, long row0, long rows) {
    const int C = F / 8;
    for (int q = threadIdx.x; q < R * C; q += blockDim.x) {
        const int row = q % R, kc = q / R;
        unsigned char *dst = tile + tc::tile_off(R, row, kc);
        if (row0 + row < rows) cp16(dst, g + (row0 + row) * F + kc * 8);
        else *reinterpret_cast<uint4 *>(dst) = make_uint4(0, 0, 0, 0);
    }
}

// Completes this thread's queued copies and publishes the tiles to the tensor core.
__device__ __forceinline__ void stage_done() {
    cp_wait_all();
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
}

// Row-major output tile in shared memory (128 rows x 256 bytes), 16-byte chunks XOR-swizzled
// by the row so that thread t writing its row and 16 threads reading one row are both free of
// bank conflicts; copy_out then writes whole 256-byte rows (coalesced).
__device__ __forceinline__ void out_put(unsigned char *tile, int row, int chunk, uint4 v) {
    *reinterpret_cast<uint4 *>(tile + row * 256 + ((chunk ^ (row & 15)) << 4)) = v;
}
__device__ __forceinline__ void copy_out(const unsigned char *tile, bf16 *g, long row0, long rows) {
    for (int q = threadIdx.x; q < kRows * 16; q += blockDim.x) {
        const int row = q >> 4, chunk = q & 15;
        if (row0 + row < rows)
            *reinterpret_cast<uint4 *>(g + (row0 + row) * kHidden + chunk * 8) =
                *reinterpret_cast<const uint4 *>(tile + row * 256 + ((chunk ^ (row & 15)) << 4));
    }
}

// Thread t reads 16 accumulator columns [col, col + 16) of its TMEM lane.
__device__ __forceinline__ void acc16(uint32_t tm, int col, float v[16]) {
    tc::tmem_ld16(tc::tmem_warp_addr(tm, col), v);
    tc::tmem_wait_ld();
}

// 32 accumulator columns [col, col + 32) of thread t's lane.
__device__ __forceinline__ void acc32(uint32_t tm, int col, float v[32]) {
    uint32_t r[32];
    tc::tmem_ld32_nowait(tc::tmem_warp_addr(tm, col), r);
    tc::tmem_wait_ld();
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

// 64 accumulator columns [col, col + 64) of thread t's lane with one wait (two x32 loads).
__device__ __forceinline__ void acc64(uint32_t tm, int col, float v[64]) {
    uint32_t r[64];
    tc::tmem_ld32_nowait(tc::tmem_warp_addr(tm, col), r);
    tc::tmem_ld32_nowait(tc::tmem_warp_addr(tm, col + 32), r + 32);
    tc::tmem_wait_ld();
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] = __uint_as_float(r[k]);
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

// Bounded waits of the tensor-core kernels: polls of mbarrier.try_wait per wait, and a
// diagnostic switch under which the kernels issue no MMA and no commit (so every wait runs
// out with nothing in flight).  Process-wide per device; set by dem_nn_debug_waits.
__device__ int g_tc_wait_limit = 1 << 22;
__device__ int g_tc_drop_mma = 0;

// The elected thread's MMA issue and commit, skipped under the diagnostic switch.
__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    if (!g_tc_drop_mma) tc::mma_bf16(tmem_d, adesc, bdesc, idesc, accumulate);
}
__device__ __forceinline__ void mma_issue_tmem_a(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                                 uint32_t accumulate) {
    if (!g_tc_drop_mma) tc::mma_bf16_tmem_a(tmem_d, tmem_a, bdesc, idesc, accumulate);
}
__device__ __forceinline__ void mma_commit_issue(uint64_t *mbar) {
    if (!g_tc_drop_mma) tc::mma_commit(mbar);
}

// End of every kernel: free the block's TMEM.  When a wait gave up (ok false), the MMA batch
// of that wait may still be running and writing TMEM: the block first waits once more, with
// the same bound, for that batch's commit (parity `phase ^ 1`: mma_wait flipped it), so TMEM
// is freed after the batch completes.  If that wait gives up too, TMEM is freed anyway and the
// error word carries DEM_ERR_TIMEOUT; the host learns of it from dem_nn_status.
__device__ __forceinline__ void tc_teardown(uint32_t tm, int ncols, bool ok, int *err, uint64_t *mbar,
                                            uint32_t phase) {
    if (!ok) {
        if (threadIdx.x == 0) (void)tc::mbar_wait(mbar, phase ^ 1u, g_tc_wait_limit);
        __syncthreads();
    }
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
    const bool ok = tc::mbar_wait(mbar, phase, g_tc_wait_limit);
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
    int resid_src0;      // the residual is source 0 of the input (read from the staged tile)
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
__global__ void __launch_bounds__(kFwdThreads, 1) k_mlp_fwd(FwdArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int KA = KIN > kHidden ? KIN : kHidden;
    unsigned char *sW1 = smem;                                // W1^T: 128 rows x KIN
    unsigned char *sW2 = sW1 + (size_t)kHidden * KIN * 2;     // W2^T: NOUT rows x 128
    unsigned char *sA = sW2 + (size_t)NOUT * kHidden * 2;     // input tile, then hidden tile
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sA + (size_t)kRows * KA * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    __shared__ int s_idx[3 * kRows];
    __shared__ float s_b1[kHidden], s_b2[kHidden];
    const int tid = threadIdx.x;
    const int t = tid & (kRows - 1);   // tile row (TMEM lane) of this thread
    const int half = tid >> 7;         // column half [64 half, 64 half + 64) of the epilogues
    // the hidden tile goes behind source 0 when the input is wide enough, so that a residual
    // taken from source 0 is still in shared memory for the second epilogue
    constexpr int HC = KIN >= 2 * kHidden ? kHidden / 8 : 0;   // first chunk of the hidden tile
    const uint32_t aH = tc::smem_u32(sA) + (uint32_t)(HC * kRows * 16);
    unsigned char *sOut = sA + (size_t)HC * kRows * 16;        // output tile (hidden tile is spent)
    if (half == 0) s_b1[t] = a.w.b1[t];
    else if (t < NOUT) s_b2[t] = a.w.b2[t];

    stage_dense(sW1, a.w.w1t, kHidden, KIN, 0, kHidden);
    stage_dense(sW2, a.w.w2t, NOUT, kHidden, 0, NOUT);
    cp_wait_all();
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
        load_row_index(s_idx, a.src, a.nsrc, row0, a.rows);
        __syncthreads();
        stage_gather(sA, a.src, a.nsrc, KIN / 8, row0, a.rows, s_idx);
        stage_done();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < KIN / 16; ++ks)
                mma_issue(tm, tc::kmajor_desc(aA, kRows, ks), tc::kmajor_desc(aW1, kHidden, ks), id1, ks > 0);
            mma_commit_issue(mbar);
        }
        ok = mma_wait(mbar, phase);
        if (!ok) break;
        // hidden = relu(acc + b1) -> bf16 tile (A operand of GEMM2), optionally saved
        for (int c64 = half; c64 < kHidden / 64; c64 += 2) {
          float w[64];
          acc64(tm, c64 * 64, w);
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) {
            const int c = c64 * 4 + cc;
            float *v = w + 16 * cc;
            for (int k = 0; k < 16; ++k) v[k] = fmaxf(v[k] + s_b1[c * 16 + k], 0.f);
            const uint4 lo = tc::pack8(v), hi = tc::pack8(v + 8);
            *reinterpret_cast<uint4 *>(sA + tc::tile_off(kRows, t, HC + 2 * c)) = lo;
            *reinterpret_cast<uint4 *>(sA + tc::tile_off(kRows, t, HC + 2 * c + 1)) = hi;
            if (a.h1 && grow < a.rows) {
                uint4 *dst = reinterpret_cast<uint4 *>(a.h1 + grow * kHidden + c * 16);
                dst[0] = lo;
                dst[1] = hi;
            }
          }
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < kHidden / 16; ++ks)
                mma_issue(tm, tc::kmajor_desc(aH, kRows, ks), tc::kmajor_desc(aW2, NOUT, ks), id2, ks > 0);
            mma_commit_issue(mbar);
        }
        ok = mma_wait(mbar, phase);
        if (!ok) break;
        constexpr bool kStaged = NOUT == kHidden;   // bf16 rows written through the output tile
        constexpr int CB = NOUT >= 64 ? 64 : NOUT;   // columns per TMEM wait
        for (int c64 = half; c64 < NOUT / CB; c64 += 2) {
          float w[64];
          if (CB == 64) acc64(tm, c64 * 64, w);
          else acc16(tm, 0, w);
#pragma unroll
          for (int cc = 0; cc < CB / 16; ++cc) {
            const int c = c64 * (CB / 16) + cc;
            float *v = w + 16 * cc;
            if (grow < a.rows) {
                for (int k = 0; k < 16; ++k) v[k] += s_b2[c * 16 + k];
                if (a.resid) {
                    float r[8];
                    uint4 r0, r1;
                    if (HC > 0 && a.resid_src0) {   // source 0 is still staged in chunks [0, 16)
                        r0 = *reinterpret_cast<const uint4 *>(sA + tc::tile_off(kRows, t, 2 * c));
                        r1 = *reinterpret_cast<const uint4 *>(sA + tc::tile_off(kRows, t, 2 * c + 1));
                    } else {
                        const uint4 *src = reinterpret_cast<const uint4 *>(a.resid + grow * NOUT + c * 16);
                        r0 = src[0];
                        r1 = src[1];
                    }
                    tc::unpack8(r0, r);
                    for (int k = 0; k < 8; ++k) v[k] += r[k];
                    tc::unpack8(r1, r);
                    for (int k = 0; k < 8; ++k) v[8 + k] += r[k];
                }
                if (a.out && kStaged) {
                    out_put(sOut, t, 2 * c, tc::pack8(v));
                    out_put(sOut, t, 2 * c + 1, tc::pack8(v + 8));
                } else if (a.out) {
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
        }
        tc::fence_before_sync();
        __syncthreads();   // TMEM and the A tile are reused by the next tile
        if (a.out && kStaged) {
            copy_out(sOut, a.out, row0, a.rows);
            __syncthreads();
        }
    }
    tc_teardown(tm, 128, ok, a.err, mbar, phase);
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
    return (size_t)kHidden * NOUT * 2 + (size_t)KIN * kHidden * 2 + (size_t)kRows * NOUT * 2 +
           2 * (size_t)kRows * kHidden * 2 + 64;
}

template <int KIN, int NOUT>
__global__ void __launch_bounds__(kThreads, 1) k_mlp_bwd(BwdArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *sW2 = smem;                                  // W2: 128 rows (in) x NOUT
    unsigned char *sW1 = sW2 + (size_t)kHidden * NOUT * 2;      // W1: KIN rows (in) x 128
    unsigned char *sY = sW1 + (size_t)KIN * kHidden * 2;        // dY tile: 128 x NOUT
    unsigned char *sZ = sY + (size_t)kRows * NOUT * 2;          // dZ tile: 128 x 128
    unsigned char *sH = sZ + (size_t)kRows * kHidden * 2;       // saved hidden tile: 128 x 128
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sH + (size_t)kRows * kHidden * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int t = threadIdx.x;
    const bool want_dx = a.dx != nullptr;

    stage_dense(sW2, a.w.w2, kHidden, NOUT, 0, kHidden);
    if (want_dx) stage_dense(sW1, a.w.w1, KIN, kHidden, 0, KIN);
    cp_wait_all();
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
        stage_dense(sH, a.h1, kRows, kHidden, row0, a.rows);
        stage_done();
        if (t == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < NOUT / 16; ++ks)
                mma_issue(tm, tc::kmajor_desc(aY, kRows, ks), tc::kmajor_desc(aW2, kHidden, ks), id1, ks > 0);
            mma_commit_issue(mbar);
        }
        ok = mma_wait(mbar, phase);
        if (!ok) break;
        for (int c = 0; c < kHidden / 16; ++c) {
            float v[16], h[8];
            acc16(tm, c * 16, v);
            if (grow < a.rows) {
                tc::unpack8(*reinterpret_cast<const uint4 *>(sH + tc::tile_off(kRows, t, 2 * c)), h);
                for (int k = 0; k < 8; ++k) v[k] = h[k] > 0.f ? v[k] : 0.f;
                tc::unpack8(*reinterpret_cast<const uint4 *>(sH + tc::tile_off(kRows, t, 2 * c + 1)), h);
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
                        mma_issue(tm + kHidden + j * NX, tc::kmajor_desc(aZ, kRows, ks),
                                     tc::kmajor_desc(aW1 + (uint32_t)(j * NX * 16), KIN, ks), idx, ks > 0);
                mma_commit_issue(mbar);
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
    tc_teardown(tm, 512, ok, a.err, mbar, phase);
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
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *sZ = smem;                                   // dZ tile: 128 rows x 128
    unsigned char *sH = sZ + (size_t)kRows * kHidden * 2;       // H tile: 128 x 128
    unsigned char *sX = sH + (size_t)kRows * kHidden * 2;       // X tile: 128 x KIN
    unsigned char *sY = sX + (size_t)kRows * KIN * 2;           // dY tile: 128 x NOUT
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sY + (size_t)kRows * NOUT * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    __shared__ int s_idx[3 * kRows];
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
        load_row_index(s_idx, a.src, a.nsrc, row0, a.rows);
        __syncthreads();
        stage_dense(sZ, a.dz1, kRows, kHidden, row0, a.rows);
        stage_dense(sH, a.h1, kRows, kHidden, row0, a.rows);
        stage_gather(sX, a.src, a.nsrc, KIN / 8, row0, a.rows, s_idx);
        stage_dense(sY, a.dy, kRows, NOUT, row0, a.rows);
        stage_done();
        if (t == 0) {
            tc::fence_after_sync();
            for (int j = 0; j < KIN / NX; ++j)   // dW1^T[:, j*NX .. ] += dZ^T X_j
                for (int ks = 0; ks < kRows / 16; ++ks)
                    mma_issue(tm + j * NX, tc::mnmajor_desc(aZ, kRows, ks),
                                 tc::mnmajor_desc(aX + (uint32_t)(j * (NX / 8) * kRows * 16), kRows, ks), idx,
                                 (!first || ks > 0) ? 1u : 0u);
            for (int ks = 0; ks < kRows / 16; ++ks) {
                if (NOUT == kHidden)   // dW2^T += dY^T H
                    mma_issue(tm + KIN, tc::mnmajor_desc(aY, kRows, ks), tc::mnmajor_desc(aH, kRows, ks), id2,
                                 (!first || ks > 0) ? 1u : 0u);
                else                   // dW2 += H^T dY (M = 128 hidden, N = NOUT)
                    mma_issue(tm + KIN, tc::mnmajor_desc(aH, kRows, ks), tc::mnmajor_desc(aY, kRows, ks), id2,
                                 (!first || ks > 0) ? 1u : 0u);
            }
            mma_commit_issue(mbar);
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
    tc_teardown(tm, TC, ok, a.err, mbar, phase);
}

// Sum the per-CTA partials in block order and add them to the gradient buffers:
// g_w1t [128][KIN], g_b1 [128], g_w2t [NOUT][128], g_b2 [NOUT].
__global__ void k_wgrad_reduce(const float *part, int nblocks, int kin, int nout, float *g_w1t, int ld_w1, float *g_b1,
                               float *g_w2t, float *g_b2) {
    const int nw2 = nout == kHidden ? kHidden : nout;
    const int nc = kin + nw2 + 2;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kRows * nc; e += gridDim.x * blockDim.x) {
        const int r = e / nc, c = e % nc;
        float s = 0.f;
        for (int b = 0; b < nblocks; ++b) s += part[((long)b * kRows + r) * nc + c];
        if (c < kin) g_w1t[(long)r * ld_w1 + c] += s;
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
// ------------------------------------------------------------------------------------
// factorised edge layer:  z = W1e e + P[recv] + Q[send] + b1,  PQ = [W1i h | W1j h]
// (W1 = [W1e | W1i | W1j] of the 384-wide edge-update perceptron), e' = e + W2 relu(z) + b2
// ------------------------------------------------------------------------------------
struct LinArgs {
    long rows;
    const bf16 *x;      // [rows][KIN]
    const bf16 *wt;     // [NOUT][KIN] (out x in)
    bf16 *out;          // [rows][NOUT]
    float *acc_out;     // [rows][NOUT] FP32, added to (used instead of out when set)
    int *err;
};

// out = x W^T (no bias), M = 128 rows per tile, N = NOUT (<= 256), K = KIN.
template <int KIN, int NOUT>
constexpr size_t lin_smem() { return (size_t)NOUT * KIN * 2 + (size_t)kRows * KIN * 2 + 64; }

template <int KIN, int NOUT>
__global__ void __launch_bounds__(kThreads, 1) k_linear(LinArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *sW = smem;                                  // NOUT rows x KIN
    unsigned char *sA = sW + (size_t)NOUT * KIN * 2;           // 128 rows x KIN
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sA + (size_t)kRows * KIN * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int t = threadIdx.x;
    constexpr int TC = NOUT <= 128 ? 128 : 256;
    stage_dense(sW, a.wt, NOUT, KIN, 0, NOUT);
    cp_wait_all();
    const uint32_t tm = tc_setup(mbar, tslot, TC);
    const uint32_t aW = tc::smem_u32(sW), aA = tc::smem_u32(sA);
    constexpr uint32_t id = tc::idesc_bf16(kRows, NOUT, false, false);
    uint32_t phase = 0;
    bool ok = true;
    const long ntiles = (a.rows + kRows - 1) / kRows;
    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long row0 = tile * kRows, grow = row0 + t;
        stage_dense(sA, a.x, kRows, KIN, row0, a.rows);
        stage_done();
        if (t == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < KIN / 16; ++ks)
                mma_issue(tm, tc::kmajor_desc(aA, kRows, ks), tc::kmajor_desc(aW, NOUT, ks), id, ks > 0);
            mma_commit_issue(mbar);
        }
        ok = mma_wait(mbar, phase);
        if (!ok) break;
        for (int c = 0; c < NOUT / 16; ++c) {
            float v[16];
            acc16(tm, c * 16, v);
            if (grow < a.rows) {
                if (a.acc_out) {
                    float4 *d = reinterpret_cast<float4 *>(a.acc_out + grow * NOUT + c * 16);
                    for (int k = 0; k < 4; ++k) {
                        float4 o = d[k];
                        o.x += v[4 * k];
                        o.y += v[4 * k + 1];
                        o.z += v[4 * k + 2];
                        o.w += v[4 * k + 3];
                        d[k] = o;
                    }
                } else {
                    uint4 *d = reinterpret_cast<uint4 *>(a.out + grow * NOUT + c * 16);
                    d[0] = tc::pack8(v);
                    d[1] = tc::pack8(v + 8);
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
    }
    tc_teardown(tm, TC, ok, a.err, mbar, phase);
}

struct EdgeArgs {
    long rows;
    const bf16 *e;       // [rows][128] input latent, also the residual
    const bf16 *pq;      // [nodes][256]
    const int *recv, *send;
    const bf16 *w1e_t;   // [128][128]
    const float *b1;
    const bf16 *w2t;     // [128][128]
    const float *b2;
    bf16 *out;           // [rows][128]
    bf16 *h1;            // [rows][128] or null
    int *err;
};

constexpr size_t edge_smem() { return 3 * (size_t)kRows * kHidden * 2 + 64; }

// Two CTAs of 256 threads per SM (96 KB of shared memory each), so that one CTA's tensor-core
// and memory waits overlap the other's epilogues.  Thread (row t, half) prefetches the half
// rows of P[recv] and Q[send] it needs into registers before the first product, reloads its
// residual half row (an L2 hit) while the second product runs, and writes its output through
// the spent tile so that whole 256-byte rows leave the SM.
__global__ void __launch_bounds__(kFwdThreads, 2) k_edge_fwd(EdgeArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr size_t T = (size_t)kRows * kHidden * 2;
    unsigned char *sW1 = smem;          // W1e^T 128 x 128
    unsigned char *sW2 = sW1 + T;       // W2^T 128 x 128
    unsigned char *sA = sW2 + T;        // e tile -> hidden tile -> output tile
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sA + T);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    __shared__ float s_b1[kHidden], s_b2[kHidden];
    const int tid = threadIdx.x;
    const int t = tid & (kRows - 1);   // tile row (TMEM lane)
    const int half = tid >> 7;         // features [64 half, 64 half + 64)
    if (half == 0) s_b1[t] = a.b1[t];
    else s_b2[t] = a.b2[t];
    stage_dense(sW1, a.w1e_t, kHidden, kHidden, 0, kHidden);
    stage_dense(sW2, a.w2t, kHidden, kHidden, 0, kHidden);
    cp_wait_all();
    const uint32_t tm = tc_setup(mbar, tslot, 128);
    const uint32_t aW1 = tc::smem_u32(sW1), aW2 = tc::smem_u32(sW2), aA = tc::smem_u32(sA);
    constexpr uint32_t id = tc::idesc_bf16(kRows, kHidden, false, false);
    uint32_t phase = 0;
    bool ok = true;
    const long ntiles = (a.rows + kRows - 1) / kRows;
    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long row0 = tile * kRows, grow = row0 + t;
        const bool live = grow < a.rows;
        stage_dense(sA, a.e, kRows, kHidden, row0, a.rows);
        uint4 p[8], q[8];
        {
            const long r = live ? a.recv[grow] : 0, c = live ? a.send[grow] : 0;
            const uint4 *ps = reinterpret_cast<const uint4 *>(a.pq + r * 2 * kHidden + half * 64);
            const uint4 *qs = reinterpret_cast<const uint4 *>(a.pq + c * 2 * kHidden + kHidden + half * 64);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                p[k] = ps[k];
                q[k] = qs[k];
            }
        }
        stage_done();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < kHidden / 16; ++ks)
                mma_issue(tm, tc::kmajor_desc(aA, kRows, ks), tc::kmajor_desc(aW1, kHidden, ks), id, ks > 0);
            mma_commit_issue(mbar);
        }
        ok = mma_wait(mbar, phase);
        if (!ok) break;
#pragma unroll
        for (int b = 0; b < 2; ++b) {   // two batches of 32 columns keep the P/Q registers live
            float w[32];
            acc32(tm, half * 64 + b * 32, w);
#pragma unroll
            for (int c2 = 0; c2 < 2; ++c2) {
                const int cc = 2 * b + c2;
                const int c = half * 4 + cc;   // 16-feature group
                float *v = w + 16 * c2, pf[8], qf[8];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    tc::unpack8(p[2 * cc + h], pf);
                    tc::unpack8(q[2 * cc + h], qf);
                    for (int k = 0; k < 8; ++k)
                        v[8 * h + k] = fmaxf(v[8 * h + k] + s_b1[c * 16 + 8 * h + k] + pf[k] + qf[k], 0.f);
                }
                const uint4 lo = tc::pack8(v), hi = tc::pack8(v + 8);
                *reinterpret_cast<uint4 *>(sA + tc::tile_off(kRows, t, 2 * c)) = lo;
                *reinterpret_cast<uint4 *>(sA + tc::tile_off(kRows, t, 2 * c + 1)) = hi;
                if (a.h1 && live) {
                    uint4 *dst = reinterpret_cast<uint4 *>(a.h1 + grow * kHidden + c * 16);
                    dst[0] = lo;
                    dst[1] = hi;
                }
            }
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < kHidden / 16; ++ks)
                mma_issue(tm, tc::kmajor_desc(aA, kRows, ks), tc::kmajor_desc(aW2, kHidden, ks), id, ks > 0);
            mma_commit_issue(mbar);
        }
        {   // residual half row while the second product runs
            const uint4 *es = reinterpret_cast<const uint4 *>(a.e + (live ? grow : 0) * kHidden + half * 64);
#pragma unroll
            for (int k = 0; k < 8; ++k) p[k] = es[k];
        }
        ok = mma_wait(mbar, phase);
        if (!ok) break;
        {
            float w[64];
            acc64(tm, half * 64, w);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const int c = half * 4 + cc;
                float *v = w + 16 * cc, r[8];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    tc::unpack8(p[2 * cc + h], r);
                    for (int k = 0; k < 8; ++k) v[8 * h + k] += s_b2[c * 16 + 8 * h + k] + r[k];
                }
                out_put(sA, t, 2 * c, tc::pack8(v));
                out_put(sA, t, 2 * c + 1, tc::pack8(v + 8));
            }
        }
        tc::fence_before_sync();
        __syncthreads();
        copy_out(sA, a.out, row0, a.rows);
        __syncthreads();
    }
    tc_teardown(tm, 128, ok, a.err, mbar, phase);
}

// The same layer with its row tiles brought in by the tensor copy engine and the hidden tile
// kept in tensor memory, so that the next tile's input is in flight during this tile's
// products and epilogues.  Per CTA (two per SM, 256 threads): the e tile of 128 rows arrives as
// two 64-feature boxes of a tiled tensor copy in the 128-byte swizzle layout (one elected thread
// issues them on an mbarrier, one tile ahead: as soon as the first product of the current tile
// has read the buffer); the first product reads it from shared memory; the epilogue writes the
// hidden activations as BF16 pairs into tensor memory (tcgen05.st), which is the A operand of
// the second product; the second epilogue stores each thread's half row straight to global
// memory.  Same arithmetic, in the same order, as k_edge_fwd.
constexpr size_t edge_tma_smem() { return 1024 + 3 * (size_t)kRows * kHidden * 2 + 64; }

__global__ void __launch_bounds__(kFwdThreads, 2) k_edge_fwd_tma(const __grid_constant__ CUtensorMap tm_e, EdgeArgs a) {
    // 1,024-byte alignment by hand: an extern array declared with it would raise the alignment of
    // every kernel's dynamic shared memory in this file (and their static padding with it)
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr uint32_t T = (uint32_t)kRows * kHidden * 2;   // one 128 x 128 BF16 tile
    unsigned char *sE = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);   // 1,024-byte aligned
    unsigned char *sW1 = sE + T;   // W1e^T 128 x 128 (row tile)
    unsigned char *sW2 = sW1 + T;  // W2^T 128 x 128 (row tile)
    uint64_t *bar_mma = reinterpret_cast<uint64_t *>(sW2 + T);
    uint64_t *bar_e = bar_mma + 1;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar_e + 1);
    __shared__ float s_b1[kHidden], s_b2[kHidden];
    const int tid = threadIdx.x;
    const int t = tid & (kRows - 1);   // tile row (TMEM lane)
    const int half = tid >> 7;         // features [64 half, 64 half + 64)
    if (half == 0) s_b1[t] = a.b1[t];
    else s_b2[t] = a.b2[t];
    stage_dense(sW1, a.w1e_t, kHidden, kHidden, 0, kHidden);
    stage_dense(sW2, a.w2t, kHidden, kHidden, 0, kHidden);
    cp_wait_all();
    if (tid == 0) {
        tc::mbar_init(bar_mma, 1);
        tc::mbar_init(bar_e, 1);
        tc::mbar_init_fence();
    }
    if (tid < 32) {
        tc::tmem_alloc(tslot, 256);
        tc::tmem_relinquish();
    }
    tc::fence_async_smem();   // the weight tiles, complete, visible to the tensor core
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = *tslot;
    const uint32_t tacc = tm;         // accumulator, 128 columns (both products)
    const uint32_t ta = tm + 128;     // hidden tile as the second product's A operand, 64 columns
    const uint32_t aE = tc::smem_u32(sE), aW1 = tc::smem_u32(sW1), aW2 = tc::smem_u32(sW2);
    constexpr uint32_t id = tc::idesc_bf16(kRows, kHidden, false, false);
    const long ntiles = (a.rows + kRows - 1) / kRows;
    auto issue_e = [&](long tile) {   // thread 0: the tile's two feature boxes
        tc::mbar_arrive_expect(bar_e, T);
        tc::tma_load_2d(sE, &tm_e, 0, (int)(tile * kRows), bar_e);
        tc::tma_load_2d(sE + T / 2, &tm_e, 64, (int)(tile * kRows), bar_e);
    };
    uint32_t ph_mma = 0, ph_e = 0;
    bool ok = true, e_pending = false;   // e_pending: thread 0 has a tile copy not yet waited for
    if (tid == 0 && (long)blockIdx.x < ntiles) {
        issue_e(blockIdx.x);
        e_pending = true;
    }
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long row0 = tile * kRows, grow = row0 + t;
        const bool live = grow < a.rows;
        uint4 p[8], q[8];
        {
            const long r = live ? a.recv[grow] : 0, c = live ? a.send[grow] : 0;
            const uint4 *ps = reinterpret_cast<const uint4 *>(a.pq + r * 2 * kHidden + half * 64);
            const uint4 *qs = reinterpret_cast<const uint4 *>(a.pq + c * 2 * kHidden + kHidden + half * 64);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                p[k] = ps[k];
                q[k] = qs[k];
            }
        }
        // the e tile; the block barrier also orders every thread's reads of the previous tile's
        // accumulator before this tile's first product
        const bool e_ok = tc::mbar_wait(bar_e, ph_e, g_tc_wait_limit);
        if (!__syncthreads_and(e_ok)) {
            ok = false;
            break;
        }
        ph_e ^= 1u;
        if (tid == 0) {
            e_pending = false;
            tc::fence_after_sync();
            for (int ks = 0; ks < kHidden / 16; ++ks)
                mma_issue(tacc, tc::sdesc_sw128(aE + (uint32_t)(ks >> 2) * (T / 2) + (uint32_t)(ks & 3) * 32u),
                          tc::kmajor_desc(aW1, kHidden, ks), id, ks > 0);
            mma_commit_issue(bar_mma);
        }
        ok = mma_wait(bar_mma, ph_mma);
        if (!ok) break;
        // the first product has read the e tile: the next tile's copy goes into its buffer
        if (tid == 0 && tile + gridDim.x < ntiles) {
            issue_e(tile + gridDim.x);
            e_pending = true;
        }
#pragma unroll
        for (int b = 0; b < 2; ++b) {   // two batches of 32 columns keep the P/Q registers live
            float w[32];
            acc32(tacc, half * 64 + b * 32, w);
            uint32_t hw[16];
#pragma unroll
            for (int c2 = 0; c2 < 2; ++c2) {
                const int cc = 2 * b + c2;
                const int c = half * 4 + cc;   // 16-feature group
                float *v = w + 16 * c2, pf[8], qf[8];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    tc::unpack8(p[2 * cc + h], pf);
                    tc::unpack8(q[2 * cc + h], qf);
                    for (int k = 0; k < 8; ++k)
                        v[8 * h + k] = fmaxf(v[8 * h + k] + s_b1[c * 16 + 8 * h + k] + pf[k] + qf[k], 0.f);
                }
                const uint4 lo = tc::pack8(v), hi = tc::pack8(v + 8);
                hw[8 * c2 + 0] = lo.x;
                hw[8 * c2 + 1] = lo.y;
                hw[8 * c2 + 2] = lo.z;
                hw[8 * c2 + 3] = lo.w;
                hw[8 * c2 + 4] = hi.x;
                hw[8 * c2 + 5] = hi.y;
                hw[8 * c2 + 6] = hi.z;
                hw[8 * c2 + 7] = hi.w;
                if (a.h1 && live) {
                    uint4 *dst = reinterpret_cast<uint4 *>(a.h1 + grow * kHidden + c * 16);
                    dst[0] = lo;
                    dst[1] = hi;
                }
            }
            // features [64 half + 32 b, + 32) as 16 columns of BF16 pairs
            tc::tmem_st16(tc::tmem_warp_addr(ta, half * 32 + b * 16), hw);
        }
        tc::tmem_wait_st();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int ks = 0; ks < kHidden / 16; ++ks)
                mma_issue_tmem_a(tacc, ta + (uint32_t)ks * 8u, tc::kmajor_desc(aW2, kHidden, ks), id, ks > 0);
            mma_commit_issue(bar_mma);
        }
        {   // residual half row while the second product runs
            const uint4 *es = reinterpret_cast<const uint4 *>(a.e + (live ? grow : 0) * kHidden + half * 64);
#pragma unroll
            for (int k = 0; k < 8; ++k) p[k] = es[k];
        }
        ok = mma_wait(bar_mma, ph_mma);
        if (!ok) break;
        {
            float w[64];
            acc64(tacc, half * 64, w);
            uint4 o[8];
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const int c = half * 4 + cc;
                float *v = w + 16 * cc, r[8];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    tc::unpack8(p[2 * cc + h], r);
                    for (int k = 0; k < 8; ++k) v[8 * h + k] += s_b2[c * 16 + 8 * h + k] + r[k];
                }
                o[2 * cc] = tc::pack8(v);
                o[2 * cc + 1] = tc::pack8(v + 8);
            }
            if (live) {
                uint4 *dst = reinterpret_cast<uint4 *>(a.out + grow * kHidden + half * 64);
#pragma unroll
                for (int k = 0; k < 8; ++k) dst[k] = o[k];
            }
        }
        tc::fence_before_sync();
    }
    // a wait gave up with a tile copy in flight: let it land before the block's memory goes
    if (tid == 0 && e_pending) (void)tc::mbar_wait(bar_e, ph_e, g_tc_wait_limit);
    tc_teardown(tm, 256, ok, a.err, bar_mma, ph_mma);
}

// dW^T [256][128] partials: D_half[o][k] = sum_rows A[row][128 half + o] B[row][k]
struct LinWgradArgs {
    long rows;
    const bf16 *a;     // [rows][256]
    const bf16 *b;     // [rows][128]
    float *part;       // [gridDim.x][128][256]
    int *err;
};
constexpr size_t linw_smem() { return (size_t)kRows * 256 * 2 + (size_t)kRows * kHidden * 2 + 64; }

__global__ void __launch_bounds__(kThreads, 1) k_linear_wgrad(LinWgradArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *sA = smem;                              // 128 rows x 256
    unsigned char *sB = sA + (size_t)kRows * 256 * 2;      // 128 rows x 128
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sB + (size_t)kRows * kHidden * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int t = threadIdx.x;
    const uint32_t tm = tc_setup(mbar, tslot, 256);
    const uint32_t aA = tc::smem_u32(sA), aB = tc::smem_u32(sB);
    constexpr uint32_t id = tc::idesc_bf16(kRows, kHidden, true, true);
    uint32_t phase = 0;
    bool ok = true, first = true;
    const long ntiles = (a.rows + kRows - 1) / kRows;
    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long row0 = tile * kRows;
        stage_dense(sA, a.a, kRows, 256, row0, a.rows);
        stage_dense(sB, a.b, kRows, kHidden, row0, a.rows);
        stage_done();
        if (t == 0) {
            tc::fence_after_sync();
            for (int h = 0; h < 2; ++h)
                for (int ks = 0; ks < kRows / 16; ++ks)
                    mma_issue(tm + h * kHidden, tc::mnmajor_desc(aA + (uint32_t)(h * 16 * kRows * 16), kRows, ks),
                                 tc::mnmajor_desc(aB, kRows, ks), id, (!first || ks > 0) ? 1u : 0u);
            mma_commit_issue(mbar);
        }
        ok = mma_wait(mbar, phase);
        first = false;
        tc::fence_before_sync();
        __syncthreads();
    }
    float *dst = a.part + ((long)blockIdx.x * kRows + t) * 256;
    if (ok && !first) {
        tc::fence_after_sync();
        for (int c = 0; c < 256 / 16; ++c) {
            float v[16];
            acc16(tm, c * 16, v);
            for (int k = 0; k < 16; ++k) dst[c * 16 + k] = v[k];
        }
    } else {
        for (int c = 0; c < 256; ++c) dst[c] = 0.f;
    }
    tc_teardown(tm, 256, ok, a.err, mbar, phase);
}

// g[o * ld + col0 + c] += sum over blocks of part[b][o][c]   (o < 128, c < 256)
__global__ void k_linw_reduce(const float *part, int nblocks, float *g, int ld, int col0) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kRows * 256; e += gridDim.x * blockDim.x) {
        const int o = e / 256, c = e % 256;
        float s = 0.f;
        for (int b = 0; b < nblocks; ++b) s += part[((long)b * kRows + o) * 256 + c];
        g[(long)o * ld + col0 + c] += s;
    }
}

template <typename K, typename A>
int launch_tc(K kernel, size_t smem, int tmem_cols, long rows, A args, cudaStream_t s, int max_blocks = 148,
              int threads = kThreads) {
    if (rows <= 0) return DEM_OK;
    const size_t floor_bytes = tmem_cols >= 512 ? 116 * 1024 : (tmem_cols >= 256 ? 80 * 1024 : 0);
    if (smem < floor_bytes) smem = floor_bytes;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return DEM_ERR_CUDA;
    const long ntiles = (rows + kRows - 1) / kRows;
    if (max_blocks <= 0) {   // as many CTAs as the SMs hold (shared memory and TMEM), persistent
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return DEM_ERR_CUDA;
        const size_t per = smem + fa.sharedSizeBytes + 1024;
        int fit = (int)((228 * 1024) / per);
        fit = fit < 512 / tmem_cols ? fit : 512 / tmem_cols;
        max_blocks = 148 * (fit > 0 ? fit : 1);
    }
    const int grid = (int)(ntiles < max_blocks ? ntiles : max_blocks);
    kernel<<<grid, threads, smem, s>>>(args);
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
    a.resid_src0 = (resid && resid == src[0].data && !src[0].index && src[0].width == m.nout) ? 1 : 0;
    a.out = (bf16 *)out;
    a.out_f32 = out_f32;
    a.h1 = (bf16 *)h1;
    a.err = err;
#define X(KI, NO) \
    if (m.kin == KI && m.nout == NO)                                                                        \
        return launch_tc(k_mlp_fwd<KI, NO>, fwd_smem<KI, NO>(), 128, rows, a, s, 0, kFwdThreads);
    B200_NN_SHAPES(X)
#undef X
    return DEM_ERR_UNSUPPORTED;
}

int nn_mlp_backward(const dem_nn_mlp &m, long rows, const dem_nn_rows *src, int nsrc, const void *dy, const void *h1,
                    void *dz1, float *dx, float *g_w1t, int ld_w1, float *g_b1, float *g_w2t, float *g_b2,
                    float *part, int *err, cudaStream_t s) {
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
    k_wgrad_reduce<<<64, 256, 0, s>>>(part, nblocks, m.kin, m.nout, g_w1t, ld_w1, g_b1, g_w2t, g_b2);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

// PQ[rows][256] = h W1ij^T (W1ij^T: [256][128]).
int nn_linear_pq(long rows, const void *h, const void *w1ij_t, void *pq, int *err, cudaStream_t s) {
    LinArgs a{rows, (const bf16 *)h, (const bf16 *)w1ij_t, (bf16 *)pq, nullptr, err};
    return launch_tc(k_linear<128, 256>, lin_smem<128, 256>(), 256, rows, a, s, 0);
}

// dh[rows][128] += dPQ W1ij (dPQ: [rows][256] bf16, W1ij: [128][256]).
int nn_linear_pq_backward(long rows, const void *dpq, const void *w1ij, float *dh, int *err, cudaStream_t s) {
    LinArgs a{rows, (const bf16 *)dpq, (const bf16 *)w1ij, nullptr, dh, err};
    return launch_tc(k_linear<256, 128>, lin_smem<256, 128>(), 128, rows, a, s, 0);
}

// g_w1t[o][col0 + c] += sum_rows dPQ[row][c'] h[row][k] arranged as dW1ij^T (ld = row stride).
int nn_linear_pq_wgrad(long rows, const void *dpq, const void *h, float *g_w1t, int ld, int col0, float *part,
                       int *err, cudaStream_t s) {
    if (rows <= 0) return DEM_OK;
    LinWgradArgs a{rows, (const bf16 *)dpq, (const bf16 *)h, part, err};
    const int st = launch_tc(k_linear_wgrad, linw_smem(), 256, rows, a, s);
    if (st) return st;
    const long ntiles = (rows + kRows - 1) / kRows;
    k_linw_reduce<<<64, 256, 0, s>>>(part, (int)(ntiles < 148 ? ntiles : 148), g_w1t, ld, col0);
    return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

namespace {
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the driver
// library); null when the driver does not provide it.
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_tiled() {
    static EncodeTiled fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiled) nullptr;
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}

// Tensor map of e [rows][128] BF16 with 64 x 128 boxes in the 128-byte swizzle layout.
bool edge_map(CUtensorMap *m, const void *e, long rows) {
    const EncodeTiled enc = encode_tiled();
    if (!enc || (reinterpret_cast<uintptr_t>(e) & 15u) || rows <= 0 || rows > 0x7FFFFFFFL - kRows) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)kHidden, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kHidden * 2};
    const cuuint32_t box[2] = {64u, (cuuint32_t)kRows};
    const cuuint32_t elem[2] = {1u, 1u};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(e), dims, strides, box, elem,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

// form 0: the tensor-copy kernel (k_edge_fwd_tma) where the tensor map can be made, else the
// staged kernel; form 1: the staged kernel (k_edge_fwd); -1: the build's default
// (EDGE_FORM_DEFAULT).  Same results.
#ifndef EDGE_FORM_DEFAULT
#define EDGE_FORM_DEFAULT 0
#endif
int nn_edge_forward(long rows, const void *e, const void *pq, const int *recv, const int *send, const void *w1e_t,
                    const float *b1, const void *w2t, const float *b2, void *out, void *h1, int *err, cudaStream_t s,
                    int form) {
    EdgeArgs a{rows, (const bf16 *)e, (const bf16 *)pq, recv, send, (const bf16 *)w1e_t, b1, (const bf16 *)w2t, b2,
               (bf16 *)out, (bf16 *)h1, err};
    if (rows <= 0) return DEM_OK;
    if (form < 0) form = EDGE_FORM_DEFAULT;
    CUtensorMap m;
    if (form == 0 && edge_map(&m, e, rows)) {
        const size_t smem = edge_tma_smem();
        if (cudaFuncSetAttribute(k_edge_fwd_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return DEM_ERR_CUDA;
        int sms = 148, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const long ntiles = (rows + kRows - 1) / kRows, cap = 2L * (sms > 0 ? sms : 148);   // two CTAs per SM
        k_edge_fwd_tma<<<(int)(ntiles < cap ? ntiles : cap), kFwdThreads, smem, s>>>(m, a);
        return cudaGetLastError() == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
    }
    return launch_tc(k_edge_fwd, edge_smem(), 128, rows, a, s, 0, kFwdThreads);
}

long nn_linear_wgrad_scratch() { return 148L * kRows * 256; }

// Scratch floats the per-CTA weight-gradient partials of one backward call need.
int nn_debug_waits(int poll_limit, int drop_mma, cudaStream_t s) {
    const int lim = poll_limit > 0 ? poll_limit : (1 << 22);
    const int drop = drop_mma ? 1 : 0;
    if (cudaMemcpyToSymbolAsync(g_tc_wait_limit, &lim, sizeof(int), 0, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyToSymbolAsync(g_tc_drop_mma, &drop, sizeof(int), 0, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return DEM_ERR_CUDA;
    return DEM_OK;
}

long nn_wgrad_scratch(int kin, int nout) {
    const int nw2 = nout == kHidden ? kHidden : nout;
    return 148L * kRows * (kin + nw2 + 2);
}

}  // namespace b200dem
