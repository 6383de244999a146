// dem_surrogate.cu -- learned surrogate for the bulk flow: a message-passing network over
// the contact graph that advances quasi-2D particles by one stride of `steps_per_stride`
// DEM steps, trained on rollouts of the DEM solver, with plain DEM as the fallback.
//
// Per stride (positions p_k, p_{k-1} in caller order):
//   graph     pairs with |x_i - x_j| <= radius_graph (the cell-list build of dem_nbr.cu with a
//             fixed cutoff; frames of a training batch are its independent scenes), turned
//             into a CSR edge list sorted by (receiver, sender) with reverse-edge indices
//   features  node: d/sigma_d (d = p_k - p_{k-1}), clipped wall distances, radius;
//             edge: (x_j - x_i)/R, |x_j - x_i|/R, gap/r_mean, (d_j - d_i)/sigma_d
//   network   h = EncN(x_n), e = EncE(x_e); 3 x { e += Msg[e, h_i, h_j]; h += Upd[h, sum_j e] };
//             a = Dec(h) -- every dense layer is dem_nn.cu's tensor-core MLP; the sums over
//             a node's edges run in CSR order (deterministic)
//   update    p_{k+1} = p_k + d + sigma_a * a, projected out of the walls
// Training: mean squared error of a against (p_{k+1} - p_k) - d with noise on the inputs,
// backward through all layers (fixed-order reductions), Adam on FP32 master weights that
// refreshes both BF16 layouts.  Rollout: a network stride is kept only if its largest
// overlap and its energy rise stay under the thresholds; otherwise that stride is run by
// the DEM solver from the state before it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_bf16.h>

#include "b200dem.h"
#include "dem_internal.cuh"

using namespace b200dem;

namespace {

using bf16 = __nv_bfloat16;
constexpr int kH = 128;
constexpr int kF = 16;          // feature width of the encoders' inputs and the decoder's output
constexpr int kNL = 9;          // dense layers
constexpr int kTB = 256;
constexpr int kGS = 148 * 8;
constexpr int kSgWalls = 4;

struct Shape {
    int kin, nout;
};
constexpr Shape kShape[kNL] = {{16, 128}, {16, 128}, {384, 128}, {256, 128}, {384, 128},
                               {256, 128}, {384, 128}, {256, 128}, {128, 16}};
constexpr int L_ENC_N = 0, L_ENC_E = 1, L_DEC = 8;
inline int L_MSG(int l) { return 2 + 2 * l; }
inline int L_UPD(int l) { return 3 + 2 * l; }
inline bool is_msg(int l) { return l == 2 || l == 4 || l == 6; }

struct FeatConst {
    double inv_rg, inv_sd, sigma_a, r_mean, inv_r_mean, inv_r_std, inv_clip;
    int nwalls;
    double wx[kSgWalls][2], wn[kSgWalls][2];
};

template <class T>
cudaError_t dmalloc(T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * count);
}

// ---------------------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------------------
// Inputs -> packed positions (x, y, 0, r) for the graph build, displacement d = cur - prev
// (+ seeded Gaussian noise on both positions when noise > 0).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double unit_open(unsigned long long h) {   // (0, 1)
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ void gauss2(unsigned long long seed, long i, int k, double &a, double &b) {
    const unsigned long long h1 = mix64(seed ^ mix64((unsigned long long)(4 * i + 2 * k)));
    const unsigned long long h2 = mix64(seed ^ mix64((unsigned long long)(4 * i + 2 * k + 1)));
    const double r = sqrt(-2.0 * log(unit_open(h1))), th = 6.283185307179586 * unit_open(h2);
    a = r * cos(th);
    b = r * sin(th);
}

__global__ void k_inputs(int n, const double *prev, const double *cur, const double *rad, double noise,
                         unsigned long long seed, double4 *packed, double2 *disp, int *perm) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double cx = cur[3 * i], cy = cur[3 * i + 1], px = prev[3 * i], py = prev[3 * i + 1];
        if (noise > 0.0) {
            double a, b, c, d;
            gauss2(seed, i, 0, a, b);
            gauss2(seed, i, 1, c, d);
            cx += noise * a;
            cy += noise * b;
            px += noise * c;
            py += noise * d;
        }
        packed[i] = make_double4(cx, cy, 0.0, rad[i]);
        disp[i] = make_double2(cx - px, cy - py);
        perm[i] = i;
    }
}

// ---- CSR of the neighbour lists ----
constexpr int kScanB = 1024;
__global__ void k_scan_block(int n, const int *nn, int *offs, int *bsum) {
    __shared__ int s[kScanB];
    const int i = blockIdx.x * kScanB + threadIdx.x;
    const int v = i < n ? nn[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kScanB; o <<= 1) {
        const int a = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += a;
        __syncthreads();
    }
    if (i < n) offs[i] = s[threadIdx.x] - v;
    if (threadIdx.x == kScanB - 1) bsum[blockIdx.x] = s[kScanB - 1];
}
__global__ void k_scan_sums(int nb, int *bsum, int *total) {   // one block
    __shared__ int s[kScanB];
    int carry = 0;
    for (int base = 0; base < nb; base += kScanB) {
        const int i = base + threadIdx.x;
        const int v = i < nb ? bsum[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < kScanB; o <<= 1) {
            const int a = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += a;
            __syncthreads();
        }
        if (i < nb) bsum[i] = carry + s[threadIdx.x] - v;
        const int t = s[kScanB - 1];
        __syncthreads();
        carry += t;
    }
    if (threadIdx.x == 0) *total = carry;
}
__global__ void k_scan_add(int n, int *offs, const int *bsum, const int *total) {
    const int i = blockIdx.x * kScanB + threadIdx.x;
    if (i < n) offs[i] += bsum[blockIdx.x];
    if (i == 0) offs[n] = *total;
}
__global__ void k_csr_fill(int n, int cap, const int *nn, const int *idx, const int *offs, int *recv, int *send) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b = offs[i], c = nn[i];
        for (int k = 0; k < c; ++k) {
            recv[b + k] = i;
            send[b + k] = idx[(long)k * cap + i];
        }
    }
}
// rev[e] of e = (i <- j): the edge (j <- i), found by bisection in j's sorted senders.
__global__ void k_csr_rev(int ne, const int *recv, const int *send, const int *offs, int *rev) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const int i = recv[e], j = send[e];
        int lo = offs[j], hi = offs[j + 1] - 1, r = -1;
        while (lo <= hi) {
            const int mid = (lo + hi) >> 1;
            const int v = send[mid];
            if (v == i) {
                r = mid;
                break;
            }
            if (v < i) lo = mid + 1;
            else hi = mid - 1;
        }
        rev[e] = r;
    }
}

// ---- features ----
__device__ __forceinline__ void store16(bf16 *dst, const float v[kF]) {
    for (int k = 0; k < kF; k += 2) *reinterpret_cast<__nv_bfloat162 *>(dst + k) = __floats2bfloat162_rn(v[k], v[k + 1]);
}
__device__ __forceinline__ float clip1(double v) { return (float)fmax(-1.0, fmin(1.0, v)); }

__global__ void k_node_feat(int n, const double4 *pk, const double2 *disp, FeatConst fc, bf16 *xn) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double4 p = pk[i];
        const double2 d = disp[i];
        float v[kF] = {};
        v[0] = (float)(d.x * fc.inv_sd);
        v[1] = (float)(d.y * fc.inv_sd);
        for (int w = 0; w < fc.nwalls; ++w) {
            const double dist = (p.x - fc.wx[w][0]) * fc.wn[w][0] + (p.y - fc.wx[w][1]) * fc.wn[w][1] - p.w;
            v[2 + w] = clip1(dist * fc.inv_clip);
        }
        v[6] = (float)((p.w - fc.r_mean) * fc.inv_r_std);
        store16(xn + (long)i * kF, v);
    }
}

__global__ void k_edge_feat(int ne, const int *recv, const int *send, const double4 *pk, const double2 *disp,
                            FeatConst fc, bf16 *xe) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const int i = recv[e], j = send[e];
        const double4 a = pk[i], b = pk[j];
        const double2 da = disp[i], db = disp[j];
        const double dx = b.x - a.x, dy = b.y - a.y;
        const double dist = sqrt(dx * dx + dy * dy);
        float v[kF] = {};
        v[0] = (float)(dx * fc.inv_rg);
        v[1] = (float)(dy * fc.inv_rg);
        v[2] = (float)(dist * fc.inv_rg);
        v[3] = (float)((dist - a.w - b.w) * fc.inv_r_mean);
        v[4] = (float)((db.x - da.x) * fc.inv_sd);
        v[5] = (float)((db.y - da.y) * fc.inv_sd);
        store16(xe + (long)e * kF, v);
    }
}

// ---- aggregation over a node's edges (CSR order, FP32) ----
// agg[i] = sum_{e in edges(i)} e_val[e]  (bf16 in and out); one warp per node, 4 features/lane.
__global__ void k_segsum(int n, const int *offs, const bf16 *ev, bf16 *agg) {
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
        for (int e = offs[i]; e < offs[i + 1]; ++e) {
            const uint2 u = *reinterpret_cast<const uint2 *>(ev + (long)e * kH + 4 * lane);
            const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
            const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
            s0 += a.x;
            s1 += a.y;
            s2 += b.x;
            s3 += b.y;
        }
        __nv_bfloat162 lo = __floats2bfloat162_rn(s0, s1), hi = __floats2bfloat162_rn(s2, s3);
        uint2 o;
        o.x = *reinterpret_cast<uint32_t *>(&lo);
        o.y = *reinterpret_cast<uint32_t *>(&hi);
        *reinterpret_cast<uint2 *>(agg + (long)i * kH + 4 * lane) = o;
    }
}

// de[e] (=|+=) dn[recv[e]][c0:c0+128]
__global__ void k_edge_from_node(int ne, const int *recv, const float *dn, int ld, int c0, float *de, int accumulate) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < (long)ne * (kH / 4); q += (long)gridDim.x * blockDim.x) {
        const long e = q / (kH / 4);
        const int c = (int)(q % (kH / 4)) * 4;
        const float4 a = *reinterpret_cast<const float4 *>(dn + (long)recv[e] * ld + c0 + c);
        float4 *d = reinterpret_cast<float4 *>(de + e * kH + c);
        if (accumulate) {
            float4 v = *d;
            v.x += a.x;
            v.y += a.y;
            v.z += a.z;
            v.w += a.w;
            *d = v;
        } else {
            *d = a;
        }
    }
}

// dst[r][0:128] += src[r][c0:c0+128]
__global__ void k_add_cols(long rows, const float *src, int ld, int c0, float *dst) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < rows * (kH / 4); q += (long)gridDim.x * blockDim.x) {
        const long r = q / (kH / 4);
        const int c = (int)(q % (kH / 4)) * 4;
        const float4 a = *reinterpret_cast<const float4 *>(src + r * ld + c0 + c);
        float4 *d = reinterpret_cast<float4 *>(dst + r * kH + c);
        float4 v = *d;
        v.x += a.x;
        v.y += a.y;
        v.z += a.z;
        v.w += a.w;
        *d = v;
    }
}

__global__ void k_f2bf(long count, const float *src, bf16 *dst) {
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < count / 2; q += (long)gridDim.x * blockDim.x)
        reinterpret_cast<__nv_bfloat162 *>(dst)[q] = __floats2bfloat162_rn(src[2 * q], src[2 * q + 1]);
}

// ---- loss: mean over nodes and the 2 components of (a - target)^2 ----
constexpr int kLossBlocks = 256;
__global__ void k_loss(int n, const float *out, const double4 *pk, const double2 *disp, const double *next,
                       double inv_sa, bf16 *dout, double *part) {
    __shared__ double s[kTB];
    double acc = 0.0;
    const double scale = 1.0 / (2.0 * n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double tx = ((next[3 * i] - pk[i].x) - disp[i].x) * inv_sa;
        const double ty = ((next[3 * i + 1] - pk[i].y) - disp[i].y) * inv_sa;
        const double ex = (double)out[(long)i * kF] - tx, ey = (double)out[(long)i * kF + 1] - ty;
        acc += ex * ex + ey * ey;
        float g[kF] = {};
        g[0] = (float)(2.0 * ex * scale);
        g[1] = (float)(2.0 * ey * scale);
        store16(dout + (long)i * kF, g);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = kTB / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0] * scale;
}
__global__ void k_sum_parts(int nb, const double *part, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += part[b];
        *out = s;
    }
}

// ---- Adam + BF16 refresh ----
__global__ void k_adam(long np, float *w, const float *g, float *m, float *v, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < np; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}
// BF16 copies of one layer: W1^T [128][kin] and W1 [kin][128], W2^T [nout][128] and W2 [128][nout].
__global__ void k_refresh(int kin, int nout, const float *w1t, const float *w2t, bf16 *b_w1t, bf16 *b_w1, bf16 *b_w2t,
                          bf16 *b_w2) {
    const int n1 = kH * kin, n2 = nout * kH;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n1 + n2; q += gridDim.x * blockDim.x) {
        if (q < n1) {
            const int r = q / kin, c = q % kin;
            const bf16 x = __float2bfloat16_rn(w1t[q]);
            b_w1t[q] = x;
            b_w1[c * kH + r] = x;
        } else {
            const int k = q - n1, r = k / kH, c = k % kH;
            const bf16 x = __float2bfloat16_rn(w2t[k]);
            b_w2t[k] = x;
            b_w2[c * nout + r] = x;
        }
    }
}

// Message layers: W1 = [W1e | W1i | W1j] (128 x 384) also as W1e^T [128][128], W1e [128][128],
// W1ij^T [256][128] (row 128 h + o = W1t[o][128 + 128 h + k]) and W1ij [128][256].
__global__ void k_refresh_msg(const float *w1t, bf16 *e_t, bf16 *e, bf16 *ij_t, bf16 *ij) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kH * 384; q += gridDim.x * blockDim.x) {
        const int o = q / 384, c = q % 384;
        const bf16 x = __float2bfloat16_rn(w1t[q]);
        if (c < kH) {
            e_t[o * kH + c] = x;
            e[c * kH + o] = x;
        } else {
            const int half = (c - kH) / kH, k = (c - kH) % kH;
            const int row = half * kH + o;        // row of W1ij^T
            ij_t[row * kH + k] = x;
            ij[k * 2 * kH + row] = x;
        }
    }
}

// dPQ[i] = [sum over i's edges of dz1[e] | sum over edges sending from i of dz1[e]] (BF16 out).
__global__ void k_dpq(int n, const int *offs, const int *rev, const bf16 *dz1, bf16 *dpq) {
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
        float p[4] = {0.f, 0.f, 0.f, 0.f}, q[4] = {0.f, 0.f, 0.f, 0.f};
        for (int e = offs[i]; e < offs[i + 1]; ++e) {
            const uint2 u = *reinterpret_cast<const uint2 *>(dz1 + (long)e * kH + 4 * lane);
            const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
            const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
            p[0] += a.x; p[1] += a.y; p[2] += b.x; p[3] += b.y;
            const int r = rev[e];
            if (r >= 0) {
                const uint2 w = *reinterpret_cast<const uint2 *>(dz1 + (long)r * kH + 4 * lane);
                const float2 c = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&w.x));
                const float2 d = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&w.y));
                q[0] += c.x; q[1] += c.y; q[2] += d.x; q[3] += d.y;
            }
        }
        bf16 *o = dpq + (long)i * 2 * kH;
        *reinterpret_cast<__nv_bfloat162 *>(o + 4 * lane) = __floats2bfloat162_rn(p[0], p[1]);
        *reinterpret_cast<__nv_bfloat162 *>(o + 4 * lane + 2) = __floats2bfloat162_rn(p[2], p[3]);
        *reinterpret_cast<__nv_bfloat162 *>(o + kH + 4 * lane) = __floats2bfloat162_rn(q[0], q[1]);
        *reinterpret_cast<__nv_bfloat162 *>(o + kH + 4 * lane + 2) = __floats2bfloat162_rn(q[2], q[3]);
    }
}

// ---- stride update and checks ----
__global__ void k_integrate(int n, const double4 *pk, const double2 *disp, const float *out, double sa, FeatConst fc,
                            const double *cur3, double *next3) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double4 p = pk[i];
        double x = p.x + disp[i].x + sa * (double)out[(long)i * kF];
        double y = p.y + disp[i].y + sa * (double)out[(long)i * kF + 1];
        for (int w = 0; w < fc.nwalls; ++w) {   // project out of the walls
            const double dist = (x - fc.wx[w][0]) * fc.wn[w][0] + (y - fc.wx[w][1]) * fc.wn[w][1] - p.w;
            if (dist < 0.0) {
                x -= dist * fc.wn[w][0];
                y -= dist * fc.wn[w][1];
            }
        }
        next3[3 * i] = x;
        next3[3 * i + 1] = y;
        next3[3 * i + 2] = cur3[3 * i + 2];
    }
}

// One Jacobi sweep of contact projection on positions q (caller [n][3]) -> qo: every pair of
// the graph overlapping by more than allow * min(r_i, r_j) is pushed apart along its normal,
// each side by its mass share of the excess (times 0.5, for stability of the simultaneous
// update); walls push a particle back to contact.
__global__ void k_project(int n, const int *offs, const int *send, const double *q, const double *rad,
                          const double *mass, FeatConst fc, double allow, double *qo) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double xi = q[3 * i], yi = q[3 * i + 1], ri = rad[i], mi = mass[i];
        double dx_acc = 0.0, dy_acc = 0.0;
        for (int e = offs[i]; e < offs[i + 1]; ++e) {
            const int j = send[e];
            const double dx = q[3 * j] - xi, dy = q[3 * j + 1] - yi;
            const double d = sqrt(dx * dx + dy * dy);
            const double excess = ri + rad[j] - d - allow * fmin(ri, rad[j]);
            if (excess > 0.0 && d > 0.0) {
                const double share = 0.5 * mass[j] / (mi + mass[j]);
                dx_acc -= share * excess * dx / d;
                dy_acc -= share * excess * dy / d;
            }
        }
        double x = xi + dx_acc, y = yi + dy_acc;
        for (int w = 0; w < fc.nwalls; ++w) {
            const double dist = (x - fc.wx[w][0]) * fc.wn[w][0] + (y - fc.wx[w][1]) * fc.wn[w][1] - ri;
            if (dist < 0.0) {
                x -= dist * fc.wn[w][0];
                y -= dist * fc.wn[w][1];
            }
        }
        qo[3 * i] = x;
        qo[3 * i + 1] = y;
        qo[3 * i + 2] = q[3 * i + 2];
    }
}

__global__ void k_rad3(int n, const double *rad, double *w) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] = rad[i] * rad[i] * rad[i];
}

// Largest overlap / smaller radius over the graph's pairs at positions q (caller [n][3]) and
// the walls; kinetic energy 0.5 m |q - p|^2 / T^2, potential -m g.q, the total mass and the
// largest specific energy 0.5 |v|^2 - g.q of one particle.  Block partials, summed in block
// order.
constexpr int kChkBlocks = 256;
__global__ void k_check(int n, const int *offs, const int *send, const double *q, const double *rad, const double *mass,
                        FeatConst fc, double inv_T, double gx, double gy, const double *p, double *part) {
    __shared__ double s_ov[kTB], s_ek[kTB], s_ep[kTB], s_m[kTB], s_es[kTB];
    double ov = 0.0, ek = 0.0, ep = 0.0, ms = 0.0, es = -1e300;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double xi = q[3 * i], yi = q[3 * i + 1], ri = rad[i];
        for (int e = offs ? offs[i] : 0; e < (offs ? offs[i + 1] : 0); ++e) {
            const int j = send[e];
            const double dx = q[3 * j] - xi, dy = q[3 * j + 1] - yi;
            const double gap = ri + rad[j] - sqrt(dx * dx + dy * dy);
            ov = fmax(ov, gap / fmin(ri, rad[j]));
        }
        for (int w = 0; w < fc.nwalls; ++w) {
            const double dist = (xi - fc.wx[w][0]) * fc.wn[w][0] + (yi - fc.wx[w][1]) * fc.wn[w][1];
            ov = fmax(ov, (ri - dist) / ri);
        }
        const double vx = (xi - p[3 * i]) * inv_T, vy = (yi - p[3 * i + 1]) * inv_T;
        ek += 0.5 * mass[i] * (vx * vx + vy * vy);
        ep -= mass[i] * (gx * xi + gy * yi);
        ms += mass[i];
        es = fmax(es, 0.5 * (vx * vx + vy * vy) - (gx * xi + gy * yi));
    }
    s_ov[threadIdx.x] = ov;
    s_ek[threadIdx.x] = ek;
    s_ep[threadIdx.x] = ep;
    s_m[threadIdx.x] = ms;
    s_es[threadIdx.x] = es;
    __syncthreads();
    for (int o = kTB / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_ov[threadIdx.x] = fmax(s_ov[threadIdx.x], s_ov[threadIdx.x + o]);
            s_ek[threadIdx.x] += s_ek[threadIdx.x + o];
            s_ep[threadIdx.x] += s_ep[threadIdx.x + o];
            s_m[threadIdx.x] += s_m[threadIdx.x + o];
            s_es[threadIdx.x] = fmax(s_es[threadIdx.x], s_es[threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[5 * blockIdx.x] = s_ov[0];
        part[5 * blockIdx.x + 1] = s_ek[0];
        part[5 * blockIdx.x + 2] = s_ep[0];
        part[5 * blockIdx.x + 3] = s_m[0];
        part[5 * blockIdx.x + 4] = s_es[0];
    }
}
__global__ void k_check_sum(int nb, const double *part, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double ov = 0.0, ek = 0.0, ep = 0.0, ms = 0.0, es = -1e300;
        for (int b = 0; b < nb; ++b) {
            ov = fmax(ov, part[5 * b]);
            ek += part[5 * b + 1];
            ep += part[5 * b + 2];
            ms += part[5 * b + 3];
            es = fmax(es, part[5 * b + 4]);
        }
        out[0] = ov;
        out[1] = ek;
        out[2] = ep;
        out[3] = ms;
        out[4] = es;
    }
}

// ---- solver state <-> caller-order arrays ----
__global__ void k_from_solver(Particles P, const Ctl *ctl, double *x3, double *rad, double *mass) {
    const int cur = ctl->cur;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        const int s = P.rank[i];
        const double4 p = P.pos[cur][s];
        x3[3 * i] = p.x;
        x3[3 * i + 1] = p.y;
        x3[3 * i + 2] = p.z;
        if (rad) rad[i] = p.w;
        if (mass) mass[i] = P.mI[s];
    }
}
// Positions, velocity = displacement / T (in plane), zero spin and no contact history.
__global__ void k_to_solver(Particles P, const Ctl *ctl, const double *x3, const double *prev3, double inv_T) {
    const int cur = ctl->cur, vcur = ctl->vcur, cap = P.cap;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        const int s = P.rank[i];
        double4 p = P.pos[cur][s];
        p.x = x3[3 * i];
        p.y = x3[3 * i + 1];
        P.pos[cur][s] = p;
        P.vel[vcur][s] = (x3[3 * i] - prev3[3 * i]) * inv_T;
        P.vel[vcur][cap + s] = (x3[3 * i + 1] - prev3[3 * i + 1]) * inv_T;
        for (int d = 0; d < 3; ++d) P.omg[vcur][d * cap + s] = 0.0;
        P.cstate[s] = 0;
        for (int k = 0; k < P.mc; ++k) P.tidx[(long)k * cap + s] = -1;
        for (long k = 0; k < 3L * P.mc; ++k) P.th[k * cap + s] = 0.0;
        for (long k = 0; k < 3L * P.mw; ++k) P.sw[k * cap + s] = 0.0;
    }
}

}  // namespace

// =======================================================================================
struct dem_surrogate {
    dem_ctx *ctx = nullptr;
    dem_surrogate_params prm{};
    FeatConst fc{};
    // parameters (flat): FP32 master, gradient, Adam moments; BF16 copies
    long np = 0;
    long off[kNL + 1] = {};      // FP32 offsets per layer
    long boff[kNL + 1] = {};     // BF16 offsets per layer
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    bf16 *wb = nullptr;
    long adam_t = 0;
    // graph build
    int cap = 0;                 // node capacity (multiple of 64)
    Particles GP{};
    Particles GA{};              // unused re-sort target
    NbrList L{};
    BuildBuffers B{};
    Ctl *ctl = nullptr;
    int *perm = nullptr, *scene = nullptr;
    double4 *packed = nullptr;
    double2 *disp = nullptr;
    int *offs = nullptr, *bsum = nullptr, *d_total = nullptr;
    long ecap = 0;               // edge capacity
    int *recv = nullptr, *send = nullptr, *rev = nullptr;
    // activations
    bf16 *xn = nullptr, *xe = nullptr;
    bf16 *h[4] = {}, *e[4] = {}, *agg[3] = {};
    bf16 *h1[kNL] = {};
    float *out = nullptr;
    bf16 *dout = nullptr, *dz1 = nullptr, *dyb = nullptr;
    bf16 *pq = nullptr, *dpq = nullptr;   // [nodes][256] P | Q of a message layer and its gradient
    float *dxe = nullptr, *dxn = nullptr, *dh = nullptr, *de = nullptr;
    double *part = nullptr, *d_loss = nullptr;
    // rollout scratch (caller order)
    double *x_prev = nullptr, *x_cur = nullptr, *x_next = nullptr, *x_tmp = nullptr, *rad = nullptr,
           *mass = nullptr;
    int roll_n = 0;
    bool train_ready = false;
};

namespace {

int sg_fail(dem_surrogate *sg, int code, const char *msg) { return ctx_fail(sg->ctx, code, msg); }
#define SCK(call)                                                         \
    do {                                                                  \
        const cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return ctx_cuda(sg->ctx, _e, #call);       \
    } while (0)

#define SG0(call)               \
    do {                        \
        const int _st = (call); \
        if (_st) return _st;    \
    } while (0)

dem_nn_mlp layer_desc(dem_surrogate *sg, int l) {
    const int kin = kShape[l].kin, nout = kShape[l].nout;
    const float *w = sg->w + sg->off[l];
    const bf16 *b = sg->wb + sg->boff[l];
    dem_nn_mlp d{};
    d.kin = kin;
    d.nout = nout;
    d.w1t = b;
    d.w1 = b + (long)kH * kin;
    d.w2t = b + 2L * kH * kin;
    d.w2 = b + 2L * kH * kin + (long)nout * kH;
    d.b1 = w + (long)kH * kin;
    d.b2 = w + (long)kH * kin + kH + (long)nout * kH;
    return d;
}

void grad_ptrs(dem_surrogate *sg, int l, float **gw1t, float **gb1, float **gw2t, float **gb2) {
    const int kin = kShape[l].kin, nout = kShape[l].nout;
    float *gg = sg->g + sg->off[l];
    *gw1t = gg;
    *gb1 = gg + (long)kH * kin;
    *gw2t = gg + (long)kH * kin + kH;
    *gb2 = gg + (long)kH * kin + kH + (long)nout * kH;
}

int refresh_bf16(dem_surrogate *sg) {
    cudaStream_t s = ctx_stream(sg->ctx);
    for (int l = 0; l < kNL; ++l) {
        const int kin = kShape[l].kin, nout = kShape[l].nout;
        const float *w = sg->w + sg->off[l];
        bf16 *b = sg->wb + sg->boff[l];
        k_refresh<<<128, kTB, 0, s>>>(kin, nout, w, w + (long)kH * kin + kH, b, b + (long)kH * kin,
                                      b + 2L * kH * kin, b + 2L * kH * kin + (long)nout * kH);
        if (is_msg(l)) {
            bf16 *x = b + 2L * kH * kin + 2L * nout * kH;
            k_refresh_msg<<<128, kTB, 0, s>>>(w, x, x + kH * kH, x + 2 * kH * kH, x + 4 * kH * kH);
        }
    }
    SCK(cudaGetLastError());
    return DEM_OK;
}

// Node-capacity buffers (graph build, node activations).
int ensure_nodes(dem_surrogate *sg, int n, int nframes) {
    if (n <= sg->cap && nframes <= sg->B.nscenes) return DEM_OK;
    if (n > sg->prm.max_nodes) return sg_fail(sg, DEM_ERR_INVALID, "surrogate: more nodes than max_nodes");
    if (nframes > sg->prm.max_frames) return sg_fail(sg, DEM_ERR_INVALID, "surrogate: more frames than max_frames");
    return sg_fail(sg, DEM_ERR_INVALID, "surrogate: buffers not allocated");
}

int alloc_nodes(dem_surrogate *sg) {
    const int cap = (sg->prm.max_nodes + 63) / 64 * 64;
    const int nf = std::max(1, sg->prm.max_frames);
    sg->cap = cap;
    BuildBuffers &B = sg->B;
    B.cell_cap = (int)std::min<long>(std::max<long>(8L * cap, 32768L), 1L << 28);
    B.nscenes = nf;
    SCK(dmalloc(&B.grid, nf));
    SCK(dmalloc(&B.total, 1));
    SCK(dmalloc(&B.key, cap));
    SCK(dmalloc(&B.cell_start, (size_t)B.cell_cap + 1));
    SCK(dmalloc(&B.cell_fill, (size_t)B.cell_cap + 1));
    SCK(dmalloc(&B.cell_items, cap));
    SCK(dmalloc(&B.block_sums, (size_t)B.cell_cap / 2048 + 2));
    SCK(dmalloc(&B.bbox, 8 * (size_t)nf));
    SCK(dmalloc(&sg->ctl, 1));
    SCK(dmalloc(&sg->perm, cap));
    SCK(dmalloc(&sg->scene, cap));
    SCK(dmalloc(&sg->packed, cap));
    SCK(dmalloc(&sg->disp, cap));
    SCK(dmalloc(&sg->offs, (size_t)cap + 1));
    SCK(dmalloc(&sg->bsum, (size_t)cap / kScanB + 2));
    SCK(dmalloc(&sg->d_total, 1));
    sg->L.maxnb = 32;
    SCK(dmalloc(&sg->L.nn, cap));
    SCK(dmalloc(&sg->L.idx, (size_t)sg->L.maxnb * cap));
    SCK(dmalloc(&sg->xn, (size_t)cap * kF));
    for (int k = 0; k < 4; ++k) SCK(dmalloc(&sg->h[k], (size_t)cap * kH));
    for (int k = 0; k < 3; ++k) SCK(dmalloc(&sg->agg[k], (size_t)cap * kH));
    SCK(dmalloc(&sg->out, (size_t)cap * kF));
    SCK(dmalloc(&sg->pq, (size_t)cap * 2 * kH));
    SCK(dmalloc(&sg->part, 8 * (size_t)std::max(kLossBlocks, kChkBlocks)));
    SCK(dmalloc(&sg->d_loss, 16));
    Particles &P = sg->GP;
    P = Particles{};
    P.n = 0;
    P.cap = cap;
    P.pos[0] = P.pos[1] = sg->packed;
    P.perm = sg->perm;
    return DEM_OK;
}

// Edge-capacity buffers (grown on demand).
int ensure_edges(dem_surrogate *sg, long ne, bool training) {
    const bool need_train = training && !sg->train_ready;
    if (ne <= sg->ecap && !need_train) return DEM_OK;
    const long cap = std::max<long>(ne + ne / 4, sg->ecap);
    cudaStream_t s = ctx_stream(sg->ctx);
    SCK(cudaStreamSynchronize(s));
    if (cap > sg->ecap) {
        cudaFree(sg->recv); cudaFree(sg->send); cudaFree(sg->rev); cudaFree(sg->xe);
        for (int k = 0; k < 4; ++k) cudaFree(sg->e[k]);
        SCK(dmalloc(&sg->recv, cap));
        SCK(dmalloc(&sg->send, cap));
        SCK(dmalloc(&sg->rev, cap));
        SCK(dmalloc(&sg->xe, (size_t)cap * kF));
        for (int k = 0; k < 4; ++k) SCK(dmalloc(&sg->e[k], (size_t)cap * kH));
    }
    if (training && (cap > sg->ecap || !sg->train_ready)) {
        const long rows = std::max<long>(cap, sg->cap);
        for (int l = 0; l < kNL; ++l) cudaFree(sg->h1[l]);
        cudaFree(sg->dz1); cudaFree(sg->dyb); cudaFree(sg->dxe); cudaFree(sg->de);
        for (int l = 0; l < kNL; ++l) {
            const bool edge = (l == L_ENC_E) || (l == L_MSG(0)) || (l == L_MSG(1)) || (l == L_MSG(2));
            SCK(dmalloc(&sg->h1[l], (size_t)(edge ? cap : sg->cap) * kH));
        }
        SCK(dmalloc(&sg->dz1, (size_t)rows * kH));
        SCK(dmalloc(&sg->dyb, (size_t)rows * kH));
        SCK(dmalloc(&sg->dxe, (size_t)cap * kH));
        SCK(dmalloc(&sg->de, (size_t)cap * kH));
        if (!sg->dxn) {
            SCK(dmalloc(&sg->dxn, (size_t)sg->cap * 256));
            SCK(dmalloc(&sg->dh, (size_t)sg->cap * kH));
            SCK(dmalloc(&sg->dout, (size_t)sg->cap * kF));
            SCK(dmalloc(&sg->dpq, (size_t)sg->cap * 2 * kH));
        }
        sg->train_ready = true;
    }
    sg->ecap = cap;
    return DEM_OK;
}

// Graph of the packed positions (sg->packed, sg->GP.n nodes): CSR offs/recv/send/rev.
// Returns the edge count in *ne.
int build_graph(dem_surrogate *sg, int n, const int *frame, int nframes, bool training, long *ne_out) {
    cudaStream_t s = ctx_stream(sg->ctx);
    Particles &P = sg->GP;
    P.n = n;
    P.scene = (frame && nframes > 1) ? sg->scene : nullptr;
    if (P.scene) SCK(cudaMemcpyAsync(sg->scene, frame, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    BuildBuffers B = sg->B;
    B.nscenes = P.scene ? nframes : 1;
    for (int attempt = 0; attempt < 4; ++attempt) {
        SCK(cudaMemsetAsync(sg->ctl, 0, sizeof(Ctl), s));
        launch_build(P, sg->GA, sg->L, B, sg->ctl, sg->prm.radius_graph, 0.0, false, false, s);
        SCK(cudaGetLastError());
        Ctl c{};
        SCK(cudaMemcpyAsync(&c, sg->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
        SCK(cudaStreamSynchronize(s));
        if (c.status & DEM_ERR_NAN) return sg_fail(sg, DEM_ERR_NAN, "surrogate: non-finite positions");
        if (!(c.status & DEM_ERR_NEIGHBOR_OVERFLOW)) break;
        if (c.max_nbr > 128 || attempt == 3) return sg_fail(sg, DEM_ERR_NEIGHBOR_OVERFLOW, "surrogate: > 128 graph neighbours");
        const int want = std::min(std::max(2 * sg->L.maxnb, c.max_nbr + 8), 128);
        cudaFree(sg->L.idx);
        sg->L.maxnb = want;
        SCK(dmalloc(&sg->L.idx, (size_t)want * sg->cap));
    }
    const int nb = (n + kScanB - 1) / kScanB;
    k_scan_block<<<nb, kScanB, 0, s>>>(n, sg->L.nn, sg->offs, sg->bsum);
    k_scan_sums<<<1, kScanB, 0, s>>>(nb, sg->bsum, sg->d_total);
    k_scan_add<<<nb, kScanB, 0, s>>>(n, sg->offs, sg->bsum, sg->d_total);
    int total = 0;
    SCK(cudaMemcpyAsync(&total, sg->d_total, sizeof(int), cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
    int st = ensure_edges(sg, total, training);
    if (st) return st;
    k_csr_fill<<<kGS, kTB, 0, s>>>(n, sg->cap, sg->L.nn, sg->L.idx, sg->offs, sg->recv, sg->send);
    k_csr_rev<<<kGS, kTB, 0, s>>>(total, sg->recv, sg->send, sg->offs, sg->rev);
    SCK(cudaGetLastError());
    *ne_out = total;
    return DEM_OK;
}

int mlp_fwd(dem_surrogate *sg, int l, long rows, const dem_nn_rows *src, int nsrc, const bf16 *resid, bf16 *out,
            float *out_f32, bf16 *h1) {
    int *err;
    float *part;
    int st = ctx_nn_scratch(sg->ctx, 0, &err, &part);
    if (st) return st;
    const dem_nn_mlp d = layer_desc(sg, l);
    st = nn_mlp_forward(d, rows, src, nsrc, resid, out, out_f32, h1, err, ctx_stream(sg->ctx));
    return st ? sg_fail(sg, st, "surrogate: dense layer forward") : DEM_OK;
}

int mlp_bwd(dem_surrogate *sg, int l, long rows, const dem_nn_rows *src, int nsrc, const bf16 *dy, float *dx) {
    int *err;
    float *part;
    int st = ctx_nn_scratch(sg->ctx, nn_wgrad_scratch(kShape[l].kin, kShape[l].nout), &err, &part);
    if (st) return st;
    const dem_nn_mlp d = layer_desc(sg, l);
    float *gw1t, *gb1, *gw2t, *gb2;
    grad_ptrs(sg, l, &gw1t, &gb1, &gw2t, &gb2);
    st = nn_mlp_backward(d, rows, src, nsrc, dy, sg->h1[l], sg->dz1, dx, gw1t, kShape[l].kin, gb1, gw2t, gb2, part,
                         err, ctx_stream(sg->ctx));
    return st ? sg_fail(sg, st, "surrogate: dense layer backward") : DEM_OK;
}

// BF16 copies of a message layer: W1e^T, W1e, W1ij^T, W1ij.
void msg_copies(dem_surrogate *sg, int l, const bf16 **e_t, const bf16 **e, const bf16 **ij_t, const bf16 **ij) {
    const bf16 *x = sg->wb + sg->boff[l] + 2L * kH * 384 + 2L * kH * kH;
    *e_t = x;
    *e = x + kH * kH;
    *ij_t = x + 2 * kH * kH;
    *ij = x + 4 * kH * kH;
}

// e_out = e_in + Msg[e_in, h[recv], h[send]] through PQ = [W1i h | W1j h].
int msg_fwd(dem_surrogate *sg, int l, int n, long ne, const bf16 *h, const bf16 *ein, bf16 *eout, bf16 *h1) {
    int *err;
    float *part;
    SG0(ctx_nn_scratch(sg->ctx, 0, &err, &part));
    const bf16 *e_t, *e, *ij_t, *ij;
    msg_copies(sg, l, &e_t, &e, &ij_t, &ij);
    const dem_nn_mlp d = layer_desc(sg, l);
    cudaStream_t s = ctx_stream(sg->ctx);
    int st = nn_linear_pq(n, h, ij_t, sg->pq, err, s);
    if (!st) st = nn_edge_forward(ne, ein, sg->pq, sg->recv, sg->send, e_t, d.b1, d.w2t, d.b2, eout, h1, err, s);
    return st ? sg_fail(sg, st, "surrogate: message layer forward") : DEM_OK;
}

// Backward of msg_fwd: dy (BF16 [ne][128]) -> dE_in (sg->dxe, FP32 [ne][128]), dh += dMsg/dh,
// weight gradients added.
int msg_bwd(dem_surrogate *sg, int l, int n, long ne, const bf16 *h, const bf16 *ein, const bf16 *dy, float *dh) {
    int *err;
    float *part;
    const long need = std::max(nn_wgrad_scratch(128, 128), nn_linear_wgrad_scratch());
    SG0(ctx_nn_scratch(sg->ctx, need, &err, &part));
    const bf16 *e_t, *e, *ij_t, *ij;
    msg_copies(sg, l, &e_t, &e, &ij_t, &ij);
    const dem_nn_mlp full = layer_desc(sg, l);
    dem_nn_mlp d = full;
    d.kin = 128;
    d.w1t = e_t;
    d.w1 = e;
    float *gw1t, *gb1, *gw2t, *gb2;
    grad_ptrs(sg, l, &gw1t, &gb1, &gw2t, &gb2);
    cudaStream_t s = ctx_stream(sg->ctx);
    dem_nn_rows src{ein, nullptr, kH};
    int st = nn_mlp_backward(d, ne, &src, 1, dy, sg->h1[l], sg->dz1, sg->dxe, gw1t, 384, gb1, gw2t, gb2, part, err, s);
    if (st) return sg_fail(sg, st, "surrogate: message layer backward");
    k_dpq<<<kGS, kTB, 0, s>>>(n, sg->offs, sg->rev, sg->dz1, sg->dpq);
    st = nn_linear_pq_backward(n, sg->dpq, ij, dh, err, s);
    if (!st) st = nn_linear_pq_wgrad(n, sg->dpq, h, gw1t, 384, kH, part, err, s);
    return st ? sg_fail(sg, st, "surrogate: message layer backward") : DEM_OK;
}

#define SG(call)                \
    do {                        \
        const int _st = (call); \
        if (_st) return _st;    \
    } while (0)

// Network forward on the current graph; `training` keeps the hidden activations.
int forward(dem_surrogate *sg, int n, long ne, bool training) {
    cudaStream_t s = ctx_stream(sg->ctx);
    k_node_feat<<<kGS, kTB, 0, s>>>(n, sg->packed, sg->disp, sg->fc, sg->xn);
    if (ne > 0) k_edge_feat<<<kGS, kTB, 0, s>>>((int)ne, sg->recv, sg->send, sg->packed, sg->disp, sg->fc, sg->xe);
    SCK(cudaGetLastError());
    auto H1 = [&](int l) { return training ? sg->h1[l] : nullptr; };
    {
        dem_nn_rows xn{sg->xn, nullptr, kF};
        SG(mlp_fwd(sg, L_ENC_N, n, &xn, 1, nullptr, sg->h[0], nullptr, H1(L_ENC_N)));
        dem_nn_rows xe{sg->xe, nullptr, kF};
        SG(mlp_fwd(sg, L_ENC_E, ne, &xe, 1, nullptr, sg->e[0], nullptr, H1(L_ENC_E)));
    }
    for (int l = 0; l < 3; ++l) {
        // inference keeps two edge latents (ping-pong); training keeps all four
        bf16 *ein = training ? sg->e[l] : sg->e[l & 1];
        bf16 *eout = training ? sg->e[l + 1] : sg->e[(l + 1) & 1];
        SG(msg_fwd(sg, L_MSG(l), n, ne, sg->h[l], ein, eout, H1(L_MSG(l))));
        k_segsum<<<kGS, kTB, 0, s>>>(n, sg->offs, eout, sg->agg[l]);
        dem_nn_rows us[2] = {{sg->h[l], nullptr, kH}, {sg->agg[l], nullptr, kH}};
        SG(mlp_fwd(sg, L_UPD(l), n, us, 2, sg->h[l], sg->h[l + 1], nullptr, H1(L_UPD(l))));
    }
    dem_nn_rows ds{sg->h[3], nullptr, kH};
    SG(mlp_fwd(sg, L_DEC, n, &ds, 1, nullptr, nullptr, sg->out, H1(L_DEC)));
    SCK(cudaGetLastError());
    return DEM_OK;
}

int backward(dem_surrogate *sg, int n, long ne) {
    cudaStream_t s = ctx_stream(sg->ctx);
    SCK(cudaMemsetAsync(sg->g, 0, sizeof(float) * sg->np, s));
    {   // decoder: dh = dDec/dh3
        dem_nn_rows ds{sg->h[3], nullptr, kH};
        SG(mlp_bwd(sg, L_DEC, n, &ds, 1, sg->dout, sg->dh));
    }
    SCK(cudaMemsetAsync(sg->de, 0, sizeof(float) * (size_t)std::max<long>(ne, 1) * kH, s));
    for (int l = 2; l >= 0; --l) {
        // h_{l+1} = h_l + Upd[h_l, agg_l]
        k_f2bf<<<kGS, kTB, 0, s>>>((long)n * kH, sg->dh, sg->dyb);
        dem_nn_rows us[2] = {{sg->h[l], nullptr, kH}, {sg->agg[l], nullptr, kH}};
        SG(mlp_bwd(sg, L_UPD(l), n, us, 2, sg->dyb, sg->dxn));
        k_add_cols<<<kGS, kTB, 0, s>>>(n, sg->dxn, 256, 0, sg->dh);            // dh_l = dh_{l+1} + dUpd/dh_l
        if (ne > 0) {
            // agg_l = sum over edges of e_{l+1}: de_{l+1} += dagg[recv]
            k_edge_from_node<<<kGS, kTB, 0, s>>>((int)ne, sg->recv, sg->dxn, 256, 128, sg->de, 1);
            // e_{l+1} = e_l + Msg[e_l, h_l[recv], h_l[send]]
            k_f2bf<<<kGS, kTB, 0, s>>>(ne * kH, sg->de, sg->dyb);
            SG(msg_bwd(sg, L_MSG(l), n, ne, sg->h[l], sg->e[l], sg->dyb, sg->dh));   // dh += dMsg/dh_l
            k_add_cols<<<kGS, kTB, 0, s>>>(ne, sg->dxe, kH, 0, sg->de);       // de_l = de_{l+1} + dMsg/de_l
        }
    }
    if (ne > 0) {
        k_f2bf<<<kGS, kTB, 0, s>>>(ne * kH, sg->de, sg->dyb);
        dem_nn_rows xe{sg->xe, nullptr, kF};
        SG(mlp_bwd(sg, L_ENC_E, ne, &xe, 1, sg->dyb, nullptr));
    }
    k_f2bf<<<kGS, kTB, 0, s>>>((long)n * kH, sg->dh, sg->dyb);
    dem_nn_rows xn{sg->xn, nullptr, kF};
    SG(mlp_bwd(sg, L_ENC_N, n, &xn, 1, sg->dyb, nullptr));
    SCK(cudaGetLastError());
    return DEM_OK;
}

int prepare_inputs(dem_surrogate *sg, int n, const double *prev, const double *cur, const double *rad, double noise,
                   unsigned long long seed) {
    cudaStream_t s = ctx_stream(sg->ctx);
    k_inputs<<<kGS, kTB, 0, s>>>(n, prev, cur, rad, noise, seed, sg->packed, sg->disp, sg->perm);
    SCK(cudaGetLastError());
    return DEM_OK;
}

int loss_grad(dem_surrogate *sg, int n, const double *prev, const double *cur, const double *next, const double *rad,
              const int *frame, int nframes, double noise, unsigned long long seed, double *loss) {
    SG(ensure_nodes(sg, n, std::max(nframes, 1)));
    SG(prepare_inputs(sg, n, prev, cur, rad, noise, seed));
    long ne = 0;
    SG(build_graph(sg, n, frame, nframes, true, &ne));
    SG(ensure_edges(sg, ne, true));
    SG(forward(sg, n, ne, true));
    cudaStream_t s = ctx_stream(sg->ctx);
    k_loss<<<kLossBlocks, kTB, 0, s>>>(n, sg->out, sg->packed, sg->disp, next, 1.0 / sg->prm.sigma_a, sg->dout, sg->part);
    k_sum_parts<<<1, 32, 0, s>>>(kLossBlocks, sg->part, sg->d_loss);
    SG(backward(sg, n, ne));
    SCK(cudaMemcpyAsync(loss, sg->d_loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
    int *err;
    float *part;
    SG(ctx_nn_scratch(sg->ctx, 0, &err, &part));
    int e = 0;
    SCK(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return sg_fail(sg, e, "surrogate: tensor-core kernel gave up waiting");
    return DEM_OK;
}

// Contact projection of q in place (tmp: scratch of the same size), on the current graph.
int project(dem_surrogate *sg, int n, double *q, double *tmp, const double *rad, const double *mass) {
    cudaStream_t s = ctx_stream(sg->ctx);
    const int it = sg->prm.project_iters;
    for (int k = 0; k < it; ++k) {
        k_project<<<kGS, kTB, 0, s>>>(n, sg->offs, sg->send, k % 2 == 0 ? q : tmp, rad, mass, sg->fc,
                                      sg->prm.project_allow, k % 2 == 0 ? tmp : q);
    }
    if (it % 2 == 1) SCK(cudaMemcpyAsync(q, tmp, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, s));
    SCK(cudaGetLastError());
    return DEM_OK;
}

// One network stride from (sg->x_prev, sg->x_cur) into sg->x_next for the rollout.
// now[0..4] / before[0..4]: largest overlap fraction, kinetic energy, potential energy, total
// mass and largest specific energy of the new state (velocity (next - cur)/T) and of the
// current one.
int net_stride(dem_surrogate *sg, int n, double T, double now[5], double before[5]) {
    cudaStream_t s = ctx_stream(sg->ctx);
    SG(prepare_inputs(sg, n, sg->x_prev, sg->x_cur, sg->rad, 0.0, 0));
    long ne = 0;
    SG(build_graph(sg, n, nullptr, 1, false, &ne));
    SG(forward(sg, n, ne, false));
    k_integrate<<<kGS, kTB, 0, s>>>(n, sg->packed, sg->disp, sg->out, sg->prm.sigma_a, sg->fc, sg->x_cur, sg->x_next);
    SG(project(sg, n, sg->x_next, sg->x_tmp, sg->rad, sg->mass));
    const double gx = sg->prm.gravity[0], gy = sg->prm.gravity[1];
    k_check<<<kChkBlocks, kTB, 0, s>>>(n, sg->offs, sg->send, sg->x_next, sg->rad, sg->mass, sg->fc, 1.0 / T, gx, gy,
                                       sg->x_cur, sg->part);
    k_check_sum<<<1, 32, 0, s>>>(kChkBlocks, sg->part, sg->d_loss);
    k_check<<<kChkBlocks, kTB, 0, s>>>(n, sg->offs, sg->send, sg->x_cur, sg->rad, sg->mass, sg->fc, 1.0 / T, gx, gy,
                                       sg->x_prev, sg->part);
    k_check_sum<<<1, 32, 0, s>>>(kChkBlocks, sg->part, sg->d_loss + 5);
    SCK(cudaGetLastError());
    double v[10];
    SCK(cudaMemcpyAsync(v, sg->d_loss, 10 * sizeof(double), cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
    for (int k = 0; k < 5; ++k) {
        now[k] = v[k];
        before[k] = v[5 + k];
    }
    return DEM_OK;
}

}  // namespace

// =======================================================================================
extern "C" int dem_surrogate_create(dem_ctx *ctx, const dem_surrogate_params *prm, dem_surrogate **out) {
    if (!ctx || !prm || !out) return DEM_ERR_INVALID;
    *out = nullptr;
    if (!(prm->radius_graph > 0.0) || prm->steps_per_stride <= 0 || !(prm->dt > 0.0) || !(prm->sigma_d > 0.0) ||
        !(prm->sigma_a > 0.0) || !(prm->r_mean > 0.0) || !(prm->r_std > 0.0) || prm->nwalls < 0 ||
        prm->nwalls > kSgWalls || prm->max_nodes <= 0 || !(prm->wall_clip > 0.0) || prm->project_iters < 0 ||
        prm->project_iters > 64 || !(prm->project_allow >= 0.0))
        return ctx_fail(ctx, DEM_ERR_INVALID, "dem_surrogate_create: bad parameters");
    dem_surrogate *sg = new dem_surrogate();
    sg->ctx = ctx;
    sg->prm = *prm;
    if (sg->prm.max_frames <= 0) sg->prm.max_frames = 1;
    FeatConst &fc = sg->fc;
    fc.inv_rg = 1.0 / prm->radius_graph;
    fc.inv_sd = 1.0 / prm->sigma_d;
    fc.sigma_a = prm->sigma_a;
    fc.r_mean = prm->r_mean;
    fc.inv_r_mean = 1.0 / prm->r_mean;
    fc.inv_r_std = 1.0 / prm->r_std;
    fc.inv_clip = 1.0 / prm->wall_clip;
    fc.nwalls = prm->nwalls;
    for (int w = 0; w < prm->nwalls; ++w) {
        const double nx = prm->wall_n[w][0], ny = prm->wall_n[w][1];
        const double len = std::sqrt(nx * nx + ny * ny);
        if (!(len > 0.0)) {
            delete sg;
            return ctx_fail(ctx, DEM_ERR_INVALID, "dem_surrogate_create: wall normal has no in-plane part");
        }
        fc.wx[w][0] = prm->wall_x[w][0];
        fc.wx[w][1] = prm->wall_x[w][1];
        fc.wn[w][0] = nx / len;
        fc.wn[w][1] = ny / len;
    }
    long o = 0, b = 0;
    for (int l = 0; l < kNL; ++l) {
        sg->off[l] = o;
        sg->boff[l] = b;
        const long kin = kShape[l].kin, nout = kShape[l].nout;
        o += kH * kin + kH + nout * kH + nout;
        b += 2 * (kH * kin) + 2 * (nout * kH);
        if (is_msg(l)) b += 2L * kH * kH + 2L * 2 * kH * kH;   // W1e^T, W1e, W1ij^T, W1ij
    }
    sg->off[kNL] = o;
    sg->boff[kNL] = b;
    sg->np = o;
    int st = DEM_OK;
    auto A = [&](cudaError_t e) {
        if (st == DEM_OK && e != cudaSuccess) st = ctx_cuda(ctx, e, "dem_surrogate_create");
    };
    A(dmalloc(&sg->w, o));
    A(dmalloc(&sg->g, o));
    A(dmalloc(&sg->m, o));
    A(dmalloc(&sg->v, o));
    A(dmalloc(&sg->wb, b));
    if (st == DEM_OK) st = alloc_nodes(sg);
    if (st == DEM_OK) {
        cudaStream_t s = ctx_stream(ctx);
        A(cudaMemsetAsync(sg->m, 0, sizeof(float) * o, s));
        A(cudaMemsetAsync(sg->v, 0, sizeof(float) * o, s));
        A(cudaMemsetAsync(sg->g, 0, sizeof(float) * o, s));
    }
    if (st == DEM_OK) st = dem_surrogate_init_params(sg, 1);
    if (st) {
        dem_surrogate_destroy(sg);
        return st;
    }
    *out = sg;
    return DEM_OK;
}

extern "C" int dem_surrogate_destroy(dem_surrogate *sg) {
    if (!sg) return DEM_ERR_INVALID;
    cudaStreamSynchronize(ctx_stream(sg->ctx));
    void *ptrs[] = {sg->w, sg->g, sg->m, sg->v, sg->wb, sg->ctl, sg->perm, sg->scene, sg->packed, sg->disp, sg->offs,
                    sg->bsum, sg->d_total, sg->recv, sg->send, sg->rev, sg->xn, sg->xe, sg->out, sg->dout, sg->dz1,
                    sg->dyb, sg->dxe, sg->dxn, sg->dh, sg->de, sg->pq, sg->dpq, sg->part, sg->d_loss, sg->x_prev, sg->x_cur,
                    sg->x_next, sg->x_tmp, sg->rad, sg->mass, sg->L.nn, sg->L.idx, sg->B.grid, sg->B.total, sg->B.key,
                    sg->B.cell_start, sg->B.cell_fill, sg->B.cell_items, sg->B.block_sums, sg->B.bbox};
    for (void *p : ptrs) cudaFree(p);
    for (int k = 0; k < 4; ++k) {
        cudaFree(sg->h[k]);
        cudaFree(sg->e[k]);
    }
    for (int k = 0; k < 3; ++k) cudaFree(sg->agg[k]);
    for (int l = 0; l < kNL; ++l) cudaFree(sg->h1[l]);
    delete sg;
    return DEM_OK;
}

extern "C" long dem_surrogate_num_params(dem_surrogate *sg) { return sg ? sg->np : -1; }

extern "C" int dem_surrogate_get_params(dem_surrogate *sg, float *host, long n) {
    if (!sg || !host || n != sg->np) return DEM_ERR_INVALID;
    cudaStream_t s = ctx_stream(sg->ctx);
    SCK(cudaMemcpyAsync(host, sg->w, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    SCK(cudaStreamSynchronize(s));
    return DEM_OK;
}

extern "C" int dem_surrogate_set_params(dem_surrogate *sg, const float *host, long n) {
    if (!sg || !host || n != sg->np) return DEM_ERR_INVALID;
    cudaStream_t s = ctx_stream(sg->ctx);
    SCK(cudaMemcpyAsync(sg->w, host, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    SCK(cudaMemsetAsync(sg->m, 0, sizeof(float) * n, s));
    SCK(cudaMemsetAsync(sg->v, 0, sizeof(float) * n, s));
    sg->adam_t = 0;
    SG(refresh_bf16(sg));
    SCK(cudaStreamSynchronize(s));
    return DEM_OK;
}

// He-normal first layers, residual branches and the decoder scaled down (seeded, host RNG).
extern "C" int dem_surrogate_init_params(dem_surrogate *sg, unsigned long long seed) {
    if (!sg) return DEM_ERR_INVALID;
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    std::vector<float> w((size_t)sg->np, 0.f);
    for (int l = 0; l < kNL; ++l) {
        const int kin = kShape[l].kin, nout = kShape[l].nout;
        float *p = w.data() + sg->off[l];
        const float s1 = std::sqrt(2.f / (float)kin);
        const float s2 = std::sqrt(1.f / (float)kH) * (l == L_DEC ? 0.1f : (l >= 2 ? 0.5f : 1.f));
        for (long k = 0; k < (long)kH * kin; ++k) p[k] = s1 * nd(rng);
        float *w2 = p + (long)kH * kin + kH;
        for (long k = 0; k < (long)nout * kH; ++k) w2[k] = s2 * nd(rng);
    }
    return dem_surrogate_set_params(sg, w.data(), sg->np);
}

extern "C" int dem_surrogate_loss_grad(dem_surrogate *sg, int n, const double *pos_prev, const double *pos_cur,
                                       const double *pos_next, const double *rad, const int *frame, int nframes,
                                       double noise, unsigned long long seed, double *loss, float *grads_host) {
    if (!sg || n <= 0 || !pos_prev || !pos_cur || !pos_next || !rad || !loss) return DEM_ERR_INVALID;
    SG(loss_grad(sg, n, pos_prev, pos_cur, pos_next, rad, frame, nframes, noise, seed, loss));
    if (grads_host) {
        cudaStream_t s = ctx_stream(sg->ctx);
        SCK(cudaMemcpyAsync(grads_host, sg->g, sizeof(float) * sg->np, cudaMemcpyDeviceToHost, s));
        SCK(cudaStreamSynchronize(s));
    }
    return DEM_OK;
}

extern "C" int dem_surrogate_train_step(dem_surrogate *sg, int n, const double *pos_prev, const double *pos_cur,
                                        const double *pos_next, const double *rad, const int *frame, int nframes,
                                        double noise, unsigned long long seed, double lr, double *loss) {
    if (!sg || n <= 0 || !pos_prev || !pos_cur || !pos_next || !rad || !loss) return DEM_ERR_INVALID;
    SG(loss_grad(sg, n, pos_prev, pos_cur, pos_next, rad, frame, nframes, noise, seed, loss));
    sg->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)sg->adam_t), c2 = 1.f - std::pow(b2, (float)sg->adam_t);
    cudaStream_t s = ctx_stream(sg->ctx);
    k_adam<<<kGS, kTB, 0, s>>>(sg->np, sg->w, sg->g, sg->m, sg->v, (float)lr, b1, b2, 1e-8f, c1, c2);
    SCK(cudaGetLastError());
    return refresh_bf16(sg);
}

extern "C" int dem_surrogate_predict(dem_surrogate *sg, int n, const double *pos_prev, const double *pos_cur,
                                     const double *rad, const int *frame, int nframes, double *pos_next) {
    if (!sg || n <= 0 || !pos_prev || !pos_cur || !rad || !pos_next) return DEM_ERR_INVALID;
    SG(ensure_nodes(sg, n, std::max(nframes, 1)));
    SG(prepare_inputs(sg, n, pos_prev, pos_cur, rad, 0.0, 0));
    long ne = 0;
    SG(build_graph(sg, n, frame, nframes, false, &ne));
    SG(forward(sg, n, ne, false));
    cudaStream_t s = ctx_stream(sg->ctx);
    k_integrate<<<kGS, kTB, 0, s>>>(n, sg->packed, sg->disp, sg->out, sg->prm.sigma_a, sg->fc, pos_cur, pos_next);
    if (sg->prm.project_iters > 0) {
        double *tmp = nullptr, *w = nullptr;
        SCK(dmalloc(&tmp, 3 * (size_t)n));
        SCK(dmalloc(&w, (size_t)n));
        k_rad3<<<kGS, kTB, 0, s>>>(n, rad, w);   // mass weights of equal-density particles
        const int st = project(sg, n, pos_next, tmp, rad, w);
        SCK(cudaStreamSynchronize(s));
        cudaFree(tmp);
        cudaFree(w);
        if (st) return st;
    }
    SCK(cudaGetLastError());
    SCK(cudaStreamSynchronize(s));
    return DEM_OK;
}

extern "C" int dem_surrogate_rollout(dem_surrogate *sg, dem_solver *solver, int nstrides, int use_network,
                                     dem_rollout_stats *stats) {
    if (!sg || !solver || nstrides < 0) return DEM_ERR_INVALID;
    dem_rollout_stats st{};
    SolverView V{};
    SG(solver_view(solver, &V));
    const int n = V.P.n;
    SG(ensure_nodes(sg, n, 1));
    cudaStream_t s = ctx_stream(sg->ctx);
    if (V.stream != s) return sg_fail(sg, DEM_ERR_INVALID, "dem_surrogate_rollout: solver and surrogate need one context");
    if (sg->roll_n < n) {
        cudaFree(sg->x_prev); cudaFree(sg->x_cur); cudaFree(sg->x_next); cudaFree(sg->x_tmp); cudaFree(sg->rad);
        cudaFree(sg->mass);
        SCK(dmalloc(&sg->x_prev, 3 * (size_t)n));
        SCK(dmalloc(&sg->x_tmp, 3 * (size_t)n));
        SCK(dmalloc(&sg->x_cur, 3 * (size_t)n));
        SCK(dmalloc(&sg->x_next, 3 * (size_t)n));
        SCK(dmalloc(&sg->rad, n));
        SCK(dmalloc(&sg->mass, n));
        sg->roll_n = n;
    }
    const int steps = sg->prm.steps_per_stride;
    const double T = steps * sg->prm.dt;
    auto dem_stride = [&]() -> int {
        k_from_solver<<<kGS, kTB, 0, s>>>(V.P, V.ctl, sg->x_prev, sg->rad, sg->mass);
        SCK(cudaGetLastError());
        const int rs = dem_solver_run(solver, steps);
        if (rs) return rs;
        SG(solver_view(solver, &V));
        k_from_solver<<<kGS, kTB, 0, s>>>(V.P, V.ctl, sg->x_cur, nullptr, nullptr);
        SCK(cudaGetLastError());
        st.strides_dem += 1;
        return DEM_OK;
    };
    bool solver_stale = false;   // the surrogate's state is newer than the solver's
    double e_floor = 0.0;        // lowest mechanical energy since the last DEM stride
    double s_floor = 0.0;        // lowest largest-specific-energy since the last DEM stride
    bool have_floor = false;
    for (int k = 0; k < nstrides; ++k) {
        if (k == 0 || !use_network) {
            SG(dem_stride());
            have_floor = false;
            continue;
        }
        double now[5], before[5];
        SG(net_stride(sg, n, T, now, before));
        // energy residual: the mechanical energy of a dissipative granular flow does not rise; a
        // network stride may not lift it above the lowest value since the last DEM stride by
        // more than energy_tol x (total weight x mean radius), so gains cannot accumulate.  The
        // same per particle: the largest specific energy (0.5 |v|^2 + lift) may not rise above
        // its lowest value since the last DEM stride by more than the lift of one diameter, so a
        // few particles thrown by the network cannot hide inside the total.
        const double g = std::sqrt(sg->prm.gravity[0] * sg->prm.gravity[0] + sg->prm.gravity[1] * sg->prm.gravity[1]);
        const double escale = now[3] * g * sg->prm.r_mean;
        if (!have_floor) {
            e_floor = before[1] + before[2];
            s_floor = before[4];
            have_floor = true;
        }
        const double e_new = now[1] + now[2];
        const bool bad_overlap = !(now[0] <= sg->prm.max_overlap);
        const bool bad_energy = !(e_new <= e_floor + sg->prm.energy_tol * escale) ||
                                !(now[4] <= s_floor + 2.0 * g * sg->prm.r_mean);
        if (!bad_overlap && !bad_energy) {
            std::swap(sg->x_prev, sg->x_cur);   // prev <- cur
            std::swap(sg->x_cur, sg->x_next);   // cur <- next
            e_floor = std::min(e_floor, e_new);
            s_floor = std::min(s_floor, now[4]);
            st.strides_network += 1;
            st.max_overlap_seen = std::max(st.max_overlap_seen, now[0]);
            solver_stale = true;
            continue;
        }
        if (bad_overlap) st.fallback_overlap += 1;
        else st.fallback_energy += 1;
        if (solver_stale) {
            k_to_solver<<<kGS, kTB, 0, s>>>(V.P, V.ctl, sg->x_cur, sg->x_prev, 1.0 / T);
            SCK(cudaGetLastError());
            solver_particles_changed(solver);
            solver_stale = false;
        }
        SG(dem_stride());
        have_floor = false;   // the next network stride starts from this DEM state's energy
    }
    if (solver_stale) {
        k_to_solver<<<kGS, kTB, 0, s>>>(V.P, V.ctl, sg->x_cur, sg->x_prev, 1.0 / T);
        SCK(cudaGetLastError());
        solver_particles_changed(solver);
    }
    SCK(cudaStreamSynchronize(s));
    if (stats) *stats = st;
    return DEM_OK;
}
