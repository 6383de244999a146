// dem_nbr.cu -- cell-list Verlet neighbour build on sm_100a (replaces Cabana's
// VerletList<FullNeighborTag, VerletLayout2D> used at src/CabanaDEM_Solver.hpp:61-63,
// :87-88 and src/CabanaBondedDEM_Particles.hpp:155-157).
//
// Pipeline (all on the device, no host round trip, so it can sit in a CUDA graph):
//   bbox      min/max of positions and max radius (ordered-integer atomics)
//   grid      cell size >= largest cutoff, Morton cell keys when they fit the table
//   count     particles per cell key;  scan  exclusive prefix sum (3 kernels)
//   fill      particle slots per cell; per-cell insertion sort by caller index
//   [resort]  permute all particle state into cell-key (Morton) order, remap partners
//   list      per particle: 27-cell stencil, keep j != i with |x_i - x_j| <= cutoff,
//             sorted by caller index (the oracle's summation order)
// Built with --fmad=false so that the distance test matches the oracle's.
#include "dem_internal.cuh"
#include "b200dem.h"

namespace b200dem {

namespace {

constexpr int kB = 256;
constexpr int kScanItems = 8;                 // per thread
constexpr int kScanTile = kB * kScanItems;    // 2048 keys per block
constexpr int kMaxCand = 128;                 // candidates kept per particle while sorting

struct __align__(32) D4 {
    double x, y, z, w;
};
__device__ __forceinline__ D4 ld4(const double4 *p, int i) { return reinterpret_cast<const D4 *>(p)[i]; }

__device__ __forceinline__ unsigned long long ord(double x) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord(unsigned long long o) {
    const unsigned long long b = (o & 0x8000000000000000ull) ? (o & 0x7fffffffffffffffull) : ~o;
    return __longlong_as_double((long long)b);
}

__device__ __forceinline__ unsigned part1by2(unsigned x) {
    x &= 0x3ff;
    x = (x | (x << 16)) & 0x030000FF;
    x = (x | (x << 8)) & 0x0300F00F;
    x = (x | (x << 4)) & 0x030C30C3;
    x = (x | (x << 2)) & 0x09249249;
    return x;
}

__device__ __forceinline__ int cell_key(const Grid &g, int cx, int cy, int cz) {
    if (g.bits > 0)
        return g.base + (int)(part1by2((unsigned)cx) | (part1by2((unsigned)cy) << 1) | (part1by2((unsigned)cz) << 2));
    return g.base + (cz * g.dims[1] + cy) * g.dims[0] + cx;
}

__device__ __forceinline__ void cell_of(const Grid &g, const D4 &p, int c[3]) {
    const double xs[3] = {p.x, p.y, p.z};
    for (int d = 0; d < 3; ++d) {
        int v = (int)floor((xs[d] - g.lo[d]) * g.inv_cell);
        v = v < 0 ? 0 : (v >= g.dims[d] ? g.dims[d] - 1 : v);
        c[d] = v;
    }
}

__device__ __forceinline__ int scene_of(const Particles &P, int i) { return P.scene ? P.scene[i] : 0; }

// 8 ordered-integer words per scene: lo[3], hi[3], rmax, unused
__global__ void k_bbox_init(unsigned long long *bb, int nscenes) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 8 * nscenes; t += gridDim.x * blockDim.x) {
        const int k = t & 7;
        bb[t] = k < 3 ? ord(1e300) : (k < 6 ? ord(-1e300) : ord(0.0));
    }
}

__global__ void k_bbox(Particles P, const Ctl *ctl, unsigned long long *bb) {
    const int cur = ctl->cur;
    if (!P.scene) {   // one scene: block reduction, one atomic per word per block
        __shared__ unsigned long long s[7];
        if (threadIdx.x < 7) s[threadIdx.x] = threadIdx.x < 3 ? ord(1e300) : (threadIdx.x < 6 ? ord(-1e300) : ord(0.0));
        __syncthreads();
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
            const D4 p = ld4(P.pos[cur], i);
            atomicMin(&s[0], ord(p.x));
            atomicMin(&s[1], ord(p.y));
            atomicMin(&s[2], ord(p.z));
            atomicMax(&s[3], ord(p.x));
            atomicMax(&s[4], ord(p.y));
            atomicMax(&s[5], ord(p.z));
            atomicMax(&s[6], ord(p.w));
        }
        __syncthreads();
        if (threadIdx.x < 3) atomicMin(&bb[threadIdx.x], s[threadIdx.x]);
        else if (threadIdx.x < 7) atomicMax(&bb[threadIdx.x], s[threadIdx.x]);
        return;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        const D4 p = ld4(P.pos[cur], i);
        unsigned long long *w = bb + 8L * P.scene[i];
        atomicMin(&w[0], ord(p.x));
        atomicMin(&w[1], ord(p.y));
        atomicMin(&w[2], ord(p.z));
        atomicMax(&w[3], ord(p.x));
        atomicMax(&w[4], ord(p.y));
        atomicMax(&w[5], ord(p.z));
        atomicMax(&w[6], ord(p.w));
    }
}

// Per-scene grids: cell >= the largest cutoff of the scene, Morton keys when every scene's
// Morton range fits the table, else linear keys, else larger cells; scene s's keys start at
// grid[s].base.  One block.  A non-finite extent (a blown-up state) or a table that no cell
// size fits gives every scene one cell and raises DEM_ERR_NAN; the cell sort and the list
// kernels then skip their work, so the build stays bounded.
__device__ bool scene_dims(const unsigned long long *w, double cell, double lo[3], int dims[3], int &bits,
                           long long &morton_codes, long long &linear_codes) {
    double hi[3];
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
        lo[d] = unord(w[d]);
        hi[d] = unord(w[3 + d]);
        if (isnan(lo[d]) || isnan(hi[d]) || isinf(hi[d] - lo[d])) ok = false;
        if (!(hi[d] >= lo[d]) || !ok) lo[d] = hi[d] = 0.0;   // empty scene, or no usable extent
    }
    int dmax = 1;
    linear_codes = 1;
    for (int d = 0; d < 3; ++d) {
        const double e = floor((hi[d] - lo[d]) / cell) + 1.0;
        dims[d] = (int)fmin(e, 1e9);
        dims[d] = dims[d] < 1 ? 1 : dims[d];
        dmax = max(dmax, dims[d]);
        linear_codes *= dims[d];
        if (linear_codes > (1LL << 40)) linear_codes = 1LL << 40;
    }
    bits = 1;
    while ((1 << bits) < dmax) ++bits;
    morton_codes = bits <= 10 ? (1LL << (3 * bits)) : (1LL << 40);
    return ok;
}

__global__ void k_grid(const unsigned long long *bb, Grid *grid, int *total, int nscenes, int cell_cap, double delta,
                       double skin, Ctl *ctl) {
    __shared__ long long sm[256], sl[256];
    __shared__ int bad[256];
    __shared__ double factor;
    __shared__ int use_morton, done, invalid;
    if (threadIdx.x == 0) {
        factor = 1.0;
        done = 0;
        use_morton = 0;
        invalid = 0;
    }
    __syncthreads();
    for (int it = 0; it < 200 && !done; ++it) {
        long long tm = 0, tl = 0;
        int nb = 0;
        for (int sc = threadIdx.x; sc < nscenes; sc += blockDim.x) {
            const double rmax = unord(bb[8L * sc + 6]);
            const double cut = delta > 0.0 ? delta : 2.0 * rmax + skin;
            const double cell = (cut > 0.0 ? cut : 1.0) * factor;
            double lo[3];
            int dims[3], bits;
            long long mc, lc;
            if (!scene_dims(bb + 8L * sc, cell, lo, dims, bits, mc, lc) || !(cell < 1e300)) ++nb;
            tm += mc;
            tl += lc;
        }
        sm[threadIdx.x] = tm;
        sl[threadIdx.x] = tl;
        bad[threadIdx.x] = nb;
        __syncthreads();
        if (threadIdx.x == 0) {
            long long a = 0, b = 0;
            int nbad = 0;
            for (int t = 0; t < (int)blockDim.x; ++t) {
                a += sm[t];
                b += sl[t];
                nbad += bad[t];
            }
            if (nbad > 0 && it == 0) {   // non-finite extent: no cell size helps
                invalid = 1;
                done = 1;
            } else if (a <= cell_cap) {
                use_morton = 1;
                done = 1;
            } else if (b <= cell_cap) {
                use_morton = 0;
                done = 1;
            } else {
                factor *= 1.26;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && !done) invalid = 1;
    __syncthreads();
    for (int sc = threadIdx.x; sc < nscenes; sc += blockDim.x) {
        Grid G;
        const double rmax = unord(bb[8L * sc + 6]);
        const double cut = delta > 0.0 ? delta : 2.0 * rmax + skin;
        G.cell = (cut > 0.0 ? cut : 1.0) * factor;
        G.inv_cell = 1.0 / G.cell;
        G.rmax = rmax;
        long long mc, lc;
        int bits;
        scene_dims(bb + 8L * sc, G.cell, G.lo, G.dims, bits, mc, lc);
        G.bits = use_morton ? bits : 0;
        G.ncodes = (int)(use_morton ? mc : lc);
        if (invalid) {
            G.dims[0] = G.dims[1] = G.dims[2] = 1;
            G.bits = 0;
            G.ncodes = 1;
        }
        G.base = 0;
        grid[sc] = G;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int sc = 0; sc < nscenes; ++sc) {
            grid[sc].base = run;
            run += grid[sc].ncodes;
        }
        *total = run;
        if (invalid) atomicOr(&ctl->status, DEM_ERR_NAN);
    }
}

__global__ void k_zero(int *a, const int *total) {
    const int n = *total + 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = 0;
}

__global__ void k_count(Particles P, const Ctl *ctl, const Grid *grid, int *key, int *cnt) {
    const int cur = ctl->cur;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        const Grid &G = grid[scene_of(P, i)];
        int c[3];
        cell_of(G, ld4(P.pos[cur], i), c);
        const int k = cell_key(G, c[0], c[1], c[2]);
        key[i] = k;
        atomicAdd(&cnt[k], 1);
    }
}

// Exclusive scan of cnt[0..total) into start[0..total]; 3 passes.
__global__ void k_scan_tiles(const int *cnt, int *start, int *sums, const int *total) {
    __shared__ int s[kB];
    const int n = *total;
    const long base = (long)blockIdx.x * kScanTile;
    if (base >= n) return;
    int v[kScanItems];
    int t = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const long idx = base + (long)threadIdx.x * kScanItems + k;
        v[k] = idx < n ? cnt[idx] : 0;
        t += v[k];
    }
    s[threadIdx.x] = t;
    __syncthreads();
    for (int o = 1; o < kB; o <<= 1) {
        const int a = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += a;
        __syncthreads();
    }
    int run = s[threadIdx.x] - t;
    for (int k = 0; k < kScanItems; ++k) {
        const long idx = base + (long)threadIdx.x * kScanItems + k;
        if (idx < n) start[idx] = run;
        run += v[k];
    }
    if (threadIdx.x == kB - 1) sums[blockIdx.x] = s[kB - 1];
}

__global__ void k_scan_sums(int *sums, const int *total, int *start) {
    // single block of kB threads; the tile sums are scanned kB at a time
    __shared__ int s[kB];
    const int n = *total;
    const int tiles = (n + kScanTile - 1) / kScanTile;
    int carry = 0;
    for (int base = 0; base < tiles; base += kB) {
        const int idx = base + threadIdx.x;
        const int v = idx < tiles ? sums[idx] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < kB; o <<= 1) {
            const int a = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += a;
            __syncthreads();
        }
        if (idx < tiles) sums[idx] = carry + s[threadIdx.x] - v;
        const int tot = s[kB - 1];
        __syncthreads();
        carry += tot;
    }
    if (threadIdx.x == 0) start[n] = carry;
}

__global__ void k_scan_add(int *start, int *fill, const int *sums, const int *total) {
    const int n = *total;
    const long base = (long)blockIdx.x * kScanTile;
    if (base >= n) return;
    const int add = sums[blockIdx.x];
    for (int k = threadIdx.x; k < kScanTile; k += blockDim.x) {
        const long idx = base + k;
        if (idx < n) {
            const int v = start[idx] + add;
            start[idx] = v;
            fill[idx] = v;
        }
    }
}

__global__ void k_fill(int n, const int *key, int *fill, int *items) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = atomicAdd(&fill[key[i]], 1);
        items[slot] = i;
    }
}

// Deterministic order inside each cell: ascending caller index.
__global__ void k_cell_sort(const int *start, int *items, const int *perm, const int *total, const Ctl *ctl) {
    if (ctl->status & DEM_ERR_NAN) return;   // one cell per scene: the list is not built
    const int n = *total;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int b = start[c], e = start[c + 1];
        for (int a = b + 1; a < e; ++a) {
            const int v = items[a];
            const int kv = perm[v];
            int t = a - 1;
            while (t >= b && perm[items[t]] > kv) {
                items[t + 1] = items[t];
                --t;
            }
            items[t + 1] = v;
        }
    }
}

// Re-sort: new index p takes old particle src[p] = items[p].
__global__ void k_make_dst(int n, const int *items, int *dst) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) dst[items[p]] = p;
}

__global__ void k_permute(Particles P, Particles A, const Ctl *ctl, const int *items, const int *dst) {
    const int n = P.n, cap = P.cap, cur = ctl->cur, nxt = cur ^ 1, vcur = ctl->vcur, vnxt = vcur ^ 1;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int q = items[p];
        reinterpret_cast<D4 *>(P.pos[nxt])[p] = ld4(P.pos[cur], q);
        for (int d = 0; d < 3; ++d) {
            P.vel[vnxt][d * cap + p] = P.vel[vcur][d * cap + q];
            P.omg[vnxt][d * cap + p] = P.omg[vcur][d * cap + q];
            A.force[d * cap + p] = P.force[d * cap + q];
            A.torque[d * cap + p] = P.torque[d * cap + q];
            if (P.ext) A.ext[d * cap + p] = P.ext[d * cap + q];
        }
        A.mI[p] = P.mI[q];
        A.mI[cap + p] = P.mI[cap + q];
        A.mat[p] = P.mat[q];
        if (P.scene) A.scene[p] = P.scene[q];
        A.fix[p] = P.fix[q];
        const int cs = P.cstate[q];
        A.cstate[p] = cs;
        // live history only: the tracked slots below the contact count and the walls whose
        // history bit is set (every other slot holds -1 / 0, see k_hist_back)
        const int cnt = cs & 0xff;
        const unsigned wm = (unsigned)cs >> 8;
        for (int k = 0; k < cnt; ++k) {
            const int t = P.tidx[(long)k * cap + q];
            A.tidx[(long)k * cap + p] = (t >= 0 && t < n) ? dst[t] : t;
            for (int d = 0; d < 3; ++d) A.th[((long)d * P.mc + k) * cap + p] = P.th[((long)d * P.mc + k) * cap + q];
        }
        for (int w = 0; w < P.mw; ++w)
            if ((wm >> w) & 1u)
                for (int d = 0; d < 3; ++d) A.sw[((long)d * P.mw + w) * cap + p] = P.sw[((long)d * P.mw + w) * cap + q];
        const int orig = P.perm[q];
        A.perm[p] = orig;
        P.rank[orig] = p;
    }
}

// Re-sort, history back into place: slot p takes the live slots k_permute gathered for its new
// particle, and the slots its previous particle used beyond them are reset (partner -1,
// history 0), so that every slot past a particle's contact count, and every wall slot whose
// history bit is clear, keeps holding -1 / 0 as the contact kernels leave them.  Reads the
// old contact word at p (P.cstate, before it is replaced by the gathered one).
__global__ void k_hist_back(Particles P, Particles A) {
    const int n = P.n, cap = P.cap;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int nc = A.cstate[p], oc = P.cstate[p];
        const int ncnt = nc & 0xff, ocnt = oc & 0xff;
        for (int k = 0; k < ncnt; ++k) {
            P.tidx[(long)k * cap + p] = A.tidx[(long)k * cap + p];
            for (int d = 0; d < 3; ++d) P.th[((long)d * P.mc + k) * cap + p] = A.th[((long)d * P.mc + k) * cap + p];
        }
        for (int k = ncnt; k < ocnt; ++k) {
            P.tidx[(long)k * cap + p] = -1;
            for (int d = 0; d < 3; ++d) P.th[((long)d * P.mc + k) * cap + p] = 0.;
        }
        const unsigned nm = (unsigned)nc >> 8, om = (unsigned)oc >> 8;
        for (int w = 0; w < P.mw; ++w) {
            if ((nm >> w) & 1u)
                for (int d = 0; d < 3; ++d) P.sw[((long)d * P.mw + w) * cap + p] = A.sw[((long)d * P.mw + w) * cap + p];
            else if ((om >> w) & 1u)
                for (int d = 0; d < 3; ++d) P.sw[((long)d * P.mw + w) * cap + p] = 0.;
        }
    }
}

__global__ void k_flip(Ctl *ctl) {
    if (threadIdx.x == 0) {
        ctl->cur ^= 1;
        ctl->vcur ^= 1;
    }
}

__global__ void __launch_bounds__(128) k_list(Particles P, NbrList L, Ctl *ctl, const Grid *g, const int *start,
                                              const int *items, double delta, double skin) {
    const int cur = ctl->cur, cap = P.cap;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool invalid = (ctl->status & DEM_ERR_NAN) != 0;
    int count = 0;
    if (i < P.n && invalid) L.nn[i] = 0;
    if (i < P.n && !invalid) {
        const Grid G = g[scene_of(P, i)];
        const double4 *pc = P.pos[cur];
        const D4 pi = ld4(pc, i);
        int c[3];
        cell_of(G, pi, c);
        int cand[kMaxCand];
        int ckey[kMaxCand];
        for (int dz = -1; dz <= 1; ++dz) {
            const int z = c[2] + dz;
            if (z < 0 || z >= G.dims[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int y = c[1] + dy;
                if (y < 0 || y >= G.dims[1]) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = c[0] + dx;
                    if (x < 0 || x >= G.dims[0]) continue;
                    const int key = cell_key(G, x, y, z);
                    const int e = start[key + 1];
                    for (int s = start[key]; s < e; ++s) {
                        const int j = items[s];
                        if (j == i) continue;
                        const D4 pj = ld4(pc, j);
                        const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
                        const double r2 = px * px + py * py + pz * pz;
                        const double cut = delta > 0.0 ? delta : pi.w + pj.w + skin;
                        if (r2 <= cut * cut) {
                            if (count < kMaxCand) {
                                // insertion by caller index
                                const int kj = P.perm[j];
                                int t = count - 1;
                                while (t >= 0 && ckey[t] > kj) {
                                    ckey[t + 1] = ckey[t];
                                    cand[t + 1] = cand[t];
                                    --t;
                                }
                                ckey[t + 1] = kj;
                                cand[t + 1] = j;
                            }
                            ++count;
                        }
                    }
                }
            }
        }
        // at most kMaxCand candidates were kept, whatever the list capacity
        const int lim = L.maxnb < kMaxCand ? L.maxnb : kMaxCand;
        const int keep = count < lim ? count : lim;
        for (int k = 0; k < keep; ++k) L.idx[(long)k * cap + i] = cand[k];
        L.nn[i] = keep;
    }
    // block max of the list length
    __shared__ int smax;
    if (threadIdx.x == 0) smax = 0;
    __syncthreads();
    atomicMax(&smax, count);
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicMax(&ctl->max_nbr, smax);
        if (smax > L.maxnb || smax > kMaxCand) atomicOr(&ctl->status, DEM_ERR_NEIGHBOR_OVERFLOW);
    }
}

// Re-sort partition, pass 1: class of cell slot s (cell order of the old storage): 0 when its
// particle has no neighbour within the list cutoff (the predicate of k_list: its list will be
// empty), 1 when, in the Verlet-skin mode, every listed neighbour's gap |x_i - x_j| - r_i - r_j
// exceeds skin/2 (no contact possible while twice the displacement bound stays below skin/2),
// else 2.  Per-block counts of classes 0 and 1 into sums[0][b], sums[1][b].
__global__ void __launch_bounds__(kPartBlock) k_part_flag(Particles P, const Ctl *ctl, const Grid *g, const int *start,
                                                          const int *items, double delta, double skin, int *cls,
                                                          int *sums, int nb, int classes) {
    const int cur = ctl->cur, n = P.n;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    int c_s = 2;
    if (s < n && classes && !(ctl->status & DEM_ERR_NAN)) {
        const int q = items[s];
        const Grid G = g[scene_of(P, q)];
        const double4 *pc = P.pos[cur];
        const D4 pi = ld4(pc, q);
        const bool skin_mode = !(delta > 0.0) && skin > 0.0;
        int c[3];
        cell_of(G, pi, c);
        bool any = false, near = false;
        for (int dz = -1; dz <= 1 && !near; ++dz) {
            const int z = c[2] + dz;
            if (z < 0 || z >= G.dims[2]) continue;
            for (int dy = -1; dy <= 1 && !near; ++dy) {
                const int y = c[1] + dy;
                if (y < 0 || y >= G.dims[1]) continue;
                for (int dx = -1; dx <= 1 && !near; ++dx) {
                    const int x = c[0] + dx;
                    if (x < 0 || x >= G.dims[0]) continue;
                    const int key = cell_key(G, x, y, z);
                    const int e = start[key + 1];
                    for (int t = start[key]; t < e; ++t) {
                        const int j = items[t];
                        if (j == q) continue;
                        const D4 pj = ld4(pc, j);
                        const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
                        const double r2 = px * px + py * py + pz * pz;
                        const double cut = delta > 0.0 ? delta : pi.w + pj.w + skin;
                        if (r2 <= cut * cut) {
                            any = true;
                            if (!skin_mode || !(sqrt(r2) - (pi.w + pj.w) > 0.5 * skin)) {
                                near = true;
                                break;
                            }
                        }
                    }
                }
            }
        }
        c_s = !any ? 0 : (near ? 2 : 1);
    }
    if (s < n) cls[s] = c_s;
    __shared__ int cnt[2];
    if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int w0 = __popc(__ballot_sync(0xffffffffu, s < n && c_s == 0));
    const int w1 = __popc(__ballot_sync(0xffffffffu, s < n && c_s == 1));
    if ((threadIdx.x & 31) == 0) {
        if (w0) atomicAdd(&cnt[0], w0);
        if (w1) atomicAdd(&cnt[1], w1);
    }
    __syncthreads();
    if (threadIdx.x < 2) sums[threadIdx.x * (nb + 1) + blockIdx.x] = cnt[threadIdx.x];
}

// Re-sort partition, pass 1 with the lists: the class of cell slot s as k_part_flag gives it,
// from the full list search of k_list done here, in the old storage order -- the list of the
// particle q = items[s] goes to nn_old[q], idx_old[k][q] (old indices, ascending caller index),
// and k_list_remap re-indexes it into the new order after the permutation, instead of a second
// 27-cell search over the permuted storage.  Same candidates, same order, same overflow rule as
// k_list (kMaxCand kept, DEM_ERR_NEIGHBOR_OVERFLOW when a list exceeds the capacity).
__global__ void __launch_bounds__(kPartBlock) k_part_list(Particles P, NbrList L, Ctl *ctl, const Grid *g,
                                                          const int *start, const int *items, double delta,
                                                          double skin, int *cls, int *sums, int nb, int classes) {
    const int cur = ctl->cur, n = P.n, cap = P.cap;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool invalid = (ctl->status & DEM_ERR_NAN) != 0;
    int c_s = 2, count = 0;
    if (s < n && invalid) L.nn_old[items[s]] = 0;
    if (s < n && !invalid) {
        const int q = items[s];
        const Grid G = g[scene_of(P, q)];
        const double4 *pc = P.pos[cur];
        const D4 pi = ld4(pc, q);
        const bool skin_mode = !(delta > 0.0) && skin > 0.0;
        int c[3];
        cell_of(G, pi, c);
        int cand[kMaxCand];
        int ckey[kMaxCand];
        bool near = false;
        for (int dz = -1; dz <= 1; ++dz) {
            const int z = c[2] + dz;
            if (z < 0 || z >= G.dims[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int y = c[1] + dy;
                if (y < 0 || y >= G.dims[1]) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = c[0] + dx;
                    if (x < 0 || x >= G.dims[0]) continue;
                    const int key = cell_key(G, x, y, z);
                    const int e = start[key + 1];
                    for (int t = start[key]; t < e; ++t) {
                        const int j = items[t];
                        if (j == q) continue;
                        const D4 pj = ld4(pc, j);
                        const double px = pi.x - pj.x, py = pi.y - pj.y, pz = pi.z - pj.z;
                        const double r2 = px * px + py * py + pz * pz;
                        const double cut = delta > 0.0 ? delta : pi.w + pj.w + skin;
                        if (r2 <= cut * cut) {
                            if (!skin_mode || !(sqrt(r2) - (pi.w + pj.w) > 0.5 * skin)) near = true;
                            if (count < kMaxCand) {
                                // insertion by caller index
                                const int kj = P.perm[j];
                                int u = count - 1;
                                while (u >= 0 && ckey[u] > kj) {
                                    ckey[u + 1] = ckey[u];
                                    cand[u + 1] = cand[u];
                                    --u;
                                }
                                ckey[u + 1] = kj;
                                cand[u + 1] = j;
                            }
                            ++count;
                        }
                    }
                }
            }
        }
        const int lim = L.maxnb < kMaxCand ? L.maxnb : kMaxCand;
        const int keep = count < lim ? count : lim;
        for (int k = 0; k < keep; ++k) L.idx_old[(long)k * cap + q] = cand[k];
        L.nn_old[q] = keep;
        c_s = !classes ? 2 : count == 0 ? 0 : (near ? 2 : 1);
    }
    if (s < n) cls[s] = c_s;
    __shared__ int cnt[2];
    __shared__ int smax;
    if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0) smax = 0;
    __syncthreads();
    const int w0 = __popc(__ballot_sync(0xffffffffu, s < n && c_s == 0));
    const int w1 = __popc(__ballot_sync(0xffffffffu, s < n && c_s == 1));
    if ((threadIdx.x & 31) == 0) {
        if (w0) atomicAdd(&cnt[0], w0);
        if (w1) atomicAdd(&cnt[1], w1);
    }
    atomicMax(&smax, count);
    __syncthreads();
    if (threadIdx.x < 2) sums[threadIdx.x * (nb + 1) + blockIdx.x] = cnt[threadIdx.x];
    if (threadIdx.x == 0) {
        atomicMax(&ctl->max_nbr, smax);
        if (smax > L.maxnb || smax > kMaxCand) atomicOr(&ctl->status, DEM_ERR_NEIGHBOR_OVERFLOW);
    }
}

// The lists of k_part_list into the new order: new position p holds old particle
// newitems[p]; partners are renamed by dst (old index -> new position).
__global__ void k_list_remap(int n, int cap, NbrList L, const int *newitems, const int *dst) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int q = newitems[p];
        const int c = L.nn_old[q];
        for (int k = 0; k < c; ++k) L.idx[(long)k * cap + p] = dst[L.idx_old[(long)k * cap + q]];
        L.nn[p] = c;
    }
}

// Pass 2, one block: exclusive scans of both per-block counts (block order); totals into
// nlone and nclear.
__global__ void __launch_bounds__(1024) k_part_scan(int *sums, int nb, Ctl *ctl) {
    __shared__ int part[1024];
    for (int k = 0; k < 2; ++k) {
        int *sk = sums + k * (nb + 1);
        const int per = (nb + 1023) / 1024;
        const int b0 = threadIdx.x * per, b1 = min(b0 + per, nb);
        int t = 0;
        for (int b = b0; b < b1; ++b) t += sk[b];
        part[threadIdx.x] = t;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {   // inclusive scan of the thread totals
            const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
            __syncthreads();
            part[threadIdx.x] += v;
            __syncthreads();
        }
        int run = threadIdx.x > 0 ? part[threadIdx.x - 1] : 0;
        for (int b = b0; b < b1; ++b) {
            const int v = sk[b];
            sk[b] = run;
            run += v;
        }
        if (threadIdx.x == 1023) {
            if (k == 0)
                ctl->nlone = part[1023];
            else
                ctl->nclear = part[1023];
        }
        __syncthreads();
    }
}

// Pass 3: stable partition of the cell order by class (0, then 1, then 2).  New position of
// slot s: newitems[pos] = old index, and items[s] = pos (the cell table of the permuted storage).
__global__ void __launch_bounds__(kPartBlock) k_part_place(int n, const int *cls, const int *sums, int nb,
                                                           const Ctl *ctl, int *items, int *newitems) {
    __shared__ int woff[2][kPartBlock / 32];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c = s < n ? cls[s] : 2;
    const unsigned b0 = __ballot_sync(0xffffffffu, s < n && c == 0);
    const unsigned b1 = __ballot_sync(0xffffffffu, s < n && c == 1);
    if (lane == 0) {
        woff[0][warp] = __popc(b0);
        woff[1][warp] = __popc(b1);
    }
    __syncthreads();
    int before0 = 0, before1 = 0;   // slots of class 0 / 1 of this block before this warp
    for (int w = 0; w < warp; ++w) {
        before0 += woff[0][w];
        before1 += woff[1][w];
    }
    if (s >= n) return;
    const unsigned below = (1u << lane) - 1u;
    const int r0 = sums[blockIdx.x] + before0 + __popc(b0 & below);              // class-0 slots before s
    const int r1 = sums[(nb + 1) + blockIdx.x] + before1 + __popc(b1 & below);   // class-1 slots before s
    const int nl = ctl->nlone, nc = ctl->nclear;
    const int pos = c == 0 ? r0 : c == 1 ? nl + r1 : nl + nc + (s - r0 - r1);
    newitems[pos] = items[s];
    items[s] = pos;
}

__global__ void k_build_begin(Ctl *ctl) {
    if (threadIdx.x == 0) {
        ctl->max_nbr = 0;
        ctl->nlone = 0;
        ctl->nclear = 0;
    }
}

__global__ void k_build_end(Ctl *ctl) {
    if (threadIdx.x == 0) {
        ctl->disp = 0.0;
        ctl->rebuilds += 1;
    }
}

}  // namespace

void launch_build(const Particles &P, Particles &alt, const NbrList &L, BuildBuffers &B, Ctl *ctl, double delta,
                  double skin, bool resort, bool check_run, cudaStream_t s, bool classes) {
    (void)check_run;
    const int n = P.n;
    const int gs = 148 * 8;
    const int tiles = (B.cell_cap + kScanTile) / kScanTile;
    k_build_begin<<<1, 32, 0, s>>>(ctl);
    k_bbox_init<<<(8 * B.nscenes + 255) / 256, 256, 0, s>>>(B.bbox, B.nscenes);
    k_bbox<<<gs, kB, 0, s>>>(P, ctl, B.bbox);
    k_grid<<<1, 256, 0, s>>>(B.bbox, B.grid, B.total, B.nscenes, B.cell_cap, delta, skin, ctl);
    k_zero<<<gs, kB, 0, s>>>(B.cell_start, B.total);
    k_count<<<gs, kB, 0, s>>>(P, ctl, B.grid, B.key, B.cell_start);
    // cell_start holds counts now; scan into cell_fill (as start) then swap roles
    k_scan_tiles<<<tiles, kB, 0, s>>>(B.cell_start, B.cell_fill, B.block_sums, B.total);
    k_scan_sums<<<1, kB, 0, s>>>(B.block_sums, B.total, B.cell_fill);
    k_scan_add<<<tiles, kB, 0, s>>>(B.cell_fill, B.cell_start, B.block_sums, B.total);
    // now cell_fill = exclusive start (with [ncodes] = n), cell_start = running cursor
    k_fill<<<gs, kB, 0, s>>>(n, B.key, B.cell_start, B.cell_items);
    k_cell_sort<<<gs, kB, 0, s>>>(B.cell_fill, B.cell_items, P.perm, B.total, ctl);
    if (resort) {
        // new order: the cell order, split stably into particles with no listed neighbour,
        // particles whose listed neighbours all keep a gap above skin/2, and the rest, so that
        // the streaming kernel's leading warps load no list and the next ones no partner
        const int nb = (n + kPartBlock - 1) / kPartBlock;
        if (L.idx_old)   // the lists too, in the old order (re-indexed below)
            k_part_list<<<nb, kPartBlock, 0, s>>>(P, L, ctl, B.grid, B.cell_fill, B.cell_items, delta, skin, B.src,
                                                  B.part_sums, nb, classes ? 1 : 0);
        else
            k_part_flag<<<nb, kPartBlock, 0, s>>>(P, ctl, B.grid, B.cell_fill, B.cell_items, delta, skin, B.src,
                                                  B.part_sums, nb, classes ? 1 : 0);
        k_part_scan<<<1, 1024, 0, s>>>(B.part_sums, nb, ctl);
        k_part_place<<<nb, kPartBlock, 0, s>>>(n, B.src, B.part_sums, nb, ctl, B.cell_items, B.key);
        k_make_dst<<<gs, kB, 0, s>>>(n, B.key, B.dst);
        k_permute<<<gs, kB, 0, s>>>(P, alt, ctl, B.key, B.dst);
        const size_t cap = (size_t)P.cap;
        cudaMemcpyAsync(P.force, alt.force, 3 * cap * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(P.torque, alt.torque, 3 * cap * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (P.ext) cudaMemcpyAsync(P.ext, alt.ext, 3 * cap * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(P.mI, alt.mI, 2 * cap * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(P.mat, alt.mat, cap, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(P.fix, alt.fix, cap, cudaMemcpyDeviceToDevice, s);
        k_hist_back<<<gs, kB, 0, s>>>(P, alt);   // before the contact words are replaced
        cudaMemcpyAsync(P.cstate, alt.cstate, cap * sizeof(int), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(P.perm, alt.perm, cap * sizeof(int), cudaMemcpyDeviceToDevice, s);
        if (P.scene) cudaMemcpyAsync(P.scene, alt.scene, cap * sizeof(int), cudaMemcpyDeviceToDevice, s);
        k_flip<<<1, 32, 0, s>>>(ctl);
    }
    if (resort && L.idx_old)
        k_list_remap<<<gs, kB, 0, s>>>(n, P.cap, L, B.key, B.dst);
    else
        k_list<<<(n + 127) / 128, 128, 0, s>>>(P, L, ctl, B.grid, B.cell_fill, B.cell_items, delta, skin);
    k_build_end<<<1, 32, 0, s>>>(ctl);
}

}  // namespace b200dem
