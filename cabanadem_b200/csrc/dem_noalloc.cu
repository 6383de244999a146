// dem_noalloc.cu -- neighbour-list build that allocates no memory.
//
// dem_build_neighbors needs scratch memory (cell table, sort keys, scan partials) that the
// solver allocates with cudaMalloc when it is created.  Some callers cannot allocate at the
// point where they need a neighbour list: code whose device memory is owned by another
// allocator (a framework's caching pool, a fixed memory budget handed out up front), code
// that must not stall the GPU (cudaMalloc and cudaFree can synchronise the device, which
// breaks a latency-bound time loop sharing the GPU with other work), and code that runs
// where no allocation API may be called at all.  dem_neighbor_list_noalloc serves them:
// the caller passes inputs and outputs, and the scratch comes from the fixed array below.
//
// Limits and sharing rules:
//  - at most DEM_NOALLOC_MAX_PARTICLES particles per call and at most
//    DEM_NOALLOC_MAX_NEIGHBORS list entries per particle (the list build keeps that many
//    candidates per particle); larger values are rejected with DEM_ERR_INVALID;
//  - every GPU that loads this library holds the array (about 2.4 MB) until the process
//    exits, whether or not the function is called;
//  - all calls on a device share the one array, which keeps the last call's contents; the
//    function clears what has to start at zero itself, but two calls whose work overlaps
//    on the GPU (different streams, no ordering between them) race on it and must not be
//    issued;
//  - the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that first call
//    before any stream capture begins.  The cache is per process and is not refreshed: after
//    a cudaDeviceReset on that device the cached address is stale, so a process that resets
//    a device must not call this function on it again.
#include <cstring>
#include <mutex>

#include "b200dem.h"
#include "dem_internal.cuh"

using namespace b200dem;

namespace {

constexpr int kNoAllocCellCap = 4 * DEM_NOALLOC_MAX_PARTICLES;

// byte offsets of the regions inside the scratch array (each 256-byte aligned)
constexpr size_t al(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffCtl = 0;
constexpr size_t kOffGrid = al(kOffCtl + sizeof(Ctl));
constexpr size_t kOffTotal = al(kOffGrid + sizeof(Grid));
constexpr size_t kOffBbox = al(kOffTotal + sizeof(int));
constexpr size_t kOffPos = al(kOffBbox + 8 * sizeof(unsigned long long));
constexpr size_t kOffPerm = al(kOffPos + sizeof(double4) * DEM_NOALLOC_MAX_PARTICLES);
constexpr size_t kOffKey = al(kOffPerm + sizeof(int) * DEM_NOALLOC_MAX_PARTICLES);
constexpr size_t kOffItems = al(kOffKey + sizeof(int) * DEM_NOALLOC_MAX_PARTICLES);
constexpr size_t kOffStart = al(kOffItems + sizeof(int) * DEM_NOALLOC_MAX_PARTICLES);
constexpr size_t kOffFill = al(kOffStart + sizeof(int) * (kNoAllocCellCap + 1));
constexpr size_t kOffSums = al(kOffFill + sizeof(int) * (kNoAllocCellCap + 1));
constexpr size_t kScratchBytes = al(kOffSums + sizeof(int) * (kNoAllocCellCap / 2048 + 2));

static __device__ __align__(256) unsigned char g_nbr_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
void *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// Device address of g_nbr_scratch on the current device (looked up once per device).
int scratch_address(void **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DEM_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_nbr_scratch) != cudaSuccess || !p) return DEM_ERR_CUDA;
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return DEM_OK;
}

__global__ void k_pack(const double *x, const double *rad, int n, double4 *pos, int *perm) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        pos[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], rad[i]);
        perm[i] = i;
    }
}

}  // namespace

extern "C" int dem_neighbor_list_noalloc(const double *x, const double *rad, int n, double delta, double skin,
                                         int max_neighbors, int *nn, int *idx, void *stream) {
    if (!x || !rad || !nn || !idx || n <= 0 || max_neighbors <= 0) return DEM_ERR_INVALID;
    if (n > DEM_NOALLOC_MAX_PARTICLES || max_neighbors > DEM_NOALLOC_MAX_NEIGHBORS) return DEM_ERR_INVALID;
    if (!(delta > 0.0) && !(skin >= 0.0)) return DEM_ERR_INVALID;
    void *base = nullptr;
    int st = scratch_address(&base);
    if (st) return st;
    unsigned char *b = static_cast<unsigned char *>(base);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    Particles P{};
    P.n = n;
    P.cap = n;
    P.pos[0] = P.pos[1] = reinterpret_cast<double4 *>(b + kOffPos);
    P.perm = reinterpret_cast<int *>(b + kOffPerm);
    Ctl *ctl = reinterpret_cast<Ctl *>(b + kOffCtl);
    BuildBuffers B{};
    B.grid = reinterpret_cast<Grid *>(b + kOffGrid);
    B.total = reinterpret_cast<int *>(b + kOffTotal);
    B.nscenes = 1;
    B.bbox = reinterpret_cast<unsigned long long *>(b + kOffBbox);
    B.key = reinterpret_cast<int *>(b + kOffKey);
    B.cell_items = reinterpret_cast<int *>(b + kOffItems);
    B.cell_start = reinterpret_cast<int *>(b + kOffStart);
    B.cell_fill = reinterpret_cast<int *>(b + kOffFill);
    B.block_sums = reinterpret_cast<int *>(b + kOffSums);
    B.cell_cap = kNoAllocCellCap;
    NbrList L{};
    L.nn = nn;
    L.idx = idx;
    L.maxnb = max_neighbors;

    // the control word carries the overflow flag and the buffer index: start from zero
    if (cudaMemsetAsync(ctl, 0, sizeof(Ctl), s) != cudaSuccess) return DEM_ERR_CUDA;
    k_pack<<<(n + 255) / 256, 256, 0, s>>>(x, rad, n, P.pos[0], P.perm);
    Particles unused{};
    launch_build(P, unused, L, B, ctl, delta > 0.0 ? delta : 0.0, skin, false, false, s);
    if (cudaGetLastError() != cudaSuccess) return DEM_ERR_CUDA;
    int status = 0;
    if (cudaMemcpyAsync(&status, &ctl->status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return DEM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return DEM_ERR_CUDA;
    return status & (DEM_ERR_NEIGHBOR_OVERFLOW | DEM_ERR_NAN);
}
