// rp_sort.cu -- re-sorting the particle state by grid and cell.
//
// The step is one thread per particle, so a warp's 32 particles gather
// from 32 places of the frame ring.  Releases are random in space, and
// particles drift; ordering the state by (grid, tile of 4 x 4 cells, cell)
// makes a warp's gathers hit the same or neighbouring columns, which turns
// scattered 32-byte sector reads into shared L1/L2 lines.  Each particle's
// arithmetic does not depend on where it sits in the arrays (its noise is
// keyed on its id), so results are unchanged, bit for bit.
//
// Counting sort: key histogram (atomics), exclusive scan, scatter of the
// particle index to its slot (order inside a cell is arbitrary), then every
// state column is gathered through the permutation.
#include <cuda_runtime.h>

#include "rp_internal.h"

namespace rp {

constexpr int kTile = 4;            // tile edge in cells
constexpr int kScanBlock = 1024;    // elements scanned per block

// key of a position (fractional 1-based indices) in grid g; base = first
// key of the grid
__device__ __forceinline__ uint32_t sort_key(const RpGridDev& g, double x, double y, uint32_t base) {
    int I = (x >= 1.0 && x < (double)g.nx) ? (int)x : (x >= (double)g.nx ? g.nx : 1);
    int J = (y >= 1.0 && y < (double)g.ny) ? (int)y : (y >= (double)g.ny ? g.ny : 1);
    if (!(x == x)) I = 1;           // NaN
    if (!(y == y)) J = 1;
    const int ntx = (g.nx + kTile - 1) / kTile;
    const int ti = (I - 1) / kTile, tj = (J - 1) / kTile;
    const int li = (I - 1) % kTile, lj = (J - 1) % kTile;
    return base + (uint32_t)((tj * ntx + ti) * (kTile * kTile) + lj * kTile + li);
}

__global__ void k_sort_keys(const __grid_constant__ RpStepArgs A, int mixed, const uint32_t* __restrict__ gbase,
                            uint32_t* __restrict__ keys, uint32_t* __restrict__ hist) {
    const RpParticlesDev& P = A.p;
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.n) return;
    int gid = P.gid[n];
    if (gid < 1 || gid > A.ngrid) gid = A.ngrid;
    const double x = mixed ? (double)P.x32[n] : P.x[n];
    const double y = mixed ? (double)P.y32[n] : P.y[n];
    const uint32_t k = sort_key(A.g[gid - 1], x, y, gbase[gid - 1]);
    keys[n] = k;
    atomicAdd(hist + k, 1u);
}

// exclusive scan of v[0..count) in blocks of kScanBlock; block totals to sums
__global__ void k_scan_blocks(uint32_t* __restrict__ v, int64_t count, uint32_t* __restrict__ sums) {
    __shared__ uint32_t warp_tot[32];
    const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
    const uint32_t x = (i < count) ? v[i] : 0u;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = x;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = warp_tot[lane];
        uint32_t ti = t;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += u;
        }
        warp_tot[lane] = ti - t;                     // exclusive warp offsets
        if (lane == 31 && sums) sums[blockIdx.x] = ti;
    }
    __syncthreads();
    if (i < count) v[i] = warp_tot[wid] + incl - x;
}

__global__ void k_scan_add(uint32_t* __restrict__ v, int64_t count, const uint32_t* __restrict__ sums) {
    const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
    if (i < count && blockIdx.x > 0) v[i] += sums[blockIdx.x];
}

__global__ void k_sort_scatter(int64_t n, const uint32_t* __restrict__ keys, uint32_t* __restrict__ offs,
                               int32_t* __restrict__ perm) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    perm[atomicAdd(offs + keys[i], 1u)] = (int32_t)i;
}

template <typename T>
__global__ void k_gather(const T* __restrict__ src, T* __restrict__ dst, const int32_t* __restrict__ perm, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[perm[i]];
}

template <typename T>
__global__ void k_unsort(const T* __restrict__ src, T* __restrict__ dst, const uint32_t* __restrict__ pid, uint32_t base,
                         int64_t n, int64_t nout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t o = (int64_t)(pid[i] - base);
    if (o >= 0 && o < nout) dst[o] = src[i];
}

static unsigned blocks_for(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

int64_t sort_key_count(const RpStepArgs& A, uint32_t* gbase_host) {
    int64_t k = 0;
    for (int g = 0; g < A.ngrid; g++) {
        gbase_host[g] = (uint32_t)k;
        const int ntx = (A.g[g].nx + kTile - 1) / kTile, nty = (A.g[g].ny + kTile - 1) / kTile;
        k += (int64_t)ntx * nty * kTile * kTile;
    }
    return k;
}

template <typename T>
static cudaError_t permute_col(T* col, void* scratch, const int32_t* perm, int64_t n, cudaStream_t s) {
    if (!col) return cudaSuccess;
    T* tmp = reinterpret_cast<T*>(scratch);
    k_gather<T><<<blocks_for(n, 256), 256, 0, s>>>(col, tmp, perm, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(col, tmp, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, s);
}

cudaError_t launch_sort(const RpStepArgs& A, int mixed, const SortBufs& b, void* scratch8, cudaStream_t s,
                        int* nlaunch) {
    const int64_t n = A.p.n;
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(b.hist, 0, sizeof(uint32_t) * (size_t)b.nkeys, s);
    if (e != cudaSuccess) return e;
    k_sort_keys<<<blocks_for(n, 256), 256, 0, s>>>(A, mixed, b.gbase, b.keys, b.hist);
    const int64_t nb = (b.nkeys + kScanBlock - 1) / kScanBlock;       // <= kScanBlock by construction
    k_scan_blocks<<<(unsigned)nb, kScanBlock, 0, s>>>(b.hist, b.nkeys, b.sums);
    k_scan_blocks<<<1, kScanBlock, 0, s>>>(b.sums, nb, nullptr);
    k_scan_add<<<(unsigned)nb, kScanBlock, 0, s>>>(b.hist, b.nkeys, b.sums);
    k_sort_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, b.keys, b.hist, b.perm);
    *nlaunch += 5;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const RpParticlesDev& P = A.p;
    double* d8[] = {P.x, P.y, P.z, P.age, P.dob, P.status, P.wd, P.zeta, P.bath, mixed ? P.qwarm : nullptr,
                    mixed ? P.gwarm : nullptr, P.salt, P.temp, P.mean_salt, P.mean_temp, P.hob, P.bustr, P.bvstr,
                    P.acc, P.vort, P.behavew, P.ssf};
    for (double* c : d8) {
        if ((e = permute_col(c, scratch8, b.perm, n, s)) != cudaSuccess) return e;
        if (c) *nlaunch += 1;
    }
    float* f4[] = {mixed ? P.x32 : nullptr, mixed ? P.y32 : nullptr, mixed ? P.z32 : nullptr,
                   mixed ? P.cx : nullptr,  mixed ? P.cy : nullptr,  mixed ? P.cz : nullptr,
                   mixed ? P.qwarm2 : nullptr};
    for (float* c : f4) {
        if ((e = permute_col(c, scratch8, b.perm, n, s)) != cudaSuccess) return e;
        if (c) *nlaunch += 1;
    }
    if ((e = permute_col(P.gid, scratch8, b.perm, n, s)) != cudaSuccess) return e;
    if ((e = permute_col(P.pid, scratch8, b.perm, n, s)) != cudaSuccess) return e;
    if ((e = permute_col(P.flags, scratch8, b.perm, n, s)) != cudaSuccess) return e;
    if ((e = permute_col(P.isin, scratch8, b.perm, n, s)) != cudaSuccess) return e;
    *nlaunch += 4;
    return cudaSuccess;
}

cudaError_t launch_unsort(int elem, const void* src, void* dst, const uint32_t* pid, uint32_t base, int64_t n,
                          int64_t nout, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const unsigned nb = blocks_for(n, 256);
    if (elem == 8)
        k_unsort<uint64_t><<<nb, 256, 0, s>>>((const uint64_t*)src, (uint64_t*)dst, pid, base, n, nout);
    else if (elem == 4)
        k_unsort<uint32_t><<<nb, 256, 0, s>>>((const uint32_t*)src, (uint32_t*)dst, pid, base, n, nout);
    else
        k_unsort<uint8_t><<<nb, 256, 0, s>>>((const uint8_t*)src, (uint8_t*)dst, pid, base, n, nout);
    return cudaGetLastError();
}

}  // namespace rp
