// rp_mixed.cu -- kernels of the mixed-precision form: the step, the FP16
// frame quantisation with per-level scales, and the conversions between
// the FP64 particle columns and the compensated FP32 positions.
// Compiled with FMA contraction (the default): this form is not bit-exact.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "rp_internal.h"
#include "rp_mixed.cuh"

namespace rp {

// Fused form: one thread per particle for the whole step.
// FEAT: built with the options beyond the passive step (diagnostics,
// WETDRY, behave); the passive variant is chosen when they are all off.
// BLK: threads per block (the register cap stays that of 128 x 8 resident
// threads; the block is the scheduling unit of the grid-stride loop).
template <typename E, int NPMAX, bool FEAT, bool PREF = true, int BLK = kStepBlock>
__global__ void __launch_bounds__(BLK, kMixedMinBlocks * kStepBlock / BLK)
    k_step_mixed(const __grid_constant__ RpStepArgs A) {
    double buf[kMixedArrays * (NPMAX + 1)];
    const MSpline<NPMAX, PREF> w{buf};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride)
        m_update_one<E, FEAT>(A, n, w, nullptr);
}

// Split form: VTurb alone at a resident-thread count whose spline
// workspace stays in L2, writing each particle's displacement; then the
// rest of the step at full occupancy.
template <typename E, int NPMAX>
__global__ void __launch_bounds__(kStepBlock, kMixedVtMinBlocks) k_vturb_mixed(const __grid_constant__ RpStepArgs A,
                                                                               float* __restrict__ turbv) {
    double buf[kMixedArrays * (NPMAX + 1)];
    const MSpline<NPMAX> w{buf};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride)
        m_vturb_one<E>(A, n, w, turbv);
}

// Split form with the fit's workspace in shared memory: VTurb alone, one
// thread per particle, 64-thread blocks each holding its threads' u, factor
// prefix and column (1.1 KB per thread at NPMAX 128: 3 blocks per SM).  The
// fit's passes then read and write shared memory instead of streaming a
// local-memory workspace through L2 and HBM.
constexpr int kSmemBlock = 64;
constexpr int kSmemKs = 32;              // factor rows 2..33 held in shared memory
template <int NPMAX>
using SmemView = MSmemSpline<NPMAX, kSmemKs, NPMAX / 4, kSmemBlock>;

template <typename E, int NPMAX>
__global__ void __launch_bounds__(kSmemBlock) k_vturb_smem(const __grid_constant__ RpStepArgs A,
                                                           float* __restrict__ turbv) {
    extern __shared__ float smf[];
    float ovf[2 * (NPMAX + 1)];
    const SmemView<NPMAX> w{smf + threadIdx.x, ovf};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride)
        m_vturb_one<E>(A, n, w, turbv);
}

template <typename E, bool FEAT>
__global__ void __launch_bounds__(kStepBlock, kMixedMinBlocks) k_advect_mixed(const __grid_constant__ RpStepArgs A,
                                                             const float* __restrict__ turbv) {
    const MSpline<1> none{nullptr};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride)
        m_update_one<E, FEAT>(A, n, none, turbv);
}

// The diagnostics of the particles the step just advanced (their tdepth in
// A.diag_td; NaN for the others), as the end of update_particles computes
// them (ROMSPath.f90:935-986).  A pass of its own keeps the diagnostics'
// code and registers out of the step kernel.
__global__ void __launch_bounds__(kStepBlock) k_diag_mixed(const __grid_constant__ RpStepArgs A) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride) {
        const float td = A.diag_td[n];
        if (!(td == td)) continue;
        uint32_t fl = 0;
        m_diag_one(A, n, td, fl);
        if (fl) A.p.flags[n] |= fl;
    }
}

// behave (behavior_module.f90:186-393) of the particles the step is about to
// advance, at their start position after find_currents' stage-1 z clamp
// (the Zpar update_particles hands it, ROMSPath.f90:800-804): ZBehav to
// A.beh_z, behave's outputs to the particle columns.  A pass of its own
// keeps behave's code and registers out of the step kernel.
__global__ void __launch_bounds__(kStepBlock) k_behave_mixed(const __grid_constant__ RpStepArgs A) {
    const RpParticlesDev& Pt = A.p;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < Pt.n; n += stride) {
        if (!rp_active(A, n)) continue;
        uint32_t fl = 0;
        const RpGridDev& g = A.g[Pt.gid[n] - 1];
        const float Xpar = Pt.x32[n], Ypar = Pt.y32[n];
        float Zpar = Pt.z32[n] - Pt.cz[n];
        if (A.scheme == 1) {
            MStage S1;
            m_rho_cell(g, Xpar, Ypar, S1.rc, fl);
            m_stage_2d(m_time(A, g, 0), g, S1);
            if (Zpar < S1.tdepth) Zpar = S1.tdepth + 0.001f;
            if (Zpar > S1.zeta) Zpar = S1.zeta - 0.001f;
        }
        A.beh_z[n] = (float)m_behave(A, n, g, Xpar, Ypar, Zpar, Pt.pid[n], fl);
        if (fl) Pt.flags[n] |= fl;
    }
}

template <class K>
static cudaError_t resident_grid(K kernel, int64_t n, int num_sms, int cap_per_sm, int64_t* blocks,
                                 int blk = kStepBlock) {
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, blk, 0);
    if (e != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    if (cap_per_sm > 0 && occ > cap_per_sm) occ = cap_per_sm;
    int64_t b = (int64_t)num_sms * occ;
    const int64_t need = (n + blk - 1) / blk;
    if (need < b) b = need;
    *blocks = b < 1 ? 1 : b;
    return cudaSuccess;
}

template <typename E, int NPMAX, bool FEAT>
static cudaError_t launch_mixed_t(const RpStepArgs& A, float* turbv, int split, cudaStream_t s, int num_sms,
                                  int* nlaunch) {
    int64_t blocks = 0;
    cudaError_t e;
    if (split == 2 && A.vturb_on) {
        // the shared-memory column holds sw <= NPMAX/4 levels
        int swmax = 0;
        for (int k = 0; k < A.ngrid; k++) swmax = max(swmax, A.g[k].N + 1);
        if (swmax > NPMAX / 4) split = 1;
    }
    if (split == 2 && A.vturb_on) {
        const size_t smem = (size_t)SmemView<NPMAX>::kWords * kSmemBlock * sizeof(float);
        static bool attr_set = false;
        if (!attr_set) {
            e = cudaFuncSetAttribute(k_vturb_smem<E, NPMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_set = true;
        }
        int occ = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_vturb_smem<E, NPMAX>, kSmemBlock, smem)) !=
            cudaSuccess)
            return e;
        if (occ < 1) occ = 1;
        blocks = (A.p.n + kSmemBlock - 1) / kSmemBlock;
        if (blocks > (int64_t)num_sms * occ) blocks = (int64_t)num_sms * occ;
        k_vturb_smem<E, NPMAX><<<(unsigned)(blocks < 1 ? 1 : blocks), kSmemBlock, smem, s>>>(A, turbv);
        *nlaunch += 1;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = resident_grid(k_advect_mixed<E, FEAT>, A.p.n, num_sms, A.grid_cap, &blocks)) != cudaSuccess) return e;
        k_advect_mixed<E, FEAT><<<(unsigned)blocks, kStepBlock, 0, s>>>(A, turbv);
        *nlaunch += 1;
        return cudaGetLastError();
    }
    if ((split == 4 || split == 5) && !FEAT) {     // fused, 64- or 256-thread blocks
        if (split == 4) {
            if ((e = resident_grid(k_step_mixed<E, NPMAX, false, true, 64>, A.p.n, num_sms,
                                   A.grid_cap ? 2 * A.grid_cap : 0, &blocks, 64)) != cudaSuccess)
                return e;
            k_step_mixed<E, NPMAX, false, true, 64><<<(unsigned)blocks, 64, 0, s>>>(A);
        } else {
            if ((e = resident_grid(k_step_mixed<E, NPMAX, false, true, 256>, A.p.n, num_sms,
                                   A.grid_cap ? (A.grid_cap + 1) / 2 : 0, &blocks, 256)) != cudaSuccess)
                return e;
            k_step_mixed<E, NPMAX, false, true, 256><<<(unsigned)blocks, 256, 0, s>>>(A);
        }
        *nlaunch += 1;
        return cudaGetLastError();
    }
    if (split == 3 && !FEAT) {                     // fused, u not loaded ahead
        if ((e = resident_grid(k_step_mixed<E, NPMAX, false, false>, A.p.n, num_sms, A.grid_cap, &blocks)) !=
            cudaSuccess)
            return e;
        k_step_mixed<E, NPMAX, false, false><<<(unsigned)blocks, kStepBlock, 0, s>>>(A);
        *nlaunch += 1;
        return cudaGetLastError();
    }
    if (split >= 3 || !split || !A.vturb_on) {
        if ((e = resident_grid(k_step_mixed<E, NPMAX, FEAT>, A.p.n, num_sms, A.grid_cap, &blocks)) != cudaSuccess)
            return e;
        k_step_mixed<E, NPMAX, FEAT><<<(unsigned)blocks, kStepBlock, 0, s>>>(A);
        *nlaunch += 1;
        return cudaGetLastError();
    }
    if ((e = resident_grid(k_vturb_mixed<E, NPMAX>, A.p.n, num_sms, kMixedVtMinBlocks, &blocks)) != cudaSuccess)
        return e;
    k_vturb_mixed<E, NPMAX><<<(unsigned)blocks, kStepBlock, 0, s>>>(A, turbv);
    *nlaunch += 1;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = resident_grid(k_advect_mixed<E, FEAT>, A.p.n, num_sms, A.grid_cap, &blocks)) != cudaSuccess) return e;
    k_advect_mixed<E, FEAT><<<(unsigned)blocks, kStepBlock, 0, s>>>(A, turbv);
    *nlaunch += 1;
    return cudaGetLastError();
}

template <typename E, bool FEAT>
static cudaError_t launch_mixed_f(const RpStepArgs& A, int npmax, float* turbv, int split, cudaStream_t s,
                                  int num_sms, int* nlaunch) {
    if (npmax <= 88) return launch_mixed_t<E, 88, FEAT>(A, turbv, split, s, num_sms, nlaunch);
    if (npmax <= 128) return launch_mixed_t<E, 128, FEAT>(A, turbv, split, s, num_sms, nlaunch);
    return launch_mixed_t<E, 144, FEAT>(A, turbv, split, s, num_sms, nlaunch);
}

template <typename E>
static cudaError_t launch_mixed_e(const RpStepArgs& A, int npmax, float* turbv, int split, cudaStream_t s,
                                  int num_sms, int* nlaunch) {
    const bool feat = A.diag || A.wetdry || A.beh.behavior || A.beh.va || A.beh.wa;
    return feat ? launch_mixed_f<E, true>(A, npmax, turbv, split, s, num_sms, nlaunch)
                : launch_mixed_f<E, false>(A, npmax, turbv, split, s, num_sms, nlaunch);
}

cudaError_t launch_step_mixed(const RpStepArgs& A0, int npmax, int i16, float* turbv, int split, cudaStream_t s,
                              int num_sms, int* nlaunch) {
    RpStepArgs A = A0;
    float* td = nullptr;
    cudaError_t e;
    int64_t blocks = 0;
    if (A.beh.behavior || A.beh.va || A.beh.wa) {
        // ZBehav in the third part of the scratch (3 floats per particle)
        A.beh_z = turbv + 2 * A.p.n;
        if ((e = resident_grid(k_behave_mixed, A.p.n, num_sms, 0, &blocks)) != cudaSuccess) return e;
        k_behave_mixed<<<(unsigned)blocks, kStepBlock, 0, s>>>(A);
        *nlaunch += 1;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (A.diag) {
        // the step's tdepth per particle goes to the second half of the
        // scratch (the first half holds the split forms' VTurb displacement)
        td = turbv + A.p.n;
        A.diag_td = td;
        if ((e = cudaMemsetAsync(td, 0xff, sizeof(float) * (size_t)A.p.n, s)) != cudaSuccess) return e;   // NaN
    }
    e = i16 ? launch_mixed_e<int16_t>(A, npmax, turbv, split, s, num_sms, nlaunch)
            : launch_mixed_e<__half>(A, npmax, turbv, split, s, num_sms, nlaunch);
    if (e != cudaSuccess || !A.diag) return e;
    if ((e = resident_grid(k_diag_mixed, A.p.n, num_sms, 0, &blocks)) != cudaSuccess) return e;
    k_diag_mixed<<<(unsigned)blocks, kStepBlock, 0, s>>>(A);
    *nlaunch += 1;
    return cudaGetLastError();
}

// ------------------------------------------------------ frame upload

// one staged chunk of a Fortran-ordered field (plus the Stokes term) into
// the FP32 field buffer, same order
template <typename S>
__global__ void k_stage_f32(const S* __restrict__ src, const S* __restrict__ add, float* __restrict__ dst,
                            int64_t e0, int64_t count) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    double v = (double)src[t];
    if (add) v = v + (double)add[t];
    dst[e0 + t] = (float)v;
}

cudaError_t launch_stage_f32(int src_f32, const void* src, const void* add, float* dst, int64_t e0, int64_t count,
                             cudaStream_t s) {
    const int block = 256;
    const unsigned blocks = (unsigned)((count + block - 1) / block);
    if (blocks == 0) return cudaSuccess;
    if (src_f32)
        k_stage_f32<float><<<blocks, block, 0, s>>>((const float*)src, (const float*)add, dst, e0, count);
    else
        k_stage_f32<double><<<blocks, block, 0, s>>>((const double*)src, (const double*)add, dst, e0, count);
    return cudaGetLastError();
}

// max |v| over each level k of a Fortran-ordered field (level = slowest
// index), as the bits of a non-negative float (integer order = float order)
__global__ void k_level_maxabs(const float* __restrict__ f, int64_t plane, uint32_t* __restrict__ maxbits) {
    const int k = blockIdx.y;
    const float* lev = f + (int64_t)k * plane;
    float m = 0.f;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < plane; e += (int64_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(lev[e]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = (threadIdx.x < (blockDim.x >> 5)) ? wm[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) atomicMax(maxbits + k, __float_as_uint(m));
    }
}

// The scale of a level.  FP16: the power of two with |v| / scale <= 16384
// (exact scaling, keeps w and AKs out of the FP16 subnormal range).  int16:
// level max / 32767.
__device__ __forceinline__ float m_level_scale(uint32_t bits, bool i16) {
    const float mx = __uint_as_float(bits);
    if (!(mx > 0.f) || !(mx < 3.0e38f)) return 1.0f;
    if (i16) return mx / 32767.0f;
    int e = 0;
    frexpf(mx, &e);                        // mx = m 2^e, m in [0.5, 1)
    return ldexpf(1.0f, e - 14);
}

// FP16 stores finite values only, as the int16 form's clamp does: NaN as 0,
// +-Inf as +-65504 (the mixed form reads the spare ring slot with weight 0,
// and an upload may be filling it while steps run)
__device__ __forceinline__ void m_store16(__half* d, float v) {
    *d = __float2half_rn(v != v ? 0.f : fminf(fmaxf(v, -65504.f), 65504.f));
}
__device__ __forceinline__ void m_store16(int16_t* d, float v) {
    const float r = fminf(fmaxf(rintf(v), -32767.0f), 32767.0f);
    *d = (int16_t)r;
}

// FP32 field (Fortran order) -> 16-bit device layout [j][i][k][slot4] and
// the per-level scales qs[k][slot4].  A block takes 32 points of row j
// with all their levels: it reads level by level (coalesced along i) into
// shared memory and writes point by point, the levels of a point adjacent
// as the ring holds them, so a warp's stores cover one contiguous run of
// the ring instead of one sector per value.
constexpr int kQuantMaxLevels = kMaxNp;     // s_w <= int(s_w*sub) <= kMaxNp
template <typename E>
__global__ void __launch_bounds__(256) k_quantize(const float* __restrict__ f, const uint32_t* __restrict__ maxbits,
                                                  float* __restrict__ qs, E* __restrict__ dst, int ni, int nj, int nk,
                                                  int slot) {
    constexpr bool i16 = sizeof(E) == 2 && !std::is_same<E, __half>::value;
    __shared__ float tile[kQuantMaxLevels][33];
    __shared__ float sc[kQuantMaxLevels];
    const int i0 = blockIdx.x * 32, j = blockIdx.y;
    const int64_t plane = (int64_t)ni * nj;
    for (int k = threadIdx.x; k < nk; k += blockDim.x) {
        sc[k] = m_level_scale(maxbits[k], i16);
        if (blockIdx.x == 0 && j == 0) qs[k * RP_SLOTS + slot] = sc[k];
    }
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int npt = min(32, ni - i0);                 // points of this tile
    for (int k = threadIdx.x >> 5; k < nk; k += nw)
        if (lane < npt) tile[k][lane] = f[(int64_t)k * plane + (int64_t)j * ni + i0 + lane];
    __syncthreads();
    E* out = dst + ((int64_t)j * ni + i0) * nk * RP_SLOTS + slot;
    for (int t = threadIdx.x; t < npt * nk; t += blockDim.x) {
        const int il = t / nk, k = t - il * nk;
        const float v = tile[k][il], s = sc[k];
        m_store16(out + (int64_t)t * RP_SLOTS, i16 ? v / s : v * (1.0f / s));
    }
}

cudaError_t launch_quantize(const float* f, uint32_t* maxbits, float* qs, void* dst, int ni, int nj, int nk, int slot,
                            int i16, int num_sms, cudaStream_t s) {
    if (nk > kQuantMaxLevels || ni < 1 || nj < 1 || nj > 65535) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(maxbits, 0, sizeof(uint32_t) * nk, s);
    if (e != cudaSuccess) return e;
    const int64_t plane = (int64_t)ni * nj;
    const int block = 256;
    int64_t bx = (plane + block - 1) / block;
    const int64_t cap = (int64_t)num_sms * 4 / (nk > 0 ? nk : 1) + 1;
    if (bx > cap) bx = cap;
    k_level_maxabs<<<dim3((unsigned)bx, (unsigned)nk), block, 0, s>>>(f, plane, maxbits);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const dim3 grid((unsigned)((ni + 31) / 32), (unsigned)nj);
    if (i16) k_quantize<int16_t><<<grid, 256, 0, s>>>(f, maxbits, qs, (int16_t*)dst, ni, nj, nk, slot);
    else k_quantize<__half><<<grid, 256, 0, s>>>(f, maxbits, qs, (__half*)dst, ni, nj, nk, slot);
    return cudaGetLastError();
}

// ----------------------------------------------- particle conversions

// FP64 columns -> compensated FP32 positions (value = p - c) and no
// smoothing-parameter warm start
template <typename T>
__global__ void __launch_bounds__(256) k_clear_slot(T* ring, int64_t count, int slot) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += stride)
        ring[t * RP_SLOTS + slot] = T(0);
}

cudaError_t launch_clear_slot(void* ring, int elem, int64_t count, int slot, int num_sms, cudaStream_t s) {
    if (!ring || count <= 0) return cudaSuccess;
    int64_t blocks = (count + 255) / 256;
    if (blocks > (int64_t)num_sms * 8) blocks = (int64_t)num_sms * 8;
    if (elem == 2) k_clear_slot<uint16_t><<<(unsigned)blocks, 256, 0, s>>>((uint16_t*)ring, count, slot);
    else k_clear_slot<uint32_t><<<(unsigned)blocks, 256, 0, s>>>((uint32_t*)ring, count, slot);
    return cudaGetLastError();
}

__global__ void k_mixed_from_f64(RpParticlesDev P) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.n) return;
    const double x = P.x[n], y = P.y[n], z = P.z[n];
    const float px = (float)x, py = (float)y, pz = (float)z;
    P.x32[n] = px; P.cx[n] = (float)((double)px - x);
    P.y32[n] = py; P.cy[n] = (float)((double)py - y);
    P.z32[n] = pz; P.cz[n] = (float)((double)pz - z);
    P.qwarm[n] = -1.0;
    P.gwarm[n] = 0.0;
    P.qwarm2[n] = -1.f;
}

__global__ void k_mixed_to_f64(RpParticlesDev P) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.n) return;
    P.x[n] = (double)P.x32[n] - (double)P.cx[n];
    P.y[n] = (double)P.y32[n] - (double)P.cy[n];
    P.z[n] = (double)P.z32[n] - (double)P.cz[n];
}

cudaError_t launch_mixed_convert(const RpParticlesDev& P, int to_f64, cudaStream_t s) {
    const int block = 256;
    const unsigned blocks = (unsigned)((P.n + block - 1) / block);
    if (blocks == 0) return cudaSuccess;
    if (to_f64) k_mixed_to_f64<<<blocks, block, 0, s>>>(P);
    else k_mixed_from_f64<<<blocks, block, 0, s>>>(P);
    return cudaGetLastError();
}

}  // namespace rp
