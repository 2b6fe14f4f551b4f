// rp_noalloc.cu -- the split particle step with its scratch array in a
// static device buffer, for callers that cannot allocate device memory.
//
// The split step writes each particle's VTurb displacement into a scratch
// array that k_advect then reads.  rp_step keeps that array in the context
// (allocated by rp_create).  rp_step_noalloc instead uses the fixed buffer
// below, which the CUDA loader creates on every device that loads this
// library and keeps until the process exits; the entry point itself calls
// no cudaMalloc, cudaFree or allocating library routine.
//
// Compiled with -fmad=false, like rp_kernels.cu: the results are bit-
// identical to rp_step.  The VTurb kernel here keeps the spline workspace of
// its warp's 32 particles in shared memory (no local-memory frame), because
// a kernel with a large local-memory frame can make the driver enlarge its
// local-memory reservation at launch -- an allocation.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "rp_internal.h"
#include "rp_step.cuh"

namespace rp {

// Scratch: the VTurb displacement of up to kNoallocMaxParticles particles
// (8 MiB).  Shared by every call on a device and never cleared: each
// active particle's entry is written by k_vturb_na before k_advect_na
// reads it in the same call, and inactive particles are neither written
// nor read, so no element must start at zero.  Calls that overlap on the
// GPU (two streams, or two host threads) race on this buffer.
static __device__ __align__(256) double rp_noalloc_turbv[kNoallocMaxParticles];

namespace {

// Device address of rp_noalloc_turbv per device ordinal.  In host code the
// symbol is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress with the device current (once per device, on the
// first call there -- which must therefore come before any stream capture).
// The table is filled under a lock, so host threads driving contexts on
// the same device may make their first calls at the same time.  The
// address belongs to the device's primary context: after a cudaDeviceReset
// the module is loaded again elsewhere and the cached address is stale, so
// the entry point is not for processes that reset a device between calls.
constexpr int kMaxDevices = 64;
double* g_scratch[kMaxDevices] = {};
std::mutex g_scratch_lock;

cudaError_t scratch_for_device(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> guard(g_scratch_lock);
    if (!g_scratch[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, rp_noalloc_turbv);
        if (e != cudaSuccess) return e;
        g_scratch[device] = static_cast<double*>(p);
    }
    *out = g_scratch[device];
    return cudaSuccess;
}

}  // namespace

template <typename T, int NPMAX>
__global__ void __launch_bounds__(32, 1) k_vturb_na(const __grid_constant__ RpStepArgs A, double* __restrict__ turbv) {
    extern __shared__ double sm[];
    const SplineView<NPMAX, 32> w{sm + threadIdx.x};
    const int64_t stride = (int64_t)gridDim.x * 32;
    for (int64_t n = (int64_t)blockIdx.x * 32 + threadIdx.x; n < A.p.n; n += stride)
        rp_vturb_one<T>(A, n, w, turbv);
}

template <typename T>
__global__ void __launch_bounds__(kStepBlock) k_advect_na(const __grid_constant__ RpStepArgs A,
                                                         const double* __restrict__ turbv) {
    const SplineView<1, 1> none{nullptr};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride)
        rp_update_one<T>(A, n, none, turbv);
}

template <typename T, int NPMAX>
static cudaError_t launch_na(const RpStepArgs& A, double* scratch, cudaStream_t s, int num_sms, int* nlaunch) {
    cudaError_t e = cudaSuccess;
    if (A.vturb_on) {
        const size_t smem = (size_t)kSplineArrays * (NPMAX + 1) * 32 * sizeof(double);
        e = cudaFuncSetAttribute(k_vturb_na<T, NPMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int occ = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_vturb_na<T, NPMAX>, 32, smem);
        if (e != cudaSuccess) return e;
        int64_t blocks = std::min<int64_t>((A.p.n + 31) / 32, (int64_t)num_sms * std::max(occ, 1));
        k_vturb_na<T, NPMAX><<<(unsigned)std::max<int64_t>(blocks, 1), 32, smem, s>>>(A, scratch);
        *nlaunch += 1;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_advect_na<T>, kStepBlock, 0);
    if (e != cudaSuccess) return e;
    int64_t blocks = std::min<int64_t>((A.p.n + kStepBlock - 1) / kStepBlock, (int64_t)num_sms * std::max(occ, 1));
    k_advect_na<T><<<(unsigned)std::max<int64_t>(blocks, 1), kStepBlock, 0, s>>>(A, A.vturb_on ? scratch : nullptr);
    *nlaunch += 1;
    return cudaGetLastError();
}

cudaError_t launch_step_noalloc(const RpStepArgs& A, int field_dtype, int npmax, int device, cudaStream_t s,
                                int num_sms, int* nlaunch) {
    if (A.p.n > kNoallocMaxParticles || npmax > 128) return cudaErrorInvalidValue;
    double* scratch = nullptr;
    cudaError_t e = scratch_for_device(device, &scratch);
    if (e != cudaSuccess) return e;
    if (field_dtype == 1) {
        if (npmax <= 88) return launch_na<float, 88>(A, scratch, s, num_sms, nlaunch);
        return launch_na<float, 128>(A, scratch, s, num_sms, nlaunch);
    }
    if (npmax <= 88) return launch_na<double, 88>(A, scratch, s, num_sms, nlaunch);
    return launch_na<double, 128>(A, scratch, s, num_sms, nlaunch);
}

}  // namespace rp
