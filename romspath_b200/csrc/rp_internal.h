// rp_internal.h -- launch entry points shared between the kernel unit
// (compiled without FMA contraction) and the host-side C ABI unit.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rp_device.cuh"

namespace rp {

constexpr int kStepBlock = 128;
#ifndef RP_VTURB_MIN_BLOCKS
#define RP_VTURB_MIN_BLOCKS 8
#endif
constexpr int kVturbMinBlocks = RP_VTURB_MIN_BLOCKS;   // resident 128-thread blocks per SM
#ifndef RP_MIXED_MIN_BLOCKS
#define RP_MIXED_MIN_BLOCKS 8
#endif
constexpr int kMixedMinBlocks = RP_MIXED_MIN_BLOCKS;   // same, mixed-precision step
#ifndef RP_MIXED_VT_BLOCKS
#define RP_MIXED_VT_BLOCKS 2
#endif
constexpr int kMixedVtMinBlocks = RP_MIXED_VT_BLOCKS;  // split mixed form: VTurb kernel blocks per SM

constexpr int kMaxNp = 144;   // largest spline point count int(s_w*sub)

// variant 1: fused single kernel with a local-memory spline workspace;
// variant 0: split (k_vturb + k_advect, `turbv` is n doubles of scratch)
cudaError_t launch_step(const RpStepArgs& A, int field_dtype, int npmax, double* turbv, int variant,
                        cudaStream_t s, int num_sms, int* nlaunch);
// Split step with the scratch array in a static device buffer (no device
// allocation); at most kNoallocMaxParticles particles and np <= 128.
constexpr int64_t kNoallocMaxParticles = 1048576;
cudaError_t launch_step_noalloc(const RpStepArgs& A, int field_dtype, int npmax, int device, cudaStream_t s,
                                int num_sms, int* nlaunch);

// Mixed-precision form (rp_mixed.cu): the step, the 16-bit (FP16 or int16
// fixed point, `i16`) quantisation of a
// frame field staged as FP32 (Fortran order), and the conversions between
// the FP64 columns and the compensated FP32 positions.
// split: VTurb kernel (displacements into `turbv`, n floats) then the rest
cudaError_t launch_step_mixed(const RpStepArgs& A, int npmax, int i16, float* turbv, int split, cudaStream_t s,
                              int num_sms, int* nlaunch);
cudaError_t launch_stage_f32(int src_f32, const void* src, const void* add, float* dst, int64_t e0, int64_t count,
                             cudaStream_t s);
cudaError_t launch_quantize(const float* f, uint32_t* maxbits, float* qs, void* dst, int ni, int nj, int nk, int slot,
                            int i16, int num_sms, cudaStream_t s);
cudaError_t launch_mixed_convert(const RpParticlesDev& P, int to_f64, cudaStream_t s);
// Mixed form: clear one physical slot of a ring of `count` (point, level)
// entries of `elem` bytes per slot (2: 16-bit fields, 4: FP32), so that a
// slot read with weight 0 holds +0.
cudaError_t launch_clear_slot(void* ring, int elem, int64_t count, int slot, int num_sms, cudaStream_t s);

// Re-sorting of the particle state by (grid, tile of cells, cell) (rp_sort.cu)
struct SortBufs {
    uint32_t* keys = nullptr;      // n
    uint32_t* hist = nullptr;      // nkeys counters, then offsets
    uint32_t* sums = nullptr;      // scan block totals (<= 1024)
    int32_t* perm = nullptr;       // n: new slot -> old index
    uint32_t* gbase = nullptr;     // first key of each grid (RP_MAXNGRID_D)
    int64_t nkeys = 0;
};
constexpr int64_t kSortMaxKeys = 1024 * 1024;
int64_t sort_key_count(const RpStepArgs& A, uint32_t* gbase_host);
// sorts A.p's columns in place; `scratch8` holds n 8-byte values
cudaError_t launch_sort(const RpStepArgs& A, int mixed, const SortBufs& b, void* scratch8, cudaStream_t s,
                        int* nlaunch);
// dst[pid[i] - base] = src[i] for pid[i] - base < nout (elem = 8, 4 or 1 bytes)
cudaError_t launch_unsort(int elem, const void* src, void* dst, const uint32_t* pid, uint32_t base, int64_t n,
                          int64_t nout, cudaStream_t s);

// Adjoint pair (rp_adjoint.cu).  State columns of the adjoint model.
struct AdjStateDev {
    double* x;
    double* y;
    double* z;
    double* age;
    double* status;
    int32_t* gid;
    int8_t* isin;
};
// kind 0: step (find: search and record p in prec, else replay prec);
// 1: tangent step (t: 12 derivatives per particle); 2: reverse step
// (lx/ly/lz: lambda in/out, kbar: += dL/dkappa per particle)
cudaError_t launch_adj(int kind, const RpStepArgs& A, const AdjFrames& F, const AdjStateDev& s, double* prec, int find,
                       double kappa, double* t, double* lx, double* ly, double* lz, double* kbar, int npmax,
                       cudaStream_t st, int num_sms);
cudaError_t launch_adj_store(const double* src, const double* add, double* dst, int ni, int nj, int nk, int64_t e0,
                             int64_t count, cudaStream_t s);
cudaError_t launch_adj_tangent_init(double* t, int64_t n, cudaStream_t s);

// LL2ij of n particles in one grid (rp_init.cu)
cudaError_t launch_ll2ij(const double* lon, const double* lat, const double* angle, int nx, int ny, int spherical,
                         const double* inlon, const double* inlat, int64_t n, double* ip, double* jp, int num_sms,
                         cudaStream_t s);
cudaError_t launch_locate(const RpStepArgs& A, int field_dtype, const double* ipos, const double* jpos,
                          const double* z, const double* dob, cudaStream_t s);
cudaError_t launch_convert(int src_f32, int dst_f32, const void* src, const void* add, void* dst, int ni, int nj,
                           int nk, int slot, int64_t e0, int64_t count, cudaStream_t s);
cudaError_t launch_state_from_host(const RpParticlesDev& P, const double* gid_d, const int32_t* isin_i,
                                   uint32_t base, cudaStream_t s);
cudaError_t launch_state_to_host(const RpParticlesDev& P, double* gid_d, int32_t* isin_i, cudaStream_t s);
// dst[e * RP_SLOTS + slot] = src[e]: one WETDRY mask into its ring slot
cudaError_t launch_mask_slot(const uint8_t* src, uint8_t* dst, int64_t n, int slot, cudaStream_t s);
// the writer's resets of the diagnostics after an output record
cudaError_t launch_diag_reset(const RpParticlesDev& P, cudaStream_t s);

// One output record (dataOutput / writeNetCDF): the requested columns
// (null: not wanted) in the caller's particle order, each nout doubles.
struct OutCols {
    double* lon;
    double* lat;
    double* zp;
    double* age;
    double* status;
    double* gid;
    double* salt;
    double* temp;
    double* hob;
    double* bustr;
    double* bvstr;
};
// permuted: particle i goes to row pid[i] - base (rows >= nout dropped);
// mI: the writer's step count dividing the sums (SaltTempMean)
cudaError_t launch_output(const RpStepArgs& A, const OutCols& o, int permuted, uint32_t base, int64_t nout, int mI,
                          cudaStream_t s);

}  // namespace rp
