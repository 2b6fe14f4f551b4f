// rp_kernels.cu -- sm_100a kernels of the ROMSPath particle step.
// Compiled with -fmad=false: every FP64 expression rounds exactly as the
// reference's left-to-right evaluation (no FMA contraction).
#include <cuda_runtime.h>

#include "rp_internal.h"
#include "rp_step.cuh"

namespace rp {

// ------------------------------------------------------------ the step
//
// Split form: k_vturb_local (VTurb of each particle, spline workspace in
// local memory, many resident warps) writes each particle's displacement to
// scratch; k_advect (RK4, HTurb, hand-off, vertical update, status) then
// runs at its own register count.  Fused form: one kernel per particle.

// VTurb alone with the spline workspace in local memory, at high occupancy
// (the latency of the FP64 dependency chains and of the workspace loads is
// hidden by many resident warps).
template <typename T, int NPMAX>
__global__ void __launch_bounds__(kStepBlock, kVturbMinBlocks) k_vturb_local(const __grid_constant__ RpStepArgs A,
                                                                            double* __restrict__ turbv) {
    double buf[kSplineArrays * (NPMAX + 1)];
    const SplineView<NPMAX, 1> w{buf};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride)
        rp_vturb_one<T>(A, n, w, turbv);
}

template <typename T>
__global__ void __launch_bounds__(kStepBlock) k_advect(const __grid_constant__ RpStepArgs A,
                                                      const double* __restrict__ turbv) {
    const SplineView<1, 1> none{nullptr};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride)
        rp_update_one<T>(A, n, none, turbv);
}

template <typename T, int NPMAX>
__global__ void __launch_bounds__(kStepBlock, kVturbMinBlocks) k_step_fused(const __grid_constant__ RpStepArgs A) {
    double buf[kSplineArrays * (NPMAX + 1)];
    const SplineView<NPMAX, 1> w{buf};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < A.p.n; n += stride)
        rp_update_one<T>(A, n, w, nullptr);
}

template <class K>
static int64_t grid_for(K kernel, int block, size_t smem, int64_t n, int num_sms, cudaError_t* err, int cap = 0) {
    int occ = 0;
    *err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, block, smem);
    if (occ < 1) occ = 1;
    if (cap > 0 && occ > cap) occ = cap;
    int64_t need = (n + block - 1) / block;
    int64_t blocks = (int64_t)num_sms * occ;
    if (need < blocks) blocks = need;
    return blocks < 1 ? 1 : blocks;
}

template <typename T, int NPMAX>
static cudaError_t launch_step_t(const RpStepArgs& A, double* turbv, int variant, cudaStream_t s, int num_sms,
                                 int* nlaunch) {
    cudaError_t e = cudaSuccess;
    if (variant == 1) {
        const int64_t blocks = grid_for(k_step_fused<T, NPMAX>, kStepBlock, 0, A.p.n, num_sms, &e, A.grid_cap);
        if (e != cudaSuccess) return e;
        k_step_fused<T, NPMAX><<<(unsigned)blocks, kStepBlock, 0, s>>>(A);
        *nlaunch += 1;
        return cudaGetLastError();
    }
    if (A.vturb_on) {
        const int64_t blocks = grid_for(k_vturb_local<T, NPMAX>, kStepBlock, 0, A.p.n, num_sms, &e, A.grid_cap);
        if (e != cudaSuccess) return e;
        k_vturb_local<T, NPMAX><<<(unsigned)blocks, kStepBlock, 0, s>>>(A, turbv);
        *nlaunch += 1;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    const int64_t blocks = grid_for(k_advect<T>, kStepBlock, 0, A.p.n, num_sms, &e, A.grid_cap);
    if (e != cudaSuccess) return e;
    k_advect<T><<<(unsigned)blocks, kStepBlock, 0, s>>>(A, A.vturb_on ? turbv : nullptr);
    *nlaunch += 1;
    return cudaGetLastError();
}

cudaError_t launch_step(const RpStepArgs& A, int field_dtype, int npmax, double* turbv, int variant,
                        cudaStream_t s, int num_sms, int* nlaunch) {
    if (field_dtype == 1) {
        if (npmax <= 88) return launch_step_t<float, 88>(A, turbv, variant, s, num_sms, nlaunch);
        if (npmax <= 128) return launch_step_t<float, 128>(A, turbv, variant, s, num_sms, nlaunch);
        return launch_step_t<float, 144>(A, turbv, variant, s, num_sms, nlaunch);
    }
    if (npmax <= 88) return launch_step_t<double, 88>(A, turbv, variant, s, num_sms, nlaunch);
    if (npmax <= 128) return launch_step_t<double, 128>(A, turbv, variant, s, num_sms, nlaunch);
    return launch_step_t<double, 144>(A, turbv, variant, s, num_sms, nlaunch);
}

// -------------------------------------------- initial ownership (init)

// The grid loop of ini_ROMSPath (ROMSPath.f90:319-432): defaults, then for
// ng = 1..Ngrid the first grid whose bounds() says in-grid takes the
// particle, and zbounds() (boundary_module.f90:145-179) fixes z.  With the
// diagnostics on, their initial values (247-264, 353-355) and, for
// SaltTempOn, salinity, temperature, water depth, zeta and bathymetry at
// the particle from slot t_c (408-427).
template <typename T>
__global__ void k_locate(const __grid_constant__ RpStepArgs A, const double* ipos, const double* jpos,
                         const double* z, const double* dob) {
    const RpParticlesDev& P = A.p;
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.n) return;
    P.status[n] = 9.0;
    P.age[n] = 0.0;
    P.gid[n] = A.ngrid;
    P.isin[n] = 0;
    P.wd[n] = 9999.0;
    P.bath[n] = 9999.0;
    P.zeta[n] = 9999.0;
    P.x[n] = 1.0;
    P.y[n] = 1.0;
    P.z[n] = z[n];
    P.dob[n] = dob[n];
    P.pid[n] = A.pid_base + (uint32_t)n;
    uint32_t fl = 0;
    for (int ng = 1; ng <= A.ngrid; ng++) {
        const RpGridDev& g = A.g[ng - 1];
        const double I = ipos[(int64_t)(ng - 1) * P.n + n], J = jpos[(int64_t)(ng - 1) * P.n + n];
        bool ingrid, obound;
        rp_bounds(g, I, J, ingrid, obound);
        if (!P.isin[n] && ingrid) {
            P.x[n] = I;
            P.y[n] = J;
            P.gid[n] = ng;
            P.status[n] = 0.0;
            P.isin[n] = 1;
            bool inz = false;
            double Z = P.z[n];
            if (rp_ifloor(I) > 0) {
                RhoCell rc;
                rp_rho_cell(g, I, J, rc, fl);
                const double tdepth = -1.0 * rp_bil(g.h, rc);
                const double tzeta = rp_zeta_at<T>(g, rc, g.sb);
                if ((Z < tzeta) && (Z > tdepth)) inz = true;
                if (Z >= tzeta) {
                    Z = tzeta - 0.01;
                    inz = true;
                }
            }
            P.z[n] = Z;
            if (!inz) P.status[n] = 9.0;
        }
    }
    if (P.acc) {                           // par(:,pAcc/pVort/pbehaveW/pSSF), 343-346
        P.acc[n] = 0.0;
        P.vort[n] = 0.0;
        P.behavew[n] = 0.0;
        P.ssf[n] = 0.0;
    }
    if (A.diag & RP_DIAG_BOTTOM_D) {
        P.hob[n] = 9999.0;
        P.bustr[n] = 0.0;
        P.bvstr[n] = 0.0;
    }
    if (A.diag & RP_DIAG_SALTTEMP_D) {
        double s = 0.0, t = 0.0;
        if (P.isin[n]) {
            const RpGridDev& g = A.g[P.gid[n] - 1];
            const double X = P.x[n], Y = P.y[n], Z = P.z[n];
            RhoCell rc;
            rp_rho_cell(g, X, Y, rc, fl);
            const double tdepth = -1.0 * rp_bil(g.h, rc);
            const double zeta = rp_zeta_at<T>(g, rc, g.sc);
            double wcf[4];                                 // WETDRY: slot t_c's weights
            if (A.wetdry) rp_rho_wd_weights(g, rc, g.sc, wcf, fl);
            s = rp_tracer_at<T>(g, g.salt, rc, zeta, tdepth, Z, g.sc, A.wetdry ? wcf : nullptr);
            t = rp_tracer_at<T>(g, g.temp, rc, zeta, tdepth, Z, g.sc, A.wetdry ? wcf : nullptr);
            P.wd[n] = (-1.0 * tdepth) + zeta;
            P.zeta[n] = zeta;
            P.bath[n] = -1.0 * tdepth;
        }
        P.salt[n] = s;
        P.temp[n] = t;
        if (A.diag & RP_DIAG_MEAN_D) {
            P.mean_salt[n] = s;
            P.mean_temp[n] = t;
        }
    }
    P.flags[n] = fl;
}

cudaError_t launch_locate(const RpStepArgs& A, int field_dtype, const double* ipos, const double* jpos,
                          const double* z, const double* dob, cudaStream_t s) {
    const int block = 256;
    const unsigned blocks = (unsigned)((A.p.n + block - 1) / block);
    if (blocks == 0) return cudaSuccess;
    if (field_dtype == 1) k_locate<float><<<blocks, block, 0, s>>>(A, ipos, jpos, z, dob);
    else k_locate<double><<<blocks, block, 0, s>>>(A, ipos, jpos, z, dob);
    return cudaGetLastError();
}

// ------------------------------------------------------ frame upload

// Fortran-layout source field (i fastest, then j, then k) -> device layout
// [j][i][k][slot4].  With `add` non-null the two are summed in FP64 first
// (u += ustokes, hydrodynamic_module.f90:606-660), then rounded to T.
template <typename S, typename T>
__global__ void k_convert(const S* __restrict__ src, const S* __restrict__ add, T* __restrict__ dst, int ni,
                          int nj, int nk, int slot, int64_t e0, int64_t count) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int64_t e = e0 + t;
    const int64_t plane = (int64_t)ni * nj;
    const int k = (int)(e / plane);
    const int64_t r = e - (int64_t)k * plane;
    const int j = (int)(r / ni);
    const int i = (int)(r - (int64_t)j * ni);
    double v = (double)src[t];
    if (add) v = v + (double)add[t];
    dst[(((int64_t)j * ni + i) * nk + k) * RP_SLOTS + slot] = (T)v;
}

cudaError_t launch_convert(int src_f32, int dst_f32, const void* src, const void* add, void* dst, int ni, int nj,
                           int nk, int slot, int64_t e0, int64_t count, cudaStream_t s) {
    const int block = 256;
    const unsigned blocks = (unsigned)((count + block - 1) / block);
    if (blocks == 0) return cudaSuccess;
    if (src_f32) {
        if (dst_f32)
            k_convert<float, float><<<blocks, block, 0, s>>>((const float*)src, (const float*)add, (float*)dst, ni,
                                                             nj, nk, slot, e0, count);
        else
            k_convert<float, double><<<blocks, block, 0, s>>>((const float*)src, (const float*)add, (double*)dst,
                                                              ni, nj, nk, slot, e0, count);
    } else {
        if (dst_f32)
            k_convert<double, float><<<blocks, block, 0, s>>>((const double*)src, (const double*)add, (float*)dst,
                                                              ni, nj, nk, slot, e0, count);
        else
            k_convert<double, double><<<blocks, block, 0, s>>>((const double*)src, (const double*)add,
                                                               (double*)dst, ni, nj, nk, slot, e0, count);
    }
    return cudaGetLastError();
}

__global__ void k_mask_slot(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int64_t n, int slot) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) dst[e * RP_SLOTS + slot] = src[e];
}

cudaError_t launch_mask_slot(const uint8_t* src, uint8_t* dst, int64_t n, int slot, cudaStream_t s) {
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (blocks == 0) return cudaSuccess;
    k_mask_slot<<<blocks, 256, 0, s>>>(src, dst, n, slot);
    return cudaGetLastError();
}

// ----------------------------------------------------- state helpers

__global__ void k_state_from_host(RpParticlesDev P, const double* gid_d, const int32_t* isin_i, uint32_t base) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.n) return;
    P.gid[n] = (int32_t)gid_d[n];          // int(par(n,pGID))
    P.isin[n] = isin_i[n] ? 1 : 0;
    P.pid[n] = base + (uint32_t)n;
    P.flags[n] = 0u;
    // diagnostics as the particle read loop leaves them (ROMSPath.f90:247-264, 353-355)
    if (P.hob) {
        P.hob[n] = 9999.0;
        P.bustr[n] = 0.0;
        P.bvstr[n] = 0.0;
    }
    if (P.salt) {
        P.salt[n] = 0.0;
        P.temp[n] = 0.0;
    }
    if (P.mean_salt) {
        P.mean_salt[n] = 0.0;
        P.mean_temp[n] = 0.0;
    }
    if (P.acc) {                           // par(:,pAcc/pVort/pbehaveW/pSSF), 343-346
        P.acc[n] = 0.0;
        P.vort[n] = 0.0;
        P.behavew[n] = 0.0;
        P.ssf[n] = 0.0;
    }
}

cudaError_t launch_state_from_host(const RpParticlesDev& P, const double* gid_d, const int32_t* isin_i,
                                   uint32_t base, cudaStream_t s) {
    const int block = 256;
    const unsigned blocks = (unsigned)((P.n + block - 1) / block);
    if (blocks == 0) return cudaSuccess;
    k_state_from_host<<<blocks, block, 0, s>>>(P, gid_d, isin_i, base);
    return cudaGetLastError();
}

__global__ void k_state_to_host(RpParticlesDev P, double* gid_d, int32_t* isin_i) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.n) return;
    gid_d[n] = (double)P.gid[n];
    isin_i[n] = (int32_t)P.isin[n];
}

cudaError_t launch_state_to_host(const RpParticlesDev& P, double* gid_d, int32_t* isin_i, cudaStream_t s) {
    const int block = 256;
    const unsigned blocks = (unsigned)((P.n + block - 1) / block);
    if (blocks == 0) return cudaSuccess;
    k_state_to_host<<<blocks, block, 0, s>>>(P, gid_d, isin_i);
    return cudaGetLastError();
}

// The writer's resets after an output record (ROMSPath.f90:2030-2035,
// 2064): the running sums of salinity and temperature to 0, P_HOB to 9999.
__global__ void k_diag_reset(RpParticlesDev P) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.n) return;
    if (P.mean_salt) {
        P.mean_salt[n] = 0.0;
        P.mean_temp[n] = 0.0;
    }
    if (P.hob) P.hob[n] = 9999.0;
}

// dataOutput and the record of writeNetCDF (ROMSPath.f90:1012-1024,
// 1924-2070) for every particle: pLon, pLat by getInterp2D("lon"/"lat",
// pGID, pX, pY) (plain bilinear, 466-477), zp, age, status, GID and the
// diagnostics (salt/temp as sum / mI under SaltTempMean, 2010-2014), each
// into its row of the packed record; then the writer's resets (2030-2035,
// 2064).
__global__ void k_output(const __grid_constant__ RpStepArgs A, const OutCols o, int permuted, uint32_t base,
                         int64_t nout, int mI) {
    const RpParticlesDev& P = A.p;
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.n) return;
    const int64_t r = permuted ? (int64_t)(P.pid[n] - base) : n;
    if (r >= 0 && r < nout) {
        if (o.lon || o.lat) {
            const RpGridDev& g = A.g[P.gid[n] - 1];
            const double ip = P.x[n], jp = P.y[n];
            uint32_t fl = 0;                   // clamped, not recorded: output changes no state
            const int I = rp_ifloor(ip), J = rp_ifloor(jp);
            const double X = ip - (double)I, Y = jp - (double)J;
            const int i0 = rp_clamp(I, 1, g.nx, fl), i1 = rp_clamp(I + 1, 1, g.nx, fl);
            const int j0 = rp_clamp(J, 1, g.ny, fl), j1 = rp_clamp(J + 1, 1, g.ny, fl);
            const int64_t o00 = (int64_t)(j0 - 1) * g.nx + (i0 - 1), o10 = (int64_t)(j0 - 1) * g.nx + (i1 - 1);
            const int64_t o11 = (int64_t)(j1 - 1) * g.nx + (i1 - 1), o01 = (int64_t)(j1 - 1) * g.nx + (i0 - 1);
            const double c0 = (1 - X) * (1 - Y), c1 = X * (1 - Y), c2 = X * Y, c3 = (1 - X) * Y;
            if (o.lon)
                o.lon[r] = c0 * __ldg(g.lon + o00) + c1 * __ldg(g.lon + o10) + c2 * __ldg(g.lon + o11) +
                           c3 * __ldg(g.lon + o01);
            if (o.lat)
                o.lat[r] = c0 * __ldg(g.lat + o00) + c1 * __ldg(g.lat + o10) + c2 * __ldg(g.lat + o11) +
                           c3 * __ldg(g.lat + o01);
        }
        if (o.zp) o.zp[r] = P.z[n];
        if (o.age) o.age[r] = P.age[n];
        if (o.status) o.status[r] = P.status[n];
        if (o.gid) o.gid[r] = (double)P.gid[n];
        if (A.diag & RP_DIAG_SALTTEMP_D) {
            const bool mean = (A.diag & RP_DIAG_MEAN_D) != 0;
            if (o.salt) o.salt[r] = mean ? P.mean_salt[n] / (double)mI : P.salt[n];
            if (o.temp) o.temp[r] = mean ? P.mean_temp[n] / (double)mI : P.temp[n];
        }
        if (A.diag & RP_DIAG_BOTTOM_D) {
            if (o.hob) o.hob[r] = P.hob[n];
            if (o.bustr) o.bustr[r] = P.bustr[n];
            if (o.bvstr) o.bvstr[r] = P.bvstr[n];
        }
    }
    if (A.diag & RP_DIAG_MEAN_D) {
        P.mean_salt[n] = 0.0;
        P.mean_temp[n] = 0.0;
    }
    if (A.diag & RP_DIAG_BOTTOM_D) P.hob[n] = 9999.0;
}

cudaError_t launch_output(const RpStepArgs& A, const OutCols& o, int permuted, uint32_t base, int64_t nout, int mI,
                          cudaStream_t s) {
    const int block = 256;
    const unsigned blocks = (unsigned)((A.p.n + block - 1) / block);
    if (blocks == 0) return cudaSuccess;
    k_output<<<blocks, block, 0, s>>>(A, o, permuted, base, nout, mI);
    return cudaGetLastError();
}

cudaError_t launch_diag_reset(const RpParticlesDev& P, cudaStream_t s) {
    const int block = 256;
    const unsigned blocks = (unsigned)((P.n + block - 1) / block);
    if (blocks == 0) return cudaSuccess;
    k_diag_reset<<<blocks, block, 0, s>>>(P);
    return cudaGetLastError();
}

}  // namespace rp
