// rp_device.cuh -- device data layout and the arithmetic of the ROMSPath
// particle step for sm_100a.
//
// Layout in HBM (per grid):
//   h, pm, pn            double [j][i]               (static)
//   mask_rho/u/v         uint8  [j][i]               (static)
//   zeta                 T      [j][i][slot4]
//   u   (xi_u=nx-1)      T      [j][i][k][slot4]     k = 0..N-1
//   v   (eta_v=ny-1)     T      [j][i][k][slot4]
//   w, aks               T      [j][i][k][slot4]     k = 0..N
// The four ring slots of one (i,j,k) are adjacent, so the time stencil
// (b, c, f) of a corner and its two bracketing levels are one or two
// sectors.  T is double or float (the reference stores DOUBLE PRECISION;
// float storage keeps FP64 arithmetic on FP32-rounded values).
//
// Arithmetic: every expression keeps the reference's evaluation order and
// is compiled without FMA contraction, so results are bit-identical to the
// CPU restatement of the reference.  Work the reference repeats with
// identical operands (the nine getInterp3D level walks of a RK stage, the
// per-call mask/weight set-up, the three getWlevel S factors of a level) is
// done once here; each value is still produced by the same operations.
#pragma once

#include <cstdint>

#define RP_MAXNGRID_D 5
#define RP_SLOTS 4

// Fortran single-precision literals widened to double in the reference.
#define RP_F_0P001 ((double)0.001f)  // DBLE(0.001), advection_module.f90:174,182
#define RP_F_0P1 ((double)0.1f)      // ecut=0.1, boundary_module.f90:59
#define RP_F_1P1 ((double)1.1f)      // pStatus=1.1, ROMSPath.f90:882
#define RP_F_1P2 ((double)1.2f)      // pStatus=1.2, ROMSPath.f90:883

#define RP_FL_OOB 0x01u
#define RP_FL_NODE 0x02u
#define RP_FL_WBOT 0x04u
#define RP_FL_WTOP 0x08u
#define RP_FL_SPLINE 0x10u

struct RpGridDev {
    int nx, ny, N;                 // rho dims, s_rho
    int vtransform;
    double hc;
    const double* h;
    const double* pm;
    const double* pn;
    const uint8_t* mrho;
    const uint8_t* mu;
    const uint8_t* mv;
    const double* sr;              // s_rho[N]
    const double* csr;             // Cs_r[N]
    const double* sw;              // s_w[N+1]
    const double* csw;             // Cs_w[N+1]
    const float2* scs_r;           // (s_rho, Cs_r)[N] in FP32 (the mixed form)
    const float2* scs_w;           // (s_w, Cs_w)[N+1] in FP32
    const float2* hm;              // (h, mask_rho) per rho point in FP32 (the mixed form)
    const void* zeta;
    const void* u;
    const void* v;
    const void* w;
    const void* aks;
    // diagnostics only: salt, temp [j][i][k][slot4] (N levels); bustr on
    // the u points, bvstr on the v points, [j][i][slot4]
    const void* salt;
    const void* temp;
    const void* bustr;
    const void* bvstr;
    // WETDRY: wetdry_mask_rho / _u / _v of the frames, [j][i][slot4] (0/1)
    const uint8_t* wd_rho;
    const uint8_t* wd_u;
    const uint8_t* wd_v;
    // behave's fields (Process_VA / _WA): Accelstd_t, Vortstd_t,
    // Accelustd_w, Accelvstd_w, [j][i][k][slot4] on the N+1 w levels
    const void* turbaccel;
    const void* turbvort;
    const void* waveaccelu;
    const void* waveaccelv;
    const double* lon;             // lon_rho, lat_rho [j][i] (output only)
    const double* lat;
    double scl[RP_MAXNGRID_D][2];  // GRIDS(ng)%scl(i,1:2)
    double off[RP_MAXNGRID_D][2];
    int sb, sc, sf;                // physical ring slots of t_b, t_c, t_f
    // mixed form, per step (host-computed): the Lagrange weights by physical
    // slot ([0] zeta/AKs/depths, [1] u/v/w), and bit masks of the three
    // live slots of an FP32 float4
    float4 w4[2];
    uint4 m32;
    // mixed form: per-(level, slot) scales of the 16-bit fields, [k][slot4]
    const float* qs_u;
    const float* qs_v;
    const float* qs_w;
    const float* qs_aks;
};

struct RpParticlesDev {
    int64_t n;
    double* x;
    double* y;
    double* z;
    double* age;
    double* dob;
    double* status;
    double* wd;
    double* zeta;
    double* bath;
    int32_t* gid;
    int8_t* isin;
    uint32_t* pid;
    uint32_t* flags;
    // mixed form: FP32 positions with Kahan compensation (value = p - c)
    // and the smoothing-spline warm start (last q, < 0 for none; slope of
    // 1/sqrt(SF) in q there, <= 0 for none)
    float* x32;
    float* y32;
    float* z32;
    float* cx;
    float* cy;
    float* cz;
    double* qwarm;
    double* gwarm;
    float* qwarm2;                 // the smoothing parameter of the step before qwarm's
    // diagnostics (ROMSPath.f90:130-131): P_Salt, P_Temp, mean_salt,
    // mean_temp (running sums), P_HOB, P_bustr, P_bvstr
    double* salt;
    double* temp;
    double* mean_salt;
    double* mean_temp;
    double* hob;
    double* bustr;
    double* bvstr;
    // behave's outputs par(:,pAcc/pVort/pbehaveW/pSSF) (ROMSPath.f90:800-804)
    double* acc;
    double* vort;
    double* behavew;
    double* ssf;
};

// behave's switches and parameters (behavparam, fuchsparam; ROMSPath.h:
// 150-189; initsize = par(:,pSize), 199)
struct RpBehaviorDev {
    int behavior;                  // 0, 1, 10 or 11
    int va, wa, va_flag;           // Process_VA, Process_WA, va_flag
    double swimfast, initsize;
    double vort_cr, vort_sat, b0pv, b1pv, b0wv, b1w, acc_cr, acc_sat, b0pa, b1pa, b0wa;
};

// RpStepArgs::diag bits (namelist "other", ROMSPath.h:325-330)
#define RP_DIAG_SALTTEMP_D 1       // SaltTempOn
#define RP_DIAG_MEAN_D 2           // SaltTempMean
#define RP_DIAG_BOTTOM_D 4         // WriteBottom

// Frame-store pointers of the three time levels (b, c, f) of one step of the
// adjoint model: f[grid][field][t], field 0 zeta [j][i], 1 u, 2 v, 3 w,
// 4 AKs [j][i][k] (FP64, one frame each).
struct AdjFrames {
    const double* f[RP_MAXNGRID_D][5][3];
};

// polintd (interpolation_module.f90:72-109) at fixed nodes ex(3) and point
// x: the node-only terms, identical to the reference's subexpressions.
struct RpPolint {
    double d1;    // xa(2)-x
    double e12;   // xa(2)-xa(3)
    double e01;   // xa(1)-xa(2)
    double e02;   // xa(1)-xa(3)
    double dns;   // xa(ns)-x
    double b;     // xa(3)-x (ns==3) or xa(1)-x
    double re12, re01, re02;  // RN(1/e12), RN(1/e01), RN(1/e02)
    int ns;       // 0-based nearest node
};

struct RpStepArgs {
    double ex[3], ix[3];
    RpPolint pi;                   // polintd constants for x = ix(2)
    // mixed form: polintd at ix(2) as Lagrange weights of the b, c, f slots;
    // [0] zeta, AKs and level depths, [1] u, v, w (at ets == 1 the values
    // are (b, b, c), advection_module.f90:277-287)
    float lw[2][3];
    int ets;
    int ngrid;
    int idt, scheme, nsb, vturb_on, hturb_on, oob;
    int loop;                      // idt / int(deltat)
    int grid_cap;                  // resident blocks per SM of the step kernels (0: occupancy limit)
    int spline_max_iter;
    int diag;                      // RP_DIAG_*_D bits
    int wetdry;                    // WETDRY: time-varying masks in getInterp3D / getInterpStr
    RpBehaviorDev beh;
    double vertdist, serr, smth, sub, deltat, aksback;
    double khturb[RP_MAXNGRID_D];
    uint64_t seed, step_index;
    const double* hook;            // noise hook for this step, or nullptr
    unsigned long long* spl;       // [0] smoothing-spline fits, [1] chol1d passes; nullptr: not counted
    float* diag_td;                // mixed form with diagnostics: the step's tdepth per particle (NaN:
                                   // not stepped), read by the diagnostics pass; nullptr: none
    float* beh_z;                  // mixed form with behave: ZBehav per particle from the behave pass
    int ndraw;
    uint32_t pid_base;             // hook row of particle id p is p - pid_base
    RpGridDev g[RP_MAXNGRID_D];
    RpParticlesDev p;
};

// ------------------------------------------------------------------ basics

// Adds one fit of `passes` chol1d passes per calling thread to c[0], c[1]:
// the converged threads of the warp sum theirs and one lane adds the totals.
__device__ __forceinline__ void rp_count_fit(unsigned long long* c, int passes) {
    const unsigned m = __activemask();
    const unsigned tot = __reduce_add_sync(m, (unsigned)passes);
    unsigned lane;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(lane));
    if (lane == (unsigned)(__ffs(m) - 1)) {
        atomicAdd(c, (unsigned long long)__popc(m));
        atomicAdd(c + 1, (unsigned long long)tot);
    }
}

__device__ __forceinline__ int rp_ifloor(double x) {
    double f = floor(x);
    if (!(f >= -1.0e9)) return -1000000000;
    if (f > 1.0e9) return 1000000000;
    return (int)f;
}

__device__ __forceinline__ int rp_clamp(int v, int lo, int hi, uint32_t& fl) {
    if (v < lo) { fl |= RP_FL_OOB; return lo; }
    if (v > hi) { fl |= RP_FL_OOB; return hi; }
    return v;
}

template <typename T>
__device__ __forceinline__ double rp_ld(const void* base, int64_t idx) {
    return (double)__ldg(reinterpret_cast<const T*>(base) + idx);
}

// ------------------------------------------------------ exact division
//
// a / b rounded to nearest, given y = RN(1/b) (CUDA's __drcp_rn): two
// residual corrections q <- q + (a - b q) y with the residual formed exactly
// by an FMA.  By Markstein's theorem (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990), if y = RN(1/b) and q is within one ulp of a/b, then
// RN(q + (a - bq) y) = RN(a/b); the first correction brings RN(a y) within
// one ulp.  Operands outside [1e-150, 1e150] in magnitude (where a residual
// could underflow), zero, Inf or NaN take the IEEE division instead, so the
// result is always the correctly rounded quotient -- the value `a / b`
// gives -- while divisions sharing a denominator share one reciprocal.
__device__ __forceinline__ bool rp_div_safe(double b) {
    const double ab = fabs(b);
    return ab > 1e-150 && ab < 1e150;
}

__device__ __forceinline__ double rp_rcp(double b) { return __drcp_rn(b); }

__device__ __forceinline__ double rp_div_by(double a, double b, double y) {
    const double aa = fabs(a);
    if (!(aa > 1e-150 && aa < 1e150) || !rp_div_safe(b)) return a / b;
    const double q0 = a * y;
    const double r0 = fma(-b, q0, a);
    const double q1 = fma(r0, y, q0);
    const double r1 = fma(-b, q1, a);
    return fma(r1, y, q1);
}

__device__ __forceinline__ double rp_polintd(const RpPolint& P, double y0, double y1, double y2) {
    const double q12 = rp_div_by(y2 - y1, P.e12, P.re12);
    const double q01 = rp_div_by(y1 - y0, P.e01, P.re01);
    double c = P.d1 * q12;
    c = c - P.d1 * q01;
    c = rp_div_by(c, P.e02, P.re02);
    const double a = (P.ns == 2) ? q12 : q01;
    const double yns = (P.ns == 0) ? y0 : ((P.ns == 1) ? y1 : y2);
    return yns + P.dns * a + P.b * c;
}

// getcoeff (interpolation_module.f90:1230-1273) with the exact-node pin.
__device__ __forceinline__ void rp_getcoeff(double X, double Y, const double m[4], double cff[4],
                                            uint32_t& fl) {
    double dist[4], W[4];
    dist[0] = sqrt(X * X + Y * Y);
    dist[1] = sqrt((1 - X) * (1 - X) + Y * Y);
    dist[2] = sqrt((1 - X) * (1 - X) + (1 - Y) * (1 - Y));
    dist[3] = sqrt(X * X + (1 - Y) * (1 - Y));
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (dist[k] == 0.0) {
            fl |= RP_FL_NODE;
            if (m[k] != 0.0) {
#pragma unroll
                for (int q = 0; q < 4; q++) cff[q] = (q == k) ? 1.0 : 0.0;
                return;
            }
            W[k] = 0.0;
        } else {
            // masks are 0 or 1: m/dist is RN(1/dist) or +0
            W[k] = (m[k] != 0.0) ? rp_rcp(dist[k]) : m[k] / dist[k];
        }
    }
    const double WT = W[0] + W[1] + W[2] + W[3];
    if (WT == 0.0) {
#pragma unroll
        for (int k = 0; k < 4; k++) cff[k] = 0.0;
    } else {
        const double yWT = rp_rcp(WT);
#pragma unroll
        for (int k = 0; k < 4; k++) cff[k] = rp_div_by(W[k], WT, yWT);
    }
}

// ------------------------------------------------------------- stencils

// rho-point cell of (ip, jp): the set-up shared by getInterp2D (depth, pm,
// pn, zeta), the w/AKs paths of getInterp3D and getInterpAKs.
struct RhoCell {
    int64_t o00, o10, o11, o01;    // [j][i] offsets of corners 1..4
    double X, Y;
    double cb[4];                  // bilinear weights
    double ci[4];                  // getcoeff weights (masks of mask_rho)
    bool wet4;                     // nwater == 4
};

__device__ __forceinline__ void rp_rho_cell(const RpGridDev& g, double ip, double jp, RhoCell& c,
                                            uint32_t& fl) {
    const int I = rp_ifloor(ip), J = rp_ifloor(jp);
    c.X = ip - (double)I;
    c.Y = jp - (double)J;
    const int i0 = rp_clamp(I, 1, g.nx, fl), i1 = rp_clamp(I + 1, 1, g.nx, fl);
    const int j0 = rp_clamp(J, 1, g.ny, fl), j1 = rp_clamp(J + 1, 1, g.ny, fl);
    c.o00 = (int64_t)(j0 - 1) * g.nx + (i0 - 1);
    c.o10 = (int64_t)(j0 - 1) * g.nx + (i1 - 1);
    c.o11 = (int64_t)(j1 - 1) * g.nx + (i1 - 1);
    c.o01 = (int64_t)(j1 - 1) * g.nx + (i0 - 1);
    const double X = c.X, Y = c.Y;
    c.cb[0] = (1 - X) * (1 - Y);
    c.cb[1] = X * (1 - Y);
    c.cb[2] = X * Y;
    c.cb[3] = (1 - X) * Y;
    double m[4];
    m[0] = (double)__ldg(g.mrho + c.o00);
    m[1] = (double)__ldg(g.mrho + c.o10);
    m[2] = (double)__ldg(g.mrho + c.o11);
    m[3] = (double)__ldg(g.mrho + c.o01);
    const double nwater = m[0] + m[1] + m[2] + m[3];
    c.wet4 = !(nwater < 4.0);
    rp_getcoeff(X, Y, m, c.ci, fl);
}

// getInterp3D's weights of a rho-point field under WETDRY (interpolation_
// module.f90:769-939): the bilinear weights, or getcoeff's when a corner of
// slot `slot`'s wetdry_mask_rho is dry.
__device__ __forceinline__ void rp_rho_wd_weights(const RpGridDev& g, const RhoCell& c, int slot, double cff[4],
                                                  uint32_t& fl) {
    double m[4];
    m[0] = (double)__ldg(g.wd_rho + c.o00 * RP_SLOTS + slot);
    m[1] = (double)__ldg(g.wd_rho + c.o10 * RP_SLOTS + slot);
    m[2] = (double)__ldg(g.wd_rho + c.o11 * RP_SLOTS + slot);
    m[3] = (double)__ldg(g.wd_rho + c.o01 * RP_SLOTS + slot);
    const double nwater = m[0] + m[1] + m[2] + m[3];
    if (nwater < 4.0) {
        rp_getcoeff(c.X, c.Y, m, cff, fl);
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) cff[k] = c.cb[k];
    }
}

__device__ __forceinline__ double rp_bil(const double* a, const RhoCell& c) {
    return c.cb[0] * __ldg(a + c.o00) + c.cb[1] * __ldg(a + c.o10) + c.cb[2] * __ldg(a + c.o11) +
           c.cb[3] * __ldg(a + c.o01);
}

template <typename T>
__device__ __forceinline__ double rp_zeta_at(const RpGridDev& g, const RhoCell& c, int slot) {
    const double v0 = rp_ld<T>(g.zeta, c.o00 * RP_SLOTS + slot);
    const double v1 = rp_ld<T>(g.zeta, c.o10 * RP_SLOTS + slot);
    const double v2 = rp_ld<T>(g.zeta, c.o11 * RP_SLOTS + slot);
    const double v3 = rp_ld<T>(g.zeta, c.o01 * RP_SLOTS + slot);
    return c.ci[0] * v0 + c.ci[1] * v1 + c.ci[2] * v2 + c.ci[3] * v3;
}

// u / v corner set of getInterp3D (interpolation_module.f90:608-767).
struct UVCell {
    int64_t o[4];                  // [j][i] column offsets in the u or v grid
    double cff[4];
    bool use[4];
};

// The masks are mask_u (ms = 1, mo = 0) or, under WETDRY, the frame's
// wetdry_mask_u of one ring slot (mk = the slot ring, ms = RP_SLOTS, mo =
// the physical slot), hydrodynamic_module.f90:510-570.
__device__ __forceinline__ void rp_u_cell(const RpGridDev& g, double ip, double jp, UVCell& c,
                                          uint32_t& fl, const uint8_t* mk = nullptr, int ms = 1, int mo = 0) {
    if (!mk) mk = g.mu;
    const int xi_u = g.nx - 1, eta_u = g.ny;
    const int Jn = rp_ifloor(jp);
    const double Y = jp - (double)Jn;
    const double uvI = ip - 0.5;
    const int In = rp_ifloor(uvI);
    const double X = uvI - (double)In;
    c.cff[0] = (1 - X) * (1 - Y);
    c.cff[1] = X * (1 - Y);
    c.cff[2] = X * Y;
    c.cff[3] = (1 - X) * Y;
    const int j0 = rp_clamp(Jn, 1, eta_u, fl), j1 = rp_clamp(Jn + 1, 1, eta_u, fl);
    int ci[4];
    double m[4];
    if (In >= xi_u) {
        ci[0] = ci[1] = ci[2] = ci[3] = xi_u;
    } else if (In < 1) {
        ci[0] = ci[1] = ci[2] = ci[3] = 1;
    } else {
        ci[0] = In; ci[1] = In + 1; ci[2] = In + 1; ci[3] = In;
    }
    const int cj[4] = {j0, j0, j1, j1};
#pragma unroll
    for (int k = 0; k < 4; k++) c.o[k] = (int64_t)(cj[k] - 1) * xi_u + (ci[k] - 1);
    if (In >= xi_u) {
        m[0] = (double)__ldg(mk + c.o[0] * ms + mo); m[1] = 0; m[2] = 0; m[3] = (double)__ldg(mk + c.o[3] * ms + mo);
    } else if (In < 1) {
        m[0] = 0; m[1] = (double)__ldg(mk + c.o[1] * ms + mo); m[2] = (double)__ldg(mk + c.o[2] * ms + mo); m[3] = 0;
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) m[k] = (double)__ldg(mk + c.o[k] * ms + mo);
    }
    const double nwater = m[0] + m[1] + m[2] + m[3];
#pragma unroll
    for (int k = 0; k < 4; k++) c.use[k] = true;
    if (nwater < 4.0 && nwater > 0.0) {
#pragma unroll
        for (int k = 0; k < 4; k++) if (m[k] == 0.0) c.use[k] = false;
    } else if (nwater == 0.0) {
#pragma unroll
        for (int k = 0; k < 4; k++) { c.cff[k] = 0.0; c.use[k] = false; }
    }
}

__device__ __forceinline__ void rp_v_cell(const RpGridDev& g, double ip, double jp, UVCell& c,
                                          uint32_t& fl, const uint8_t* mk = nullptr, int ms = 1, int mo = 0) {
    if (!mk) mk = g.mv;
    const int xi_v = g.nx, eta_v = g.ny - 1;
    int In = rp_ifloor(ip);
    const double X = ip - (double)In;
    const double uvJ = jp - 0.5;
    int Jn = rp_ifloor(uvJ);
    if (Jn < 1) Jn = 1;
    if (Jn > eta_v) In = eta_v;     // interpolation_module.f90:696, kept
    const double Y = uvJ - (double)Jn;
    c.cff[0] = (1 - X) * (1 - Y);
    c.cff[1] = X * (1 - Y);
    c.cff[2] = X * Y;
    c.cff[3] = (1 - X) * Y;
    const int i0 = rp_clamp(In, 1, xi_v, fl), i1 = rp_clamp(In + 1, 1, xi_v, fl);
    const int ci[4] = {i0, i1, i1, i0};
    int cj[4];
    double m[4];
    if (Jn >= eta_v) {
        cj[0] = cj[1] = cj[2] = cj[3] = eta_v;
    } else {
        cj[0] = Jn; cj[1] = Jn; cj[2] = Jn + 1; cj[3] = Jn + 1;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) c.o[k] = (int64_t)(cj[k] - 1) * xi_v + (ci[k] - 1);
    if (Jn >= eta_v) {
        m[0] = (double)__ldg(mk + c.o[0] * ms + mo); m[1] = (double)__ldg(mk + c.o[1] * ms + mo); m[2] = 0; m[3] = 0;
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) m[k] = (double)__ldg(mk + c.o[k] * ms + mo);
    }
    const double nwater = m[0] + m[1] + m[2] + m[3];
#pragma unroll
    for (int k = 0; k < 4; k++) c.use[k] = true;
    if (nwater < 4.0 && nwater > 0.0) {
#pragma unroll
        for (int k = 0; k < 4; k++) if (m[k] == 0.0) c.use[k] = false;
    } else if (nwater == 0.0) {
#pragma unroll
        for (int k = 0; k < 4; k++) { c.cff[k] = 0.0; c.use[k] = false; }
    }
}

// --------------------------------------------------------- s-coordinates

// getSlevel / getWlevel (grid_module.f90:513-598) with h = -depth.
__device__ __forceinline__ double rp_zlevel(int vtransform, double hc, double s, double cs,
                                            double zeta, double h) {
    if (vtransform == 2) {
        const double S = (hc * s + h * cs) / (hc + h);
        return zeta + (zeta + h) * S;
    } else if (vtransform == 1) {
        const double S = hc * s + (h - hc) * cs;
        return S + zeta * (1.0 + S / h);
    }
    return zeta * (1.0 + s) + hc * s + (h - hc) * cs;
}

// getSlevel/getWlevel with the per-point divisor's reciprocal shared
// across levels (same quotients as the reference's divisions).
struct ZCtx {
    int vt;
    double hc, h, den, yden, yh;
};

__device__ __forceinline__ ZCtx rp_zctx(int vtransform, double hc, double h) {
    ZCtx c;
    c.vt = vtransform;
    c.hc = hc;
    c.h = h;
    c.den = hc + h;
    c.yden = rp_rcp(c.den);
    c.yh = rp_rcp(h);
    return c;
}

__device__ __forceinline__ double rp_zlevel_c(const ZCtx& c, double s, double cs, double zeta) {
    if (c.vt == 2) {
        const double S = rp_div_by(c.hc * s + c.h * cs, c.den, c.yden);
        return zeta + (zeta + c.h) * S;
    } else if (c.vt == 1) {
        const double S = c.hc * s + (c.h - c.hc) * cs;
        return S + zeta * (1.0 + rp_div_by(S, c.h, c.yh));
    }
    return zeta * (1.0 + s) + c.hc * s + (c.h - c.hc) * cs;
}

struct LevelPick {
    int ibot, itop;                // 1-based levels
    double z1, z2;                 // zcff(1), zcff(2)
};

// Level bracket of getInterp3D, ztype 1 (interpolation_module.f90:529-558).
__device__ __forceinline__ void rp_walk_rho(const RpGridDev& g, double zeta, double depth, double zpar,
                                            LevelPick& L) {
    const double h = -1.0 * depth;
    const ZCtx zc = rp_zctx(g.vtransform, g.hc, h);
    const int nz = g.N;
    double zl1 = depth, zl2 = 0.0;
    int i;
    for (i = 1; i <= nz; i++) {
        zl2 = rp_zlevel_c(zc, __ldg(g.sr + i - 1), __ldg(g.csr + i - 1), zeta);
        if (zl2 > zpar) break;
        zl1 = zl2;
    }
    if (i > nz) {
        L.ibot = nz; L.itop = nz; L.z1 = 0.5; L.z2 = 0.5;
    } else if (i == 1) {
        L.ibot = 1; L.itop = 1; L.z1 = 0.5; L.z2 = 0.5;
    } else {
        const double Z = (zpar - zl1) / (zl2 - zl1);
        L.ibot = i - 1; L.itop = i; L.z1 = 1.0 - Z; L.z2 = Z;
    }
}

// Level bracket of getInterp3D, ztype 2 (interpolation_module.f90:559-582),
// with the pins for z below level 1 / above level N+1.
__device__ __forceinline__ void rp_walk_w(const RpGridDev& g, double zeta, double depth, double zpar,
                                          LevelPick& L, uint32_t& fl) {
    const double h = -1.0 * depth;
    const ZCtx zc = rp_zctx(g.vtransform, g.hc, h);
    const int nz = g.N + 1;
    double zl1 = 0.0, zl2 = 0.0;
    int i;
    for (i = 1; i <= nz; i++) {
        zl2 = rp_zlevel_c(zc, __ldg(g.sw + i - 1), __ldg(g.csw + i - 1), zeta);
        if (zl2 > zpar) break;
        zl1 = zl2;
    }
    if (i > nz) {
        fl |= RP_FL_WTOP;
        L.ibot = nz; L.itop = nz; L.z1 = 0.5; L.z2 = 0.5;
    } else if (i == 1) {
        fl |= RP_FL_WBOT;
        L.ibot = 1; L.itop = 1; L.z1 = 0.5; L.z2 = 0.5;
    } else {
        const double Z = (zpar - zl1) / (zl2 - zl1);
        L.ibot = i - 1; L.itop = i; L.z1 = 1.0 - Z; L.z2 = Z;
    }
}

// zprof(ibot/itop) blend of one slot: zcff1*zprof(Ibot) + zcff2*zprof(Itop)
template <typename T>
__device__ __forceinline__ double rp_col_uv(const void* f, const UVCell& c, int nlev, const LevelPick& L,
                                            int slot) {
    double pb = 0.0, pt = 0.0;
    double vb[4], vt[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int64_t base = c.o[k] * nlev;
        vb[k] = c.use[k] ? rp_ld<T>(f, (base + L.ibot - 1) * RP_SLOTS + slot) : 0.0;
        vt[k] = c.use[k] ? rp_ld<T>(f, (base + L.itop - 1) * RP_SLOTS + slot) : 0.0;
    }
    pb = c.cff[0] * vb[0] + c.cff[1] * vb[1] + c.cff[2] * vb[2] + c.cff[3] * vb[3];
    pt = c.cff[0] * vt[0] + c.cff[1] * vt[1] + c.cff[2] * vt[2] + c.cff[3] * vt[3];
    return L.z1 * pb + L.z2 * pt;
}

template <typename T>
__device__ __forceinline__ double rp_col_rho(const void* f, const RhoCell& c, const double* cff,
                                             int nlev, const LevelPick& L, int slot) {
    const int64_t o[4] = {c.o00, c.o10, c.o11, c.o01};
    double vb[4], vt[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int64_t base = o[k] * nlev;
        vb[k] = rp_ld<T>(f, (base + L.ibot - 1) * RP_SLOTS + slot);
        vt[k] = rp_ld<T>(f, (base + L.itop - 1) * RP_SLOTS + slot);
    }
    const double pb = cff[0] * vb[0] + cff[1] * vb[1] + cff[2] * vb[2] + cff[3] * vb[3];
    const double pt = cff[0] * vt[0] + cff[1] * vt[1] + cff[2] * vt[2] + cff[3] * vt[3];
    return L.z1 * pb + L.z2 * pt;
}

// ----------------------------------------------------------- boundaries

// inside (interpolation_module.f90:269-420) for a 3-point polygon.
__device__ __forceinline__ bool rp_inside3(const double xb_[3], const double yb_[3], double xo, double yo) {
    double xb[4] = {xb_[0], xb_[1], xb_[2], xb_[0]};
    double yb[4] = {yb_[0], yb_[1], yb_[2], yb_[0]};
    int crossings = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (((xb[k + 1] - xo) * (xo - xb[k]) >= 0.0) && (xb[k] != xb[k + 1])) {
            const double dx1 = xo - xb[k];
            const double dx2 = xb[k + 1] - xo;
            const double dxy = dx2 * (yo - yb[k]) - dx1 * (yb[k + 1] - yo);
            int inc = 0;
            if ((xb[k] == xo) && (yb[k] == yo)) {
                return true;
            } else if (((dx1 == 0.0) && (yo >= yb[k])) || ((dx2 == 0.0) && (yo >= yb[k + 1]))) {
                inc = 1;
            } else if ((dx1 * dx2 > 0.0) && ((xb[k + 1] - xb[k]) * dxy >= 0.0)) {
                inc = 2;
            }
            if (xb[k + 1] > xb[k]) crossings += inc;
            else crossings -= inc;
        }
    }
    return crossings != 0;
}

// bounds (boundary_module.f90:43-143)
__device__ __forceinline__ void rp_bounds(const RpGridDev& g, double ip, double jp, bool& ingrid,
                                          bool& obound) {
    const double ecut = RP_F_0P1;
    const double fcut = 1.0 - ecut;
    ingrid = false;
    obound = false;
    const int I = rp_ifloor(ip), J = rp_ifloor(jp);
    const double X = ip - (double)I, Y = jp - (double)J;
    if ((I > 1) && (J > 1) && (I < g.nx - 1) && (J < g.ny - 1)) {
        const int64_t o = (int64_t)(J - 1) * g.nx + (I - 1);
        const double m11 = (double)__ldg(g.mrho + o);
        const double m21 = (double)__ldg(g.mrho + o + 1);
        const double m22 = (double)__ldg(g.mrho + o + g.nx + 1);
        const double m12 = (double)__ldg(g.mrho + o + g.nx);
        const int nm = (int)(m11 + m21 + m22 + m12);
        if (nm == 4) ingrid = true;
        if (nm == 3) {
            double tX[3] = {0, 0, 0}, tY[3] = {0, 0, 0};
            int n = 0;
            // (it,jt) = (1,1),(1,2),(2,1),(2,2)
            if (m11 == 1) { tX[n] = 0.0; tY[n] = 0.0; n++; }
            if (m12 == 1) { tX[n] = 0.0; tY[n] = 1.0; n++; }
            if (m21 == 1) { tX[n] = 1.0; tY[n] = 0.0; n++; }
            if (m22 == 1 && n < 3) { tX[n] = 1.0; tY[n] = 1.0; n++; }
            if (rp_inside3(tX, tY, X, Y)) ingrid = true;
        }
        if (nm == 2) {
            if (m11 == 1 && (X < ecut) && (Y < ecut)) ingrid = true;
            if (m21 == 1 && (X > fcut) && (Y < ecut)) ingrid = true;
            if (m22 == 1 && (X > fcut) && (Y > fcut)) ingrid = true;
            if (m12 == 1 && (X < ecut) && (Y > fcut)) ingrid = true;
        }
    } else {
        obound = true;
    }
}

// --------------------------------------------------------------- noise

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11)
__device__ __forceinline__ void rp_philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    }
}

// Natural log of a positive normal double: x = m 2^e, m in (sqrt(1/2),
// sqrt(2)], log m = 2 atanh(z), z = (m-1)/(m+1), by its Taylor series
// (11 terms past z; |z| <= 0.1716).  Plain IEEE operations only, so the
// host restatement produces the same bits.
#define RP_LN2_HI 0.6931471805599453
#define RP_LN2_LO 2.3190468138462996e-17
#define RP_SQRT2 1.4142135623730951
#define RP_TWOPI_HI 6.283185307179586
#define RP_TWOPI_LO 2.4492935982947064e-16

// The products and sums are written with the round-to-nearest intrinsics,
// which are never contracted into FMAs, so the noise is bit-identical in
// every compilation unit whatever its contraction setting.
#define RP_MUL(a, b) __dmul_rn((a), (b))
#define RP_ADD(a, b) __dadd_rn((a), (b))
#define RP_SUB(a, b) __dsub_rn((a), (b))

__device__ __forceinline__ double rp_log_pos(double x) {
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    int e = (int)((b >> 52) & 0x7ffull) - 1023;
    double m = __longlong_as_double((long long)((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull));
    if (m > RP_SQRT2) { m = m * 0.5; e = e + 1; }
    const double z = (m - 1.0) / (m + 1.0);
    const double z2 = RP_MUL(z, z);
    double p = 1.0 / 23.0;
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 21.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 19.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 17.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 15.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 13.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 11.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 9.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 7.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 5.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0 / 3.0);
    p = RP_ADD(RP_MUL(p, z2), 1.0);
    const double de = (double)e;
    return RP_ADD(RP_MUL(de, RP_LN2_HI), RP_ADD(RP_MUL(de, RP_LN2_LO), RP_MUL(RP_MUL(2.0, z), p)));
}

// cos(2 pi u) for u in [0,1]: exact reductions (1-u, 1/2-v, 1/4-v are exact
// by Sterbenz) to 2 pi v in [0, pi/4] for the cosine series or the sine
// series, Taylor series to x^20 / x^19.
__device__ __forceinline__ double rp_cos2pi(double u) {
    double v = (u > 0.5) ? 1.0 - u : u;
    double sign = 1.0;
    if (v > 0.25) { v = 0.5 - v; sign = -1.0; }
    double r;
    if (v <= 0.125) {
        const double x = RP_ADD(RP_MUL(v, RP_TWOPI_HI), RP_MUL(v, RP_TWOPI_LO));
        const double x2 = RP_MUL(x, x);
        double p = 1.0 / 2432902008176640000.0;                          // 1/20!
        p = RP_SUB(RP_MUL(p, x2), 1.0 / 6402373705728000.0);             // 1/18!
        p = RP_ADD(RP_MUL(p, x2), 1.0 / 20922789888000.0);               // 1/16!
        p = RP_SUB(RP_MUL(p, x2), 1.0 / 87178291200.0);                  // 1/14!
        p = RP_ADD(RP_MUL(p, x2), 1.0 / 479001600.0);                    // 1/12!
        p = RP_SUB(RP_MUL(p, x2), 1.0 / 3628800.0);                      // 1/10!
        p = RP_ADD(RP_MUL(p, x2), 1.0 / 40320.0);                        // 1/8!
        p = RP_SUB(RP_MUL(p, x2), 1.0 / 720.0);                          // 1/6!
        p = RP_ADD(RP_MUL(p, x2), 1.0 / 24.0);                           // 1/4!
        p = RP_SUB(RP_MUL(p, x2), 0.5);                                  // 1/2!
        r = RP_ADD(RP_MUL(p, x2), 1.0);
    } else {
        const double w = 0.25 - v;
        const double x = RP_ADD(RP_MUL(w, RP_TWOPI_HI), RP_MUL(w, RP_TWOPI_LO));
        const double x2 = RP_MUL(x, x);
        double p = 1.0 / 121645100408832000.0;                           // 1/19!
        p = RP_SUB(RP_MUL(p, x2), 1.0 / 355687428096000.0);              // 1/17!
        p = RP_ADD(RP_MUL(p, x2), 1.0 / 1307674368000.0);                // 1/15!
        p = RP_SUB(RP_MUL(p, x2), 1.0 / 6227020800.0);                   // 1/13!
        p = RP_ADD(RP_MUL(p, x2), 1.0 / 39916800.0);                     // 1/11!
        p = RP_SUB(RP_MUL(p, x2), 1.0 / 362880.0);                       // 1/9!
        p = RP_ADD(RP_MUL(p, x2), 1.0 / 5040.0);                         // 1/7!
        p = RP_SUB(RP_MUL(p, x2), 1.0 / 120.0);                          // 1/5!
        p = RP_ADD(RP_MUL(p, x2), 1.0 / 6.0);                            // 1/3!  (sign below)
        p = RP_MUL(p, x2);
        r = RP_SUB(x, RP_MUL(x, p));                                     // x (1 - x^2/3! + ...)
    }
    return sign * r;
}

// exp: x = k ln2 + r with |r| <= ln2/2 (ln2 split so that k * hi is
// exact), exp(r) by its Taylor series to r^13/13!, then 2^k in two factors;
// the oracle's orc_exp runs the same operations.
#define RP_LN2E_HI 0x1.62e42fee00000p-1    // ln2 truncated to 32 bits
#define RP_LN2E_LO 0x1.a39ef35793c76p-33   // ln2 - RP_LN2E_HI
#define RP_INV_LN2 1.4426950408889634

__device__ __forceinline__ double rp_pow2i(int m) {            // 2^m, -1022 <= m <= 1023
    return __longlong_as_double((long long)((unsigned long long)(m + 1023) << 52));
}

__device__ __forceinline__ double rp_exp(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return __longlong_as_double(0x7ff0000000000000ll);
    if (x < -745.1332191019412) return 0.0;
    const double k = rint(RP_MUL(x, RP_INV_LN2));
    const double r = RP_SUB(RP_SUB(x, RP_MUL(k, RP_LN2E_HI)), RP_MUL(k, RP_LN2E_LO));
    double p = 1.0 / 6227020800.0;                              // 1/13!
    p = RP_ADD(RP_MUL(p, r), 1.0 / 479001600.0);
    p = RP_ADD(RP_MUL(p, r), 1.0 / 39916800.0);
    p = RP_ADD(RP_MUL(p, r), 1.0 / 3628800.0);
    p = RP_ADD(RP_MUL(p, r), 1.0 / 362880.0);
    p = RP_ADD(RP_MUL(p, r), 1.0 / 40320.0);
    p = RP_ADD(RP_MUL(p, r), 1.0 / 5040.0);
    p = RP_ADD(RP_MUL(p, r), 1.0 / 720.0);
    p = RP_ADD(RP_MUL(p, r), 1.0 / 120.0);
    p = RP_ADD(RP_MUL(p, r), 1.0 / 24.0);
    p = RP_ADD(RP_MUL(p, r), 1.0 / 6.0);
    p = RP_ADD(RP_MUL(p, r), 0.5);
    p = RP_ADD(RP_MUL(p, r), 1.0);
    p = RP_ADD(RP_MUL(p, r), 1.0);
    const int ki = (int)k, k1 = ki / 2, k2 = ki - k1;
    return RP_MUL(RP_MUL(p, rp_pow2i(k1)), rp_pow2i(k2));
}

// log of any double: rp_log_pos for positive normals, 2^54 scaling for
// subnormals, and the special values
__device__ __forceinline__ double rp_log(double x) {
    if (x != x || x < 0.0) return __longlong_as_double(0x7ff8000000000000ll);
    if (x == 0.0) return __longlong_as_double((long long)0xfff0000000000000ull);
    if (x == __longlong_as_double(0x7ff0000000000000ll)) return x;
    if (x < 0x1p-1022)
        return RP_SUB(RP_SUB(rp_log_pos(RP_MUL(x, 0x1p54)), RP_MUL(54.0, RP_LN2_HI)), RP_MUL(54.0, RP_LN2_LO));
    return rp_log_pos(x);
}

