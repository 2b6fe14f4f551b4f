// rp_mixed.cuh -- the mixed-precision form of the particle step.
//
// Same algorithm as the FP64 form (rp_step.cuh), with
//   * positions in FP32 with Kahan-compensated accumulation (p - c),
//   * u, v, w, AKs stored in FP16 with a scale per (ring slot, level),
//     zeta in FP32; interpolation, RK4 and reflections in FP32,
//   * age in FP64,
//   * the PPPACK smoothing-spline fit and the random-displacement sub-steps
//     in FP64, with the secant search for the smoothing parameter started
//     from the particle's value of the previous step (one chol1d pass when
//     it still meets smooth()'s 1 % criterion).
// The 16-bit storage is FP16 (RP_FIELD_MIXED) or int16 fixed point
// (RP_FIELD_MIXED_I16, |v| / scale <= 32767 with scale = level max / 32767).
// Results differ from the exact form by rounding; the error is measured
// against the FP64 form on identical noise.
#pragma once

#include <cuda_fp16.h>

#include "rp_step.cuh"

constexpr float kHalfRange = 16384.0f;   // |stored value| <= 16384 after scaling

// ------------------------------------------------------------ cells (FP32)

struct MRho {
    int64_t o[4];
    float X, Y;
    float cb[4];
    float ci[4];
    bool wet4;
};

__device__ __forceinline__ int m_floor(float x) {
    const float f = floorf(x);
    if (!(f >= -1.0e9f)) return -1000000000;
    if (f > 1.0e9f) return 1000000000;
    return (int)f;
}

__device__ __forceinline__ void m_getcoeff(float X, float Y, const float m[4], float cff[4], uint32_t& fl) {
    float dist[4], W[4];
    dist[0] = sqrtf(X * X + Y * Y);
    dist[1] = sqrtf((1.f - X) * (1.f - X) + Y * Y);
    dist[2] = sqrtf((1.f - X) * (1.f - X) + (1.f - Y) * (1.f - Y));
    dist[3] = sqrtf(X * X + (1.f - Y) * (1.f - Y));
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (dist[k] == 0.f) {
            fl |= RP_FL_NODE;
            if (m[k] != 0.f) {
#pragma unroll
                for (int q = 0; q < 4; q++) cff[q] = (q == k) ? 1.f : 0.f;
                return;
            }
            W[k] = 0.f;
        } else {
            W[k] = m[k] / dist[k];
        }
    }
    const float WT = W[0] + W[1] + W[2] + W[3];
    const float r = (WT == 0.f) ? 0.f : 1.f / WT;
#pragma unroll
    for (int k = 0; k < 4; k++) cff[k] = W[k] * r;
}

__device__ __forceinline__ void m_rho_cell(const RpGridDev& g, float ip, float jp, MRho& c, uint32_t& fl) {
    const int I = m_floor(ip), J = m_floor(jp);
    c.X = ip - (float)I;
    c.Y = jp - (float)J;
    const int i0 = rp_clamp(I, 1, g.nx, fl), i1 = rp_clamp(I + 1, 1, g.nx, fl);
    const int j0 = rp_clamp(J, 1, g.ny, fl), j1 = rp_clamp(J + 1, 1, g.ny, fl);
    c.o[0] = (int64_t)(j0 - 1) * g.nx + (i0 - 1);
    c.o[1] = (int64_t)(j0 - 1) * g.nx + (i1 - 1);
    c.o[2] = (int64_t)(j1 - 1) * g.nx + (i1 - 1);
    c.o[3] = (int64_t)(j1 - 1) * g.nx + (i0 - 1);
    const float X = c.X, Y = c.Y;
    c.cb[0] = (1.f - X) * (1.f - Y);
    c.cb[1] = X * (1.f - Y);
    c.cb[2] = X * Y;
    c.cb[3] = (1.f - X) * Y;
    float m[4];
#pragma unroll
    for (int k = 0; k < 4; k++) m[k] = (float)__ldg(g.mrho + c.o[k]);
    c.wet4 = (m[0] + m[1] + m[2] + m[3]) >= 4.f;
    m_getcoeff(X, Y, m, c.ci, fl);
}

__device__ __forceinline__ float m_bil(const double* a, const MRho& c) {
    return c.cb[0] * (float)__ldg(a + c.o[0]) + c.cb[1] * (float)__ldg(a + c.o[1]) +
           c.cb[2] * (float)__ldg(a + c.o[2]) + c.cb[3] * (float)__ldg(a + c.o[3]);
}

__device__ __forceinline__ float m_zeta(const RpGridDev& g, const MRho& c, int slot) {
    const float* z = reinterpret_cast<const float*>(g.zeta);
    return c.ci[0] * __ldg(z + c.o[0] * RP_SLOTS + slot) + c.ci[1] * __ldg(z + c.o[1] * RP_SLOTS + slot) +
           c.ci[2] * __ldg(z + c.o[2] * RP_SLOTS + slot) + c.ci[3] * __ldg(z + c.o[3] * RP_SLOTS + slot);
}

struct MUV {
    int64_t o[4];
    float cff[4];
    bool use[4];
};

// u / v corner sets with the reference's edge rules (interpolation_module.f90:608-767)
__device__ __forceinline__ void m_uv_cell(const RpGridDev& g, float ip, float jp, bool is_u, MUV& c, uint32_t& fl) {
    float X, Y;
    int ci[4], cj[4];
    float m[4];
    if (is_u) {
        const int xi_u = g.nx - 1, eta_u = g.ny;
        const int Jn = m_floor(jp);
        Y = jp - (float)Jn;
        const float uvI = ip - 0.5f;
        const int In = m_floor(uvI);
        X = uvI - (float)In;
        const int j0 = rp_clamp(Jn, 1, eta_u, fl), j1 = rp_clamp(Jn + 1, 1, eta_u, fl);
        const int a = In >= xi_u ? xi_u : (In < 1 ? 1 : In);
        const int b = In >= xi_u ? xi_u : (In < 1 ? 1 : In + 1);
        ci[0] = a; ci[1] = b; ci[2] = b; ci[3] = a;
        cj[0] = j0; cj[1] = j0; cj[2] = j1; cj[3] = j1;
#pragma unroll
        for (int k = 0; k < 4; k++) c.o[k] = (int64_t)(cj[k] - 1) * xi_u + (ci[k] - 1);
#pragma unroll
        for (int k = 0; k < 4; k++) m[k] = (float)__ldg(g.mu + c.o[k]);
        if (In >= xi_u) { m[1] = 0.f; m[2] = 0.f; }
        else if (In < 1) { m[0] = 0.f; m[3] = 0.f; }
    } else {
        const int xi_v = g.nx, eta_v = g.ny - 1;
        int In = m_floor(ip);
        X = ip - (float)In;
        const float uvJ = jp - 0.5f;
        int Jn = m_floor(uvJ);
        if (Jn < 1) Jn = 1;
        if (Jn > eta_v) In = eta_v;   // interpolation_module.f90:696
        Y = uvJ - (float)Jn;
        const int i0 = rp_clamp(In, 1, xi_v, fl), i1 = rp_clamp(In + 1, 1, xi_v, fl);
        ci[0] = i0; ci[1] = i1; ci[2] = i1; ci[3] = i0;
        if (Jn >= eta_v) { cj[0] = cj[1] = cj[2] = cj[3] = eta_v; }
        else { cj[0] = Jn; cj[1] = Jn; cj[2] = Jn + 1; cj[3] = Jn + 1; }
#pragma unroll
        for (int k = 0; k < 4; k++) c.o[k] = (int64_t)(cj[k] - 1) * xi_v + (ci[k] - 1);
#pragma unroll
        for (int k = 0; k < 4; k++) m[k] = (float)__ldg(g.mv + c.o[k]);
        if (Jn >= eta_v) { m[2] = 0.f; m[3] = 0.f; }
    }
    c.cff[0] = (1.f - X) * (1.f - Y);
    c.cff[1] = X * (1.f - Y);
    c.cff[2] = X * Y;
    c.cff[3] = (1.f - X) * Y;
    const float nwater = m[0] + m[1] + m[2] + m[3];
#pragma unroll
    for (int k = 0; k < 4; k++) c.use[k] = true;
    if (nwater < 4.f && nwater > 0.f) {
#pragma unroll
        for (int k = 0; k < 4; k++) if (m[k] == 0.f) c.use[k] = false;
    } else if (nwater == 0.f) {
#pragma unroll
        for (int k = 0; k < 4; k++) { c.cff[k] = 0.f; c.use[k] = false; }
    }
}

// ------------------------------------------------------- levels (FP32)

struct MPick {
    int ibot, itop;
    float z1, z2;
};

__device__ __forceinline__ float m_zlev(int vt, float hc, float h, float den_r, float s, float cs, float zeta) {
    if (vt == 2) {
        const float S = (hc * s + h * cs) * den_r;
        return zeta + (zeta + h) * S;
    } else if (vt == 1) {
        const float S = hc * s + (h - hc) * cs;
        return S + zeta * (1.f + S / h);
    }
    return zeta * (1.f + s) + hc * s + (h - hc) * cs;
}

// first level k in 1..nz with z_k > zpar by bisection over the monotone
// levels, with the reference's boundary cases (rho: constant outside;
// w: pinned as in the FP64 form)
__device__ __forceinline__ void m_walk(const double* s, const double* cs, int nz, int vt, float hc, float zeta,
                                       float depth, float zpar, bool wlev, MPick& L, uint32_t& fl) {
    const float h = -depth;
    const float den_r = 1.f / (hc + h);
    auto zl = [&](int k) -> float { return m_zlev(vt, hc, h, den_r, (float)__ldg(s + k - 1), (float)__ldg(cs + k - 1), zeta); };
    int lo = 0, hi = nz + 1;            // z_lo <= zpar < z_hi (virtual ends)
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (zl(mid) > zpar) hi = mid; else lo = mid;
    }
    const int i = hi;                   // first level above zpar, nz+1 if none
    if (i > nz) {
        if (wlev) fl |= RP_FL_WTOP;
        L.ibot = nz; L.itop = nz; L.z1 = 0.5f; L.z2 = 0.5f;
    } else if (i == 1) {
        if (wlev) fl |= RP_FL_WBOT;
        L.ibot = 1; L.itop = 1; L.z1 = 0.5f; L.z2 = 0.5f;
    } else {
        const float za = zl(i - 1), zb = zl(i);
        const float Z = (zpar - za) / (zb - za);
        L.ibot = i - 1; L.itop = i; L.z1 = 1.f - Z; L.z2 = Z;
    }
}

// one stored 16-bit field value (before its level scale): FP16, or int16
// fixed point
__device__ __forceinline__ float m_h(const __half* f, int64_t idx) { return __half2float(__ldg(f + idx)); }
__device__ __forceinline__ float m_h(const int16_t* f, int64_t idx) { return (float)__ldg(f + idx); }

// zcff1*zprof(Ibot) + zcff2*zprof(Itop) of one slot of an FP16 field
template <typename E>
__device__ __forceinline__ float m_col(const void* fv, const float* qs, const int64_t o[4], const float cff[4],
                                       const bool use[4], int nlev, const MPick& L, int slot) {
    const E* f = reinterpret_cast<const E*>(fv);
    float pb = 0.f, pt = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int64_t base = o[k] * nlev;
        const float vb = use[k] ? m_h(f, (base + L.ibot - 1) * RP_SLOTS + slot) : 0.f;
        const float vt = use[k] ? m_h(f, (base + L.itop - 1) * RP_SLOTS + slot) : 0.f;
        pb += cff[k] * vb;
        pt += cff[k] * vt;
    }
    pb *= __ldg(qs + slot * nlev + L.ibot - 1);
    pt *= __ldg(qs + slot * nlev + L.itop - 1);
    return L.z1 * pb + L.z2 * pt;
}

struct MPol {
    float d1, dns, b, r12, r01, r02;
    int ns;
};

__device__ __forceinline__ MPol m_pol(const RpPolint& P) {
    MPol m;
    m.d1 = (float)P.d1; m.dns = (float)P.dns; m.b = (float)P.b;
    m.r12 = (float)P.re12; m.r01 = (float)P.re01; m.r02 = (float)P.re02;
    m.ns = P.ns;
    return m;
}

__device__ __forceinline__ float m_polintd(const MPol& P, float y0, float y1, float y2) {
    const float q12 = (y2 - y1) * P.r12;
    const float q01 = (y1 - y0) * P.r01;
    const float c = (P.d1 * q12 - P.d1 * q01) * P.r02;
    const float a = (P.ns == 2) ? q12 : q01;
    const float yns = (P.ns == 0) ? y0 : ((P.ns == 1) ? y1 : y2);
    return yns + P.dns * a + P.b * c;
}

struct MStage {
    MRho rc;
    float tdepth, zb, zc, zf, zeta;
};

// find_currents (advection_module.f90:129-350) in FP32 on FP16 fields
// depth and the three zeta values at the stage's cell S.rc
__device__ __forceinline__ void m_stage_2d(const MPol& P, const RpGridDev& g, MStage& S) {
    S.tdepth = -m_bil(g.h, S.rc);
    S.zb = m_zeta(g, S.rc, g.sb);
    S.zc = m_zeta(g, S.rc, g.sc);
    S.zf = m_zeta(g, S.rc, g.sf);
    S.zeta = m_polintd(P, S.zb, S.zc, S.zf);
}

// with cell_ready the caller has already filled S.rc for (X, Y); E is the
// 16-bit storage type of u, v, w (and AKs)
template <typename E>
__device__ __forceinline__ void m_find_currents(const RpStepArgs& A, const MPol& P, const RpGridDev& g, float X,
                                                float Y, float& Z, float& U, float& V, float& Wv, MStage& S,
                                                bool cell_ready, uint32_t& fl) {
    if (!cell_ready) m_rho_cell(g, X, Y, S.rc, fl);
    m_stage_2d(P, g, S);
    if (Z < S.tdepth) Z = S.tdepth + 0.001f;
    if (Z > S.zeta) Z = S.zeta - 0.001f;
    MPick Lr, Lw;
    const float hc = (float)g.hc;
    m_walk(g.sr, g.csr, g.N, g.vtransform, hc, S.zeta, S.tdepth, Z, false, Lr, fl);
    m_walk(g.sw, g.csw, g.N + 1, g.vtransform, hc, S.zeta, S.tdepth, Z, true, Lw, fl);
    const int N = g.N;
    MUV cu, cv;
    m_uv_cell(g, X, Y, true, cu, fl);
    m_uv_cell(g, X, Y, false, cv, fl);
    const float Ub = m_col<E>(g.u, g.qs_u, cu.o, cu.cff, cu.use, N, Lr, g.sb);
    const float Uc = m_col<E>(g.u, g.qs_u, cu.o, cu.cff, cu.use, N, Lr, g.sc);
    const float Vb = m_col<E>(g.v, g.qs_v, cv.o, cv.cff, cv.use, N, Lr, g.sb);
    const float Vc = m_col<E>(g.v, g.qs_v, cv.o, cv.cff, cv.use, N, Lr, g.sc);
    const bool all[4] = {true, true, true, true};
    const float* cw = S.rc.wet4 ? S.rc.cb : S.rc.ci;
    const float Wb = m_col<E>(g.w, g.qs_w, S.rc.o, cw, all, N + 1, Lw, g.sb);
    const float Wc = m_col<E>(g.w, g.qs_w, S.rc.o, cw, all, N + 1, Lw, g.sc);
    if (A.ets == 1) {
        U = m_polintd(P, Ub, Ub, Uc);
        V = m_polintd(P, Vb, Vb, Vc);
        Wv = m_polintd(P, Wb, Wb, Wc);
    } else {
        const float Uf = m_col<E>(g.u, g.qs_u, cu.o, cu.cff, cu.use, N, Lr, g.sf);
        const float Vf = m_col<E>(g.v, g.qs_v, cv.o, cv.cff, cv.use, N, Lr, g.sf);
        const float Wf = m_col<E>(g.w, g.qs_w, S.rc.o, cw, all, N + 1, Lw, g.sf);
        U = m_polintd(P, Ub, Uc, Uf);
        V = m_polintd(P, Vb, Vc, Vf);
        Wv = m_polintd(P, Wb, Wc, Wf);
    }
}

// --------------------------------------------- spline with a warm start
//
// The fit of VTurb (ver_turb_module.f90:126-189: linint resampling to np
// points, smooth with dy = serr) on exactly uniform breaks
// x_i = z_1 + (i-1) h.  On uniform breaks every band of setupq
// (pppack.f90:4726-4822) is constant: with r = serr/h, Q'D^2Q has the
// stencil (r^2, -4r^2, 6r^2, -4r^2, r^2) and R has (h, 4h, h), so the matrix
// of chol1d (pppack.f90:1428-1566) is the pentadiagonal
//   D = 6(1-p) 6r^2 + 4ph,  E = 6(1-p)(-4r^2) + ph,  F = 6(1-p) r^2
// (F = 0 on the last two rows).  The resampled values y_i are produced on
// the fly from the column's linear pieces (Q'y is never stored; y is kept
// once, by the first pass, for ppvalu), and the qu = Q u pass with its sum
// of squares runs inside back substitution.  Per chol1d pass the workspace
// traffic is three arrays written forward and read backward plus u written
// backward.

constexpr int kMixedArrays = 7;

template <int NPMAX>
struct MSpline {
    double* base;                  // kMixedArrays (NPMAX+1) doubles
    __device__ __forceinline__ double& s1(int i) const { return base[i]; }                  // ratio1(i)
    __device__ __forceinline__ double& s2(int i) const { return base[(NPMAX + 1) + i]; }    // ratio2(i)
    __device__ __forceinline__ double& u(int i) const { return base[2 * (NPMAX + 1) + i]; } // u(i)/v(i,1), then u(i)
    __device__ __forceinline__ double& y(int i) const { return base[3 * (NPMAX + 1) + i]; }  // resampled data y(i)
    __device__ __forceinline__ double& cz(int k) const { return base[4 * (NPMAX + 1) + k]; } // column z(k)
    __device__ __forceinline__ double& cm(int k) const { return base[5 * (NPMAX + 1) + k]; } // slope on [z(k), z(k+1)]
    __device__ __forceinline__ double& cb(int k) const { return base[6 * (NPMAX + 1) + k]; } // intercept
};

struct MFit {
    int np, sw;
    double z1, h, rh;              // first break, spacing, 1/h
    double serr, dy2;
};

// linint of the column at ascending points: the current piece j (slope,
// intercept and upper end) is held in registers and advanced as needed
template <int NPMAX>
struct MWalk {
    int j;
    double zn, m, b;               // cz(j+1), cm(j), cb(j)
    __device__ __forceinline__ void init(const MSpline<NPMAX>& w) {
        j = 1;
        zn = w.cz(2);
        m = w.cm(1);
        b = w.cb(1);
    }
    __device__ __forceinline__ double at(const MSpline<NPMAX>& w, int sw, double x) {
        while (j < sw - 1 && zn <= x) {
            j++;
            zn = w.cz(j + 1);
            m = w.cm(j);
            b = w.cb(j);
        }
        return m * x + b;
    }
};

// One chol1d pass at p: factorise, solve for u, form qu = Q u; returns
// sum_i qu(i)^2 dy^2 and, on request, utru = sum v4 (u(i-1)(u(i-1)+u(i)) + u(i)^2).
// With store_y the resampled values y(i) are also kept (for ppvalu).
template <int NPMAX>
__device__ double m_chol1d(const MSpline<NPMAX>& w, const MFit& f, double p, double* utru_out, bool store_y) {
    const int np = f.np;
    const double r = f.serr * f.rh;
    const double r2 = r * r;
    const double six1mp = 6.0 * (1.0 - p);
    const double D = six1mp * (6.0 * r2) + 4.0 * p * f.h;
    const double E = six1mp * (-4.0 * r2) + p * f.h;
    const double F = six1mp * r2;
    // Q'y on the fly: qty(i) = (y(i+1) - 2 y(i) + y(i-1)) / h
    MWalk<NPMAX> wk;
    wk.init(w);
    double ym = wk.at(w, f.sw, f.z1);
    double y0 = wk.at(w, f.sw, f.z1 + f.h);
    double yp = wk.at(w, f.sw, f.z1 + 2.0 * f.h);
    if (store_y) {
        w.y(1) = ym;
        w.y(2) = y0;
        w.y(3) = yp;
    }
    double a1 = D, a2 = E, b1 = D;
    double uprev = 0.0, ucur = (yp - 2.0 * y0 + ym) * f.rh, r2prev = 0.0;
#pragma unroll 2
    for (int i = 2; i <= np - 2; i++) {
        const double Fi = (i <= np - 3) ? F : 0.0;
        const double inv = 1.0 / a1;                 // one division per row
        const double ratio1 = a2 * inv;
        b1 = b1 - ratio1 * a2;
        const double c2 = E - ratio1 * Fi;
        const double ratio2 = Fi * inv;
        const double c1 = D - ratio2 * Fi;
        w.s1(i) = ratio1;
        w.s2(i) = ratio2;
        w.u(i) = ucur * inv;
        ym = y0;
        y0 = yp;
        yp = wk.at(w, f.sw, f.z1 + (double)(i + 1) * f.h);
        if (store_y) w.y(i + 2) = yp;
        const double qn = (yp - 2.0 * y0 + ym) * f.rh;     // qty(i+1)
        const double unext = qn - ratio1 * ucur - r2prev * uprev;
        uprev = ucur;
        ucur = unext;
        r2prev = ratio2;
        a1 = b1;
        a2 = c2;
        b1 = c1;
    }
    // back substitution, descending, with qu and its sum of squares:
    // raw(k) = (u(k) - u(k-1))/h for 2 <= k <= np, raw(1) = raw(np+1) = 0,
    // qu(k) = raw(k+1) - raw(k)
    const double dy2 = f.dy2;
    double up1 = 0.0;                                // u(np)
    double up2 = 0.0;                                // u(np+1), unused
    double rawp = 0.0;                               // raw(np+1)
    double sum = 0.0, utru = 0.0;
    w.u(np) = 0.0;
    {
        const double ui = ucur / a1;                 // u(np-1)
        w.u(np - 1) = ui;
        const double raw = (up1 - ui) * f.rh;        // raw(np)
        const double fin = rawp - raw;               // qu(np)
        sum = sum + fin * fin * dy2;
        utru = utru + f.h * (ui * (ui + up1) + up1 * up1);
        rawp = raw;
        up2 = up1;
        up1 = ui;
    }
#pragma unroll 2
    for (int i = np - 2; i >= 2; i--) {
        const double ui = w.u(i) - up1 * w.s1(i) - up2 * w.s2(i);
        w.u(i) = ui;
        const double raw = (up1 - ui) * f.rh;        // raw(i+1)
        const double fin = rawp - raw;               // qu(i+1)
        sum = sum + fin * fin * dy2;
        utru = utru + f.h * (ui * (ui + up1) + up1 * up1);
        rawp = raw;
        up2 = up1;
        up1 = ui;
    }
    {
        const double raw = up1 * f.rh;               // raw(2), u(1) = 0
        const double fin2 = rawp - raw;              // qu(2)
        sum = sum + fin2 * fin2 * dy2 + raw * raw * dy2;   // qu(1) = raw(2)
        utru = utru + f.h * (up1 * up1);
    }
    w.u(1) = 0.0;
    if (utru_out) *utru_out = utru;
    return sum;
}

// SF(q) = 36 sum qu^2 dy^2 / (1+q)^2 of one chol1d pass at p = q/(1+q)
template <int NPMAX>
__device__ __forceinline__ double m_sf(const MSpline<NPMAX>& w, const MFit& f, double q, bool store_y = false) {
    return 36.0 * m_chol1d(w, f, q / (1.0 + q), nullptr, store_y) / ((1.0 + q) * (1.0 + q));
}

// smooth() (pppack.f90:5108-5317): the secant search for q = p/(1-p) on
// 1/sqrt(SF) until |SF - s| <= 0.01 s.  Warm start: the particle's q of its
// previous step (one pass when it still meets the criterion) and the slope
// g of 1/sqrt(SF) in q found there, which gives a Newton step when it does
// not; then secant steps.  Falls back to the reference's cold start (p = 0,
// utru) when that does not converge.  q and g are returned in qstate and
// gstate (q = 0 for p = 0; g <= 0 when unknown).
template <int NPMAX>
__device__ double m_smooth(const MSpline<NPMAX>& w, const MFit& f, double s, int max_iter, double& qstate,
                           double& gstate, uint32_t& fl) {
    // the first pass of every path also stores y(i)
    if (s <= 0.0) {
        m_chol1d(w, f, 1.0, nullptr, true);
        return 1.0;
    }
    const double ooss = 1.0 / sqrt(s);
    double q = qstate;
    const bool warm = q > 0.0;
    if (warm) {
        double sfq = m_sf(w, f, q, true);
        if (fabs(sfq - s) <= 0.01 * s) return q / (1.0 + q);
        double prevq = q, prevsf = 1.0 / sqrt(sfq);
        const double qn = (gstate > 0.0) ? q + (ooss - prevsf) / gstate : 0.0;
        q = (qn > 0.0) ? qn : q * sqrt(sfq / s);
        for (int it = 0; it < 6 && q > 0.0; it++) {
            sfq = m_sf(w, f, q);
            const double oosf = 1.0 / sqrt(sfq);
            const double g = (oosf - prevsf) / (q - prevq);
            if (fabs(sfq - s) <= 0.01 * s) {
                qstate = q;
                gstate = g;
                return q / (1.0 + q);
            }
            const double change = (oosf - ooss) / g;
            prevq = q;
            q = q - change;
            prevsf = oosf;
        }
    }
    // cold start: the reference's sequence
    double utru = 0.0;
    double sfq = 36.0 * m_chol1d(w, f, 0.0, &utru, !warm);
    if (!(s < sfq)) {
        qstate = 0.0;
        gstate = 0.0;
        return 0.0;
    }
    double oosf = 1.0 / sqrt(sfq);
    q = -(oosf - ooss) * sfq / (6.0 * utru * oosf);
    double prevq = 0.0, prevsf = oosf;
    int it = 0;
    for (;;) {
        sfq = m_sf(w, f, q);
        oosf = 1.0 / sqrt(sfq);
        it++;
        const double g = (oosf - prevsf) / (q - prevq);
        if (fabs(sfq - s) <= 0.01 * s) {
            gstate = g;
            break;
        }
        if (it >= max_iter) {
            fl |= RP_FL_SPLINE;
            gstate = 0.0;
            break;
        }
        const double change = (oosf - ooss) / g;
        prevq = q;
        q = q - change;
        prevsf = oosf;
    }
    qstate = q;
    return q / (1.0 + q);
}

// ppvalu (pppack.f90:4246-4362) of the fit at x, the one piece it needs
// formed as smooth's epilogue forms a(:,1..4) (pppack.f90:5303-5316).
template <int NPMAX>
__device__ __forceinline__ double m_ppvalu(const MSpline<NPMAX>& w, const MFit& f, double p, double x,
                                           int jderiv) {
    const int np = f.np;
    // interv on uniform breaks: piece 1 below the first break, np-1 at or
    // above the last (also for a NaN x)
    const double t = floor((x - f.z1) * f.rh);
    const int i = (t >= 0.0 && t < (double)(np - 1)) ? (int)t + 1 : ((t >= (double)(np - 1)) ? np - 1 : 1);
    const double xi = f.z1 + (double)(i - 1) * f.h;
    const double um = (i >= 2) ? w.u(i - 1) : 0.0;
    const double u0 = w.u(i), u1 = w.u(i + 1);
    const double u2 = (i + 2 <= np) ? w.u(i + 2) : 0.0;
    const double raw0 = (i >= 2) ? (u0 - um) * f.rh : 0.0;          // raw(i)
    const double raw1 = (u1 - u0) * f.rh;                            // raw(i+1)
    const double raw2 = (i + 2 <= np) ? (u2 - u1) * f.rh : 0.0;      // raw(i+2)
    const double K1 = 6.0 * (1.0 - p) * f.dy2;
    const double a1i = w.y(i) - K1 * (raw1 - raw0);
    const double a1n = w.y(i + 1) - K1 * (raw2 - raw1);
    const double a3i = u0 * 6.0 * p;
    const double a3n = u1 * 6.0 * p;
    const double a4i = (a3n - a3i) * f.rh;
    const double a2i = (a1n - a1i) * f.rh - (a3i + a4i * (1.0 / 3.0) * f.h) * 0.5 * f.h;
    const double hx = x - xi;
    // Horner loop of ppvalu with k = 4: value = (value/fmmjdr)*h + coef(m)
    if (jderiv == 0) return ((a4i * (1.0 / 3.0) * hx + a3i) * 0.5 * hx + a2i) * hx + a1i;
    return (a4i * 0.5 * hx + a3i) * hx + a2i;
}

// VTurb (ver_turb_module.f90:31-329): column in FP32 from FP16 AKs, fit and
// random-displacement sub-steps in FP64
template <typename E, int NPMAX>
__device__ float m_vturb(const RpStepArgs& A, const MPol& P, const RpGridDev& g, const MStage& S, float Zpar,
                         uint32_t pid, double& qstate, double& gstate, uint32_t& fl, const MSpline<NPMAX>& w) {
    const int sw = g.N + 1;
    MFit f;
    f.np = (int)((double)sw * A.sub);
    f.sw = sw;
    f.serr = A.serr;
    f.dy2 = A.serr * A.serr;
    const double tdepth = (double)S.tdepth, zeta = (double)S.zeta;
    const float h = -S.tdepth;
    const float hc = (float)g.hc;
    const float den_r = 1.f / (hc + h);
    const float* cwt = S.rc.wet4 ? S.rc.cb : S.rc.ci;
    const E* aks = reinterpret_cast<const E*>(g.aks);
    const int slots[3] = {g.sb, g.sc, g.sf};
    double zprev = 0.0, kprev = 0.0;
    for (int k = 1; k <= sw; k++) {
        const float s = (float)__ldg(g.sw + k - 1), cs = (float)__ldg(g.csw + k - 1);
        double zk;
        if (k == sw) {
            zk = zeta;                                  // the top w level is zeta
        } else {
            const float zb = m_zlev(g.vtransform, hc, h, den_r, s, cs, S.zb);
            const float zcv = m_zlev(g.vtransform, hc, h, den_r, s, cs, S.zc);
            const float zf = m_zlev(g.vtransform, hc, h, den_r, s, cs, S.zf);
            zk = (double)m_polintd(P, zb, zcv, zf);
        }
        float K[3];
#pragma unroll
        for (int t = 0; t < 3; t++) {
            float a = 0.f;
#pragma unroll
            for (int q = 0; q < 4; q++) a += cwt[q] * m_h(aks, (S.rc.o[q] * sw + (k - 1)) * RP_SLOTS + slots[t]);
            K[t] = a * __ldg(g.qs_aks + slots[t] * sw + k - 1);
        }
        const double kk = (double)m_polintd(P, K[0], K[1], K[2]);
        w.cz(k) = zk;
        if (k >= 2) {
            const double m = (kk - kprev) / (zk - zprev);
            w.cm(k - 1) = m;
            w.cb(k - 1) = kprev - m * zprev;
        }
        zprev = zk;
        kprev = kk;
    }
    f.z1 = w.cz(1);
    f.h = (zeta - f.z1) / (double)(f.np - 1);
    f.rh = 1.0 / f.h;
    const double p = m_smooth(w, f, A.smth, A.spline_max_iter, qstate, gstate, fl);
    const double deltat = A.deltat;
    double ParZc = (double)Zpar;
    for (int i = 1; i <= A.loop; i++) {
        double Kprimec = 0.0;
        if (!(ParZc <= tdepth || ParZc >= zeta)) Kprimec = m_ppvalu(w, f, p, ParZc, 1);
        const double KprimeZc = Kprimec * deltat;
        const double Z3rdc = ParZc + 0.5 * KprimeZc;
        double KH3rdc;
        if (Z3rdc < tdepth || Z3rdc > zeta) {
            KH3rdc = A.aksback;
        } else {
            KH3rdc = m_ppvalu(w, f, p, Z3rdc, 0);
            if (KH3rdc < A.aksback) KH3rdc = A.aksback;
        }
        const double DEV = rp_normal(A, pid, (uint32_t)(1 + i));
        ParZc = ParZc + (KprimeZc + DEV * sqrt(2.0 * KH3rdc * deltat));
        if (ParZc <= tdepth) ParZc = tdepth + fabs(ParZc - tdepth);
        if (ParZc >= zeta) ParZc = zeta - fabs(ParZc - zeta);
    }
    return (float)(ParZc - (double)Zpar);
}

// Kahan-compensated FP32 accumulation: value = p - c
__device__ __forceinline__ void m_kahan_add(float& p, float& c, float d) {
    const float y = d - c;
    const float t = p + y;
    c = (t - p) - y;
    p = t;
}

// ----------------------------------------------------------- one particle

template <typename E, int NPMAX>
__device__ void m_update_one(const RpStepArgs& A, int64_t n, const MSpline<NPMAX>& w) {
    const RpParticlesDev& Pt = A.p;
    if (!rp_active(A, n)) return;
    Pt.age[n] = Pt.age[n] + (double)(float)A.idt;
    const MPol P = m_pol(A.pi);
    uint32_t fl = 0;
    int gid = Pt.gid[n];
    const RpGridDev& g = A.g[gid - 1];
    const uint32_t pid = Pt.pid[n];
    float x = Pt.x32[n], y = Pt.y32[n], z = Pt.z32[n];
    float cx = Pt.cx[n], cy = Pt.cy[n], cz = Pt.cz[n];
    const float Xpar = x, Ypar = y;
    float Zpar = z - cz;

    // pm, pn at the start position (ROMSPath.f90:727-728); the start cell
    // is formed again for stage 1 and for VTurb rather than kept live
    float pm, pn;
    {
        MRho c0;
        m_rho_cell(g, Xpar, Ypar, c0, fl);
        pm = m_bil(g.pm, c0);
        pn = m_bil(g.pn, c0);
    }

    float AdvectX = 0.f, AdvectY = 0.f, AdvectZ = 0.f;
    const float didt = (float)A.idt;
    const float half_dt = 0.5f * didt;
    if (A.scheme == 1) {                               // RKAdvect, advection_module.f90:20-125
        // stages 2-4 start from the (stage-1 clamped) start position plus the
        // previous stage's slope times idt/2; weights 1, 2, 2, 1
        float kx = 0.f, ky = 0.f, kz = 0.f;            // slope of the previous stage
#pragma unroll 1
        for (int st = 0; st < 4; st++) {
            float U, V, Wv;
            MStage Sx;
            float xs = Xpar, ys = Ypar, zs = Zpar;
            if (st > 0) {
                xs = Xpar + kx * half_dt;
                ys = Ypar + ky * half_dt;
                zs = Zpar + kz * half_dt;
            }
            m_find_currents<E>(A, P, g, xs, ys, zs, U, V, Wv, Sx, false, fl);
            if (st == 0) Zpar = zs;                    // Z is INOUT in find_currents
            kx = U * pm;
            ky = V * pn;
            kz = Wv;
            const float wgt = (st == 0 || st == 3) ? 1.f : 2.f;
            AdvectX += wgt * kx;
            AdvectY += wgt * ky;
            AdvectZ += wgt * kz;
        }
        AdvectX = didt * (AdvectX * (1.f / 6.f));
        AdvectY = didt * (AdvectY * (1.f / 6.f));
        AdvectZ = didt * (AdvectZ * (1.f / 6.f));
    }
    MStage S1;
    if (A.vturb_on) {
        m_rho_cell(g, Xpar, Ypar, S1.rc, fl);
        m_stage_2d(P, g, S1);
    }
    float TurbHx = 0.f, TurbHy = 0.f;
    if (A.hturb_on) {                                  // HTurb, hor_turb_module.f90:30-51
        const float sc = sqrtf(2.f * (float)A.khturb[gid - 1] * didt);
        TurbHx = (float)rp_normal(A, pid, 0u) * sc;
        TurbHy = (float)rp_normal(A, pid, 1u) * sc;
    }
    TurbHx *= pm;
    TurbHy *= pn;
    float TurbV = 0.f;
    if (A.vturb_on) {
        double q = Pt.qwarm[n], gs = Pt.gwarm[n];
        TurbV = m_vturb<E>(A, P, g, S1, Zpar, pid, q, gs, fl, w);
        Pt.qwarm[n] = q;
        Pt.gwarm[n] = gs;
    }
    // new position (Kahan), nest hand-off
    float nx = x, ncx = cx, ny = y, ncy = cy;
    m_kahan_add(nx, ncx, AdvectX + TurbHx);
    m_kahan_add(ny, ncy, AdvectY + TurbHy);
    float tx = nx, ty = ny, tcx = ncx, tcy = ncy;
    bool ingrid = false, obound = false;
    for (int i = 1; i <= A.ngrid; i++) {
        if (g.scl[i - 1][0] == 1.0 && g.scl[i - 1][1] == 1.0 && g.off[i - 1][0] == 0.0 &&
            g.off[i - 1][1] == 0.0) {
            tx = nx; ty = ny; tcx = ncx; tcy = ncy;    // identity map keeps the compensation
        } else {
            const double X = g.scl[i - 1][0] * ((double)nx - (double)ncx) + g.off[i - 1][0];
            const double Y = g.scl[i - 1][1] * ((double)ny - (double)ncy) + g.off[i - 1][1];
            tx = (float)X; ty = (float)Y;
            tcx = (float)((double)tx - X); tcy = (float)((double)ty - Y);
        }
        rp_bounds(A.g[i - 1], (double)tx, (double)ty, ingrid, obound);
        if (ingrid) { gid = i; break; }
    }
    const RpGridDev& gn = A.g[gid - 1];
    MRho rn;
    m_rho_cell(gn, tx, ty, rn, fl);
    const float tdepth = -m_bil(gn.h, rn);
    const float P_zeta = m_polintd(P, m_zeta(gn, rn, gn.sb), m_zeta(gn, rn, gn.sc), m_zeta(gn, rn, gn.sf));
    Pt.wd[n] = (double)(-tdepth + P_zeta);
    Pt.zeta[n] = (double)P_zeta;
    Pt.bath[n] = (double)(-tdepth);
    bool hbot = false, htop = false;
    float nz = z, ncz = cz;
    if (A.nsb == 0) {
        m_kahan_add(nz, ncz, AdvectZ + TurbV);
        const float zv = nz - ncz;
        if (zv < tdepth) { nz = tdepth + fabsf(zv - tdepth); ncz = 0.f; hbot = true; }
        if (nz - ncz > P_zeta) { nz = P_zeta - fabsf(nz - ncz - P_zeta); ncz = 0.f; htop = true; }
    } else if (A.nsb == 1) {
        nz = P_zeta - (float)A.vertdist; ncz = 0.f;
    } else {
        nz = tdepth + (float)A.vertdist; ncz = 0.f;
    }
    if (ingrid) {
        Pt.isin[n] = 1;
        Pt.x32[n] = tx; Pt.cx[n] = tcx;
        Pt.y32[n] = ty; Pt.cy[n] = tcy;
        Pt.z32[n] = nz; Pt.cz[n] = ncz;
        double st = 1.0;
        if (htop) st = RP_F_1P1;
        if (hbot) st = RP_F_1P2;
        Pt.status[n] = st;
        Pt.gid[n] = gid;
    } else if (obound) {
        Pt.isin[n] = 0;
        Pt.gid[n] = A.ngrid;
        Pt.status[n] = -8.0;
    } else {
        Pt.isin[n] = 1;
        Pt.status[n] = -9.0;
    }
    if (fl) Pt.flags[n] |= fl;
}
