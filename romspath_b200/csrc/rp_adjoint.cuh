// rp_adjoint.cuh -- the particle step written once over a generic scalar S
// (double, or Dual<4> carrying derivatives with respect to the step's
// starting x, y, z and the diffusivity multiplier kappa), for the adjoint
// pair rp_forward / rp_backward and the tangent-linear reference.
//
// The model is the FP64 step of update_particles (ROMSPath.f90:662-905):
// RK4 with the reference's interpolation (bilinear, inverse-distance,
// level walk, polintd in time), HTurb, VTurb with the smoothing-spline
// fit, hand-off and reflections.  Differences from the exact form that
// make it differentiable and replayable:
//   * kappa multiplies the diffusivity data (AKs) the fit is made to; at a
//     fixed smoothing parameter the fit is linear in the data, so this is
//     the same as scaling the fitted K(z);
//   * the fit uses exactly uniform breaks (as the mixed form) and a given
//     smoothing parameter p: rp_forward finds p by smooth()'s secant search
//     (pppack.f90:5108-5317) and records it per particle and step; replay,
//     tangent and adjoint runs reuse the recorded p (the search is a
//     discrete iteration, treated like the reflections: piecewise);
//   * the noise is frozen (Philox draws keyed on particle id and step).
// Branches (level brackets, reflections, land rejection, hand-off, pieces
// of the spline) are taken on values, so derivatives are those of the
// piece the trajectory is on.
#pragma once

#include "rp_step.cuh"

// ------------------------------------------------------------ dual numbers

template <int N>
struct Dual {
    double v;
    double d[N];
    __device__ __forceinline__ Dual() {}
    __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = 0.0;
    }
};

template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    const double ib = 1.0 / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
// mixed with double
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) {
    Dual<N> r = a;
    r.v = a.v + b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) { return b + a; }
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) {
    Dual<N> r = a;
    r.v = a.v - b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a - b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = -b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) {
    Dual<N> r;
    r.v = a.v / b;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] / b;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) {
    return Dual<N>(a) / b;
}

__device__ __forceinline__ double aval(double x) { return x; }
template <int N>
__device__ __forceinline__ double aval(const Dual<N>& x) { return x.v; }

__device__ __forceinline__ double asqrt(double x) { return sqrt(x); }
template <int N>
__device__ __forceinline__ Dual<N> asqrt(const Dual<N>& a) {
    Dual<N> r;
    r.v = sqrt(a.v);
    const double k = (r.v > 0.0) ? 0.5 / r.v : 0.0;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * k;
    return r;
}
template <class S>
__device__ __forceinline__ S aabs(const S& a) {
    return (aval(a) < 0.0) ? -a : a;
}

// ------------------------------------------------------------- stencils

template <class S>
struct ARho {
    int64_t o[4];
    S cb[4];
    S ci[4];
    bool wet4;
};

template <class S>
__device__ __forceinline__ void a_rho_cell(const RpGridDev& g, const S& ip, const S& jp, ARho<S>& c, uint32_t& fl) {
    const int I = rp_ifloor(aval(ip)), J = rp_ifloor(aval(jp));
    const S X = ip - (double)I, Y = jp - (double)J;
    const int i0 = rp_clamp(I, 1, g.nx, fl), i1 = rp_clamp(I + 1, 1, g.nx, fl);
    const int j0 = rp_clamp(J, 1, g.ny, fl), j1 = rp_clamp(J + 1, 1, g.ny, fl);
    c.o[0] = (int64_t)(j0 - 1) * g.nx + (i0 - 1);
    c.o[1] = (int64_t)(j0 - 1) * g.nx + (i1 - 1);
    c.o[2] = (int64_t)(j1 - 1) * g.nx + (i1 - 1);
    c.o[3] = (int64_t)(j1 - 1) * g.nx + (i0 - 1);
    c.cb[0] = (1.0 - X) * (1.0 - Y);
    c.cb[1] = X * (1.0 - Y);
    c.cb[2] = X * Y;
    c.cb[3] = (1.0 - X) * Y;
    double m[4];
#pragma unroll
    for (int k = 0; k < 4; k++) m[k] = (double)__ldg(g.mrho + c.o[k]);
    c.wet4 = !((m[0] + m[1] + m[2] + m[3]) < 4.0);
    // getcoeff (interpolation_module.f90:1230-1273) with the exact-node pin
    S dist[4], W[4];
    dist[0] = asqrt(X * X + Y * Y);
    dist[1] = asqrt((1.0 - X) * (1.0 - X) + Y * Y);
    dist[2] = asqrt((1.0 - X) * (1.0 - X) + (1.0 - Y) * (1.0 - Y));
    dist[3] = asqrt(X * X + (1.0 - Y) * (1.0 - Y));
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (aval(dist[k]) == 0.0) {
            fl |= RP_FL_NODE;
            if (m[k] != 0.0) {
#pragma unroll
                for (int q = 0; q < 4; q++) c.ci[q] = S((q == k) ? 1.0 : 0.0);
                return;
            }
            W[k] = S(0.0);
        } else {
            W[k] = m[k] / dist[k];
        }
    }
    const S WT = W[0] + W[1] + W[2] + W[3];
#pragma unroll
    for (int k = 0; k < 4; k++) c.ci[k] = (aval(WT) == 0.0) ? S(0.0) : W[k] / WT;
}

template <class S>
__device__ __forceinline__ S a_dot4(const double* a, const int64_t o[4], const S w[4]) {
    return w[0] * __ldg(a + o[0]) + w[1] * __ldg(a + o[1]) + w[2] * __ldg(a + o[2]) + w[3] * __ldg(a + o[3]);
}

// polintd (interpolation_module.f90:72-109) at the step's fixed nodes
template <class S>
__device__ __forceinline__ S a_polint(const RpPolint& P, const S& y0, const S& y1, const S& y2) {
    const S q12 = (y2 - y1) * P.re12;
    const S q01 = (y1 - y0) * P.re01;
    const S c = (P.d1 * q12 - P.d1 * q01) * P.re02;
    const S a = (P.ns == 2) ? q12 : q01;
    const S yns = (P.ns == 0) ? y0 : ((P.ns == 1) ? y1 : y2);
    return yns + P.dns * a + P.b * c;
}

template <class S>
struct AUV {
    int64_t o[4];
    S cff[4];
    bool use[4];
};

// u / v corner sets of getInterp3D (interpolation_module.f90:608-767)
template <class S>
__device__ __forceinline__ void a_uv_cell(const RpGridDev& g, const S& ip, const S& jp, bool is_u, AUV<S>& c,
                                          uint32_t& fl) {
    int ci[4], cj[4];
    double m[4];
    S X, Y;
    if (is_u) {
        const int xi_u = g.nx - 1, eta_u = g.ny;
        const int Jn = rp_ifloor(aval(jp));
        Y = jp - (double)Jn;
        const S uvI = ip - 0.5;
        const int In = rp_ifloor(aval(uvI));
        X = uvI - (double)In;
        const int j0 = rp_clamp(Jn, 1, eta_u, fl), j1 = rp_clamp(Jn + 1, 1, eta_u, fl);
        const int a = In >= xi_u ? xi_u : (In < 1 ? 1 : In);
        const int b = In >= xi_u ? xi_u : (In < 1 ? 1 : In + 1);
        ci[0] = a; ci[1] = b; ci[2] = b; ci[3] = a;
        cj[0] = j0; cj[1] = j0; cj[2] = j1; cj[3] = j1;
#pragma unroll
        for (int k = 0; k < 4; k++) c.o[k] = (int64_t)(cj[k] - 1) * xi_u + (ci[k] - 1);
#pragma unroll
        for (int k = 0; k < 4; k++) m[k] = (double)__ldg(g.mu + c.o[k]);
        if (In >= xi_u) { m[1] = 0.0; m[2] = 0.0; }
        else if (In < 1) { m[0] = 0.0; m[3] = 0.0; }
    } else {
        const int xi_v = g.nx, eta_v = g.ny - 1;
        int In = rp_ifloor(aval(ip));
        X = ip - (double)In;
        const S uvJ = jp - 0.5;
        int Jn = rp_ifloor(aval(uvJ));
        if (Jn < 1) Jn = 1;
        if (Jn > eta_v) In = eta_v;     // interpolation_module.f90:696
        Y = uvJ - (double)Jn;
        const int i0 = rp_clamp(In, 1, xi_v, fl), i1 = rp_clamp(In + 1, 1, xi_v, fl);
        ci[0] = i0; ci[1] = i1; ci[2] = i1; ci[3] = i0;
        if (Jn >= eta_v) { cj[0] = cj[1] = cj[2] = cj[3] = eta_v; }
        else { cj[0] = Jn; cj[1] = Jn; cj[2] = Jn + 1; cj[3] = Jn + 1; }
#pragma unroll
        for (int k = 0; k < 4; k++) c.o[k] = (int64_t)(cj[k] - 1) * xi_v + (ci[k] - 1);
#pragma unroll
        for (int k = 0; k < 4; k++) m[k] = (double)__ldg(g.mv + c.o[k]);
        if (Jn >= eta_v) { m[2] = 0.0; m[3] = 0.0; }
    }
    c.cff[0] = (1.0 - X) * (1.0 - Y);
    c.cff[1] = X * (1.0 - Y);
    c.cff[2] = X * Y;
    c.cff[3] = (1.0 - X) * Y;
    const double nwater = m[0] + m[1] + m[2] + m[3];
#pragma unroll
    for (int k = 0; k < 4; k++) c.use[k] = true;
    if (nwater < 4.0 && nwater > 0.0) {
#pragma unroll
        for (int k = 0; k < 4; k++) if (m[k] == 0.0) c.use[k] = false;
    } else if (nwater == 0.0) {
#pragma unroll
        for (int k = 0; k < 4; k++) { c.cff[k] = S(0.0); c.use[k] = false; }
    }
}

// getSlevel / getWlevel (grid_module.f90:513-598), h = -depth
template <class S>
__device__ __forceinline__ S a_zlev(int vt, double hc, double s, double cs, const S& zeta, const S& h) {
    if (vt == 2) {
        const S Sk = (hc * s + h * cs) / (hc + h);
        return zeta + (zeta + h) * Sk;
    } else if (vt == 1) {
        const S Sk = hc * s + (h - hc) * cs;
        return Sk + zeta * (1.0 + Sk / h);
    }
    return zeta * (1.0 + s) + hc * s + (h - hc) * cs;
}

template <class S>
struct APick {
    int ibot, itop;
    S z1, z2;
};

// level bracket of getInterp3D (interpolation_module.f90:529-582)
template <class S>
__device__ __forceinline__ void a_walk(const RpGridDev& g, bool wlev, const S& zeta, const S& depth, const S& zpar,
                                       APick<S>& L, uint32_t& fl) {
    const S h = -depth;
    const int nz = wlev ? g.N + 1 : g.N;
    const double* s = wlev ? g.sw : g.sr;
    const double* cs = wlev ? g.csw : g.csr;
    S zl1 = depth, zl2 = depth;
    int i;
    for (i = 1; i <= nz; i++) {
        zl2 = a_zlev(g.vtransform, g.hc, __ldg(s + i - 1), __ldg(cs + i - 1), zeta, h);
        if (aval(zl2) > aval(zpar)) break;
        zl1 = zl2;
    }
    if (i > nz) {
        if (wlev) fl |= RP_FL_WTOP;
        L.ibot = nz; L.itop = nz; L.z1 = S(0.5); L.z2 = S(0.5);
    } else if (i == 1) {
        if (wlev) fl |= RP_FL_WBOT;
        L.ibot = 1; L.itop = 1; L.z1 = S(0.5); L.z2 = S(0.5);
    } else {
        const S Z = (zpar - zl1) / (zl2 - zl1);
        L.ibot = i - 1; L.itop = i; L.z1 = 1.0 - Z; L.z2 = Z;
    }
}

// zcff1*zprof(Ibot) + zcff2*zprof(Itop) of one frame of a 3-D field
template <class S>
__device__ __forceinline__ S a_col(const double* f, const int64_t o[4], const S cff[4], const bool use[4], int nlev,
                                   const APick<S>& L) {
    S pb(0.0), pt(0.0);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (use[k]) {
            pb = pb + cff[k] * __ldg(f + o[k] * nlev + L.ibot - 1);
            pt = pt + cff[k] * __ldg(f + o[k] * nlev + L.itop - 1);
        }
    }
    return L.z1 * pb + L.z2 * pt;
}

template <class S>
struct AStage {
    ARho<S> rc;
    S tdepth, zb, zc, zf, zeta;
};

template <class S>
__device__ __forceinline__ void a_stage_2d(const RpStepArgs& A, const AdjFrames& F, int gi, const RpGridDev& g,
                                           AStage<S>& St) {
    St.tdepth = -a_dot4(g.h, St.rc.o, St.rc.cb);
    St.zb = a_dot4(F.f[gi][0][0], St.rc.o, St.rc.ci);
    St.zc = a_dot4(F.f[gi][0][1], St.rc.o, St.rc.ci);
    St.zf = a_dot4(F.f[gi][0][2], St.rc.o, St.rc.ci);
    St.zeta = a_polint(A.pi, St.zb, St.zc, St.zf);
}

// find_currents (advection_module.f90:129-350); Z is INOUT
template <class S>
__device__ __forceinline__ void a_find_currents(const RpStepArgs& A, const AdjFrames& F, int gi, const S& X, const S& Y,
                                                S& Z, S& U, S& V, S& W, AStage<S>& St, uint32_t& fl) {
    const RpGridDev& g = A.g[gi];
    a_rho_cell(g, X, Y, St.rc, fl);
    a_stage_2d(A, F, gi, g, St);
    if (aval(Z) < aval(St.tdepth)) Z = St.tdepth + RP_F_0P001;
    if (aval(Z) > aval(St.zeta)) Z = St.zeta - RP_F_0P001;
    APick<S> Lr, Lw;
    a_walk(g, false, St.zeta, St.tdepth, Z, Lr, fl);
    a_walk(g, true, St.zeta, St.tdepth, Z, Lw, fl);
    const int N = g.N;
    S val3[3];
    {
        AUV<S> cu;
        a_uv_cell(g, X, Y, true, cu, fl);
#pragma unroll
        for (int t = 0; t < 3; t++) val3[t] = a_col(F.f[gi][1][t], cu.o, cu.cff, cu.use, N, Lr);
        U = (A.ets == 1) ? a_polint(A.pi, val3[0], val3[0], val3[1]) : a_polint(A.pi, val3[0], val3[1], val3[2]);
    }
    {
        AUV<S> cv;
        a_uv_cell(g, X, Y, false, cv, fl);
#pragma unroll
        for (int t = 0; t < 3; t++) val3[t] = a_col(F.f[gi][2][t], cv.o, cv.cff, cv.use, N, Lr);
        V = (A.ets == 1) ? a_polint(A.pi, val3[0], val3[0], val3[1]) : a_polint(A.pi, val3[0], val3[1], val3[2]);
    }
    {
        const bool all[4] = {true, true, true, true};
        const S* cw = St.rc.wet4 ? St.rc.cb : St.rc.ci;
#pragma unroll
        for (int t = 0; t < 3; t++) val3[t] = a_col(F.f[gi][3][t], St.rc.o, cw, all, N + 1, Lw);
        W = (A.ets == 1) ? a_polint(A.pi, val3[0], val3[0], val3[1]) : a_polint(A.pi, val3[0], val3[1], val3[2]);
    }
}

// ------------------------------------------------------------- VTurb

// Workspace of one fit: column z(k), K(k) (k <= s_w) and the chol1d arrays
// (i <= np), NPMAX + 1 entries each.
template <class S, int NPMAX>
struct AFit {
    S* base;
    __device__ __forceinline__ S& zc(int k) const { return base[k]; }
    __device__ __forceinline__ S& kh(int k) const { return base[(NPMAX + 1) + k]; }
    __device__ __forceinline__ S& s1(int i) const { return base[2 * (NPMAX + 1) + i]; }
    __device__ __forceinline__ S& s2(int i) const { return base[3 * (NPMAX + 1) + i]; }
    __device__ __forceinline__ S& u(int i) const { return base[4 * (NPMAX + 1) + i]; }
    __device__ __forceinline__ S& y(int i) const { return base[5 * (NPMAX + 1) + i]; }
};
constexpr int kAdjArrays = 6;

// linint of the column at x (bisection on values; interpolation_module.f90:27-61)
template <class S, int NPMAX>
__device__ __forceinline__ S a_linint(const AFit<S, NPMAX>& w, int sw, const S& x) {
    int jlo = 1, jhi = sw;
    const double xv = aval(x);
    while (jhi - jlo > 1) {
        const int k = (jhi + jlo) / 2;
        if (aval(w.zc(k)) > xv) jhi = k; else jlo = k;
    }
    const S m = (w.kh(jlo) - w.kh(jhi)) / (w.zc(jlo) - w.zc(jhi));
    return m * x + (w.kh(jlo) - m * w.zc(jlo));
}

// chol1d (pppack.f90:1428-1566) on uniform breaks at a given p (the bands of
// the mixed form's m_chol1d); returns sum qu^2 dy^2.  Leaves u(1..np).
template <class S, int NPMAX>
__device__ S a_chol1d(const AFit<S, NPMAX>& w, int np, const S& hb, double p, double serr) {
    const S r = serr / hb;
    const S r2 = r * r;
    const double six1mp = 6.0 * (1.0 - p);
    const S D = six1mp * (6.0 * r2) + (4.0 * p) * hb;
    const S E = six1mp * (-4.0 * r2) + p * hb;
    const S F = six1mp * r2;
    const S rh = 1.0 / hb;
    S a1 = D, a2 = E, b1 = D;
    S uprev(0.0), ucur = (w.y(3) - 2.0 * w.y(2) + w.y(1)) * rh, r2prev(0.0);
    for (int i = 2; i <= np - 2; i++) {
        const S Fi = (i <= np - 3) ? F : S(0.0);
        const S ratio1 = a2 / a1;
        b1 = b1 - ratio1 * a2;
        const S c2 = E - ratio1 * Fi;
        const S ratio2 = Fi / a1;
        const S c1 = D - ratio2 * Fi;
        w.s1(i) = ratio1;
        w.s2(i) = ratio2;
        w.u(i) = ucur / a1;
        const S qn = (w.y(i + 2) - 2.0 * w.y(i + 1) + w.y(i)) * rh;      // qty(i+1)
        const S unext = qn - ratio1 * ucur - r2prev * uprev;
        uprev = ucur;
        ucur = unext;
        r2prev = ratio2;
        a1 = b1;
        a2 = c2;
        b1 = c1;
    }
    const double dy2 = serr * serr;
    w.u(np) = S(0.0);
    w.u(np - 1) = ucur / a1;
    for (int i = np - 2; i >= 2; i--) w.u(i) = w.u(i) - w.u(i + 1) * w.s1(i) - w.u(i + 2) * w.s2(i);
    w.u(1) = S(0.0);
    S prev(0.0), sum(0.0);
    for (int i = 2; i <= np; i++) {
        const S raw = (w.u(i) - w.u(i - 1)) * rh;
        const S fin = raw - prev;
        sum = sum + fin * fin * dy2;
        prev = raw;
    }
    sum = sum + prev * prev * dy2;
    return sum;
}

// smooth()'s secant search for p (pppack.f90:5108-5317, reference cold
// start) on uniform breaks; values only (double).
template <int NPMAX>
__device__ double a_find_p(const AFit<double, NPMAX>& w, int np, double hb, double serr, double s, int max_iter,
                           uint32_t& fl) {
    if (s <= 0.0) return 1.0;
    // utru needs u at p = 0
    double sfq = 36.0 * a_chol1d(w, np, hb, 0.0, serr);
    double utru = 0.0;
    for (int i = 2; i <= np; i++) {
        const double ul = w.u(i - 1), ui = w.u(i);
        utru = utru + hb * (ul * (ul + ui) + ui * ui);
    }
    if (!(s < sfq)) return 0.0;
    const double ooss = 1.0 / sqrt(s);
    double oosf = 1.0 / sqrt(sfq);
    double q = -(oosf - ooss) * sfq / (6.0 * utru * oosf);
    double prevq = 0.0, prevsf = oosf;
    for (int it = 1;; it++) {
        sfq = 36.0 * a_chol1d(w, np, hb, q / (1.0 + q), serr) / ((1.0 + q) * (1.0 + q));
        if (fabs(sfq - s) <= 0.01 * s) break;
        if (it >= max_iter) { fl |= RP_FL_SPLINE; break; }
        oosf = 1.0 / sqrt(sfq);
        const double change = (q - prevq) / (oosf - prevsf) * (oosf - ooss);
        prevq = q;
        q = q - change;
        prevsf = oosf;
    }
    return q / (1.0 + q);
}

// ppvalu (pppack.f90:4246-4362) of the fit, piece formed as smooth's
// epilogue forms a(:,1..4) (pppack.f90:5303-5316)
template <class S, int NPMAX>
__device__ __forceinline__ S a_ppvalu(const AFit<S, NPMAX>& w, int np, const S& z1, const S& hb, double p,
                                      double serr, const S& x, int jderiv) {
    const double t = floor(aval((x - z1) / hb));
    const int i = (t >= 0.0 && t < (double)(np - 1)) ? (int)t + 1 : ((t >= (double)(np - 1)) ? np - 1 : 1);
    const S rh = 1.0 / hb;
    const S xi = z1 + (double)(i - 1) * hb;
    const S um = (i >= 2) ? w.u(i - 1) : S(0.0);
    const S u0 = w.u(i), u1 = w.u(i + 1);
    const S u2 = (i + 2 <= np) ? w.u(i + 2) : S(0.0);
    const S raw0 = (i >= 2) ? (u0 - um) * rh : S(0.0);
    const S raw1 = (u1 - u0) * rh;
    const S raw2 = (i + 2 <= np) ? (u2 - u1) * rh : S(0.0);
    const double K1 = 6.0 * (1.0 - p) * serr * serr;
    const S a1i = w.y(i) - K1 * (raw1 - raw0);
    const S a1n = w.y(i + 1) - K1 * (raw2 - raw1);
    const S a3i = u0 * (6.0 * p);
    const S a3n = u1 * (6.0 * p);
    const S a4i = (a3n - a3i) * rh;
    const S a2i = (a1n - a1i) * rh - (a3i + a4i * (1.0 / 3.0) * hb) * 0.5 * hb;
    const S hx = x - xi;
    if (jderiv == 0) return ((a4i * (1.0 / 3.0) * hx + a3i) * 0.5 * hx + a2i) * hx + a1i;
    return (a4i * 0.5 * hx + a3i) * hx + a2i;
}

// VTurb (ver_turb_module.f90:31-329) with the diffusivity data scaled by
// kappa.  With find set, p is searched (values only) and returned in p;
// otherwise p is the given (recorded) value.
template <class S, int NPMAX>
__device__ S a_vturb(const RpStepArgs& A, const AdjFrames& F, int gi, const AStage<S>& St, const S& Zpar,
                     const S& kappa, uint32_t pid, bool find, double& p, uint32_t& fl, const AFit<S, NPMAX>& w) {
    const RpGridDev& g = A.g[gi];
    const int sw = g.N + 1;
    const int np = (int)((double)sw * A.sub);
    const S h = -St.tdepth;
    const S* cw = St.rc.wet4 ? St.rc.cb : St.rc.ci;
    for (int k = 1; k <= sw; k++) {
        const double s = __ldg(g.sw + k - 1), cs = __ldg(g.csw + k - 1);
        w.zc(k) = a_polint(A.pi, a_zlev(g.vtransform, g.hc, s, cs, St.zb, h),
                           a_zlev(g.vtransform, g.hc, s, cs, St.zc, h), a_zlev(g.vtransform, g.hc, s, cs, St.zf, h));
        S K3[3];
#pragma unroll
        for (int t = 0; t < 3; t++) {
            const double* a = F.f[gi][4][t];
            K3[t] = cw[0] * __ldg(a + St.rc.o[0] * sw + k - 1) + cw[1] * __ldg(a + St.rc.o[1] * sw + k - 1) +
                    cw[2] * __ldg(a + St.rc.o[2] * sw + k - 1) + cw[3] * __ldg(a + St.rc.o[3] * sw + k - 1);
        }
        w.kh(k) = kappa * a_polint(A.pi, K3[0], K3[1], K3[2]);
    }
    // resample to np uniform points (ver_turb_module.f90:126-136)
    const S z1 = w.zc(1);
    const S hb = (w.zc(sw) - z1) / (double)(np - 1);
    w.y(1) = w.kh(1);
    w.y(np) = w.kh(sw);
    for (int i = 2; i <= np - 1; i++) w.y(i) = a_linint(w, sw, z1 + (double)(i - 1) * hb);
    if (find) {
        if constexpr (sizeof(S) == sizeof(double)) {
            p = a_find_p(w, np, aval(hb), A.serr, A.smth, A.spline_max_iter, fl);
        }
    }
    a_chol1d(w, np, hb, p, A.serr);
    // random displacement sub-steps (ver_turb_module.f90:231-293)
    const double deltat = A.deltat;
    const S tdepth = St.tdepth, zeta = St.zeta;
    S ParZc = Zpar;
    for (int i = 1; i <= A.loop; i++) {
        S Kprimec(0.0);
        if (!(aval(ParZc) <= aval(tdepth) || aval(ParZc) >= aval(zeta)))
            Kprimec = a_ppvalu(w, np, z1, hb, p, A.serr, ParZc, 1);
        const S KprimeZc = Kprimec * deltat;
        const S Z3rdc = ParZc + 0.5 * KprimeZc;
        S KH3rdc;
        if (aval(Z3rdc) < aval(tdepth) || aval(Z3rdc) > aval(zeta)) {
            KH3rdc = S(A.aksback);
        } else {
            KH3rdc = a_ppvalu(w, np, z1, hb, p, A.serr, Z3rdc, 0);
            if (aval(KH3rdc) < A.aksback) KH3rdc = S(A.aksback);
        }
        const double DEV = rp_normal(A, pid, (uint32_t)(1 + i));
        ParZc = ParZc + (KprimeZc + DEV * asqrt(2.0 * KH3rdc * deltat));
        if (aval(ParZc) <= aval(tdepth)) ParZc = tdepth + aabs(ParZc - tdepth);
        if (aval(ParZc) >= aval(zeta)) ParZc = zeta - aabs(ParZc - zeta);
    }
    return ParZc - Zpar;
}

// ----------------------------------------------------------- one step

// The state a step carries besides (x, y, z).
struct AdjAux {
    double age, status;
    int gid;
    int8_t isin;
};

// One particle-step of the model (ROMSPath.f90:672-892) from (X, Y, Z) with
// auxiliary state `a`; updates X, Y, Z, a.  find: search p and return it;
// else use p.
template <class S, int NPMAX>
__device__ void a_step(const RpStepArgs& A, const AdjFrames& F, double dob, uint32_t pid, S& X, S& Y, S& Z, AdjAux& a,
                       const S& kappa, bool find, double& p, uint32_t& fl, const AFit<S, NPMAX>& w) {
    if (A.ix[2] <= dob || a.status == 9.0 || (A.oob && !a.isin)) return;      // ROMSPath.f90:672-690
    a.age = a.age + (double)(float)A.idt;
    int gid = a.gid;
    const int gi = gid - 1;
    const RpGridDev& g = A.g[gi];
    const S Xpar = X, Ypar = Y, z0 = Z;
    S Zpar = Z;
    S pm, pn;
    {
        ARho<S> c;
        a_rho_cell(g, Xpar, Ypar, c, fl);
        pm = a_dot4(g.pm, c.o, c.cb);
        pn = a_dot4(g.pn, c.o, c.cb);
    }
    S AdvectX(0.0), AdvectY(0.0), AdvectZ(0.0);
    AStage<S> S1;
    bool have_s1 = false;
    if (A.scheme == 1) {                                  // RKAdvect
        const double didt = (double)A.idt;
        S U, V, Wv, kx(0.0), ky(0.0), kz(0.0), ax(0.0), ay(0.0), az(0.0);
        for (int st = 0; st < 4; st++) {
            S xs = Xpar, ys = Ypar, zs = Zpar;
            if (st > 0) {
                xs = Xpar + kx * didt / 2.0;
                ys = Ypar + ky * didt / 2.0;
                zs = Zpar + kz * didt / 2.0;
            }
            AStage<S> Sx;
            a_find_currents(A, F, gi, xs, ys, zs, U, V, Wv, Sx, fl);
            if (st == 0) {
                Zpar = zs;                                // INOUT z of stage 1
                S1 = Sx;
                have_s1 = true;
            }
            kx = U * pm;
            ky = V * pn;
            kz = Wv;
            const double wgt = (st == 0 || st == 3) ? 1.0 : 2.0;
            ax = ax + wgt * kx;
            ay = ay + wgt * ky;
            az = az + wgt * kz;
        }
        AdvectX = didt * (ax / 6.0);
        AdvectY = didt * (ay / 6.0);
        AdvectZ = didt * (az / 6.0);
    }
    S TurbHx(0.0), TurbHy(0.0);
    if (A.hturb_on) {                                     // HTurb
        const double sc = sqrt(2.0 * A.khturb[gi] * (double)A.idt);
        TurbHx = rp_normal(A, pid, 0u) * sc * pm;
        TurbHy = rp_normal(A, pid, 1u) * sc * pn;
    }
    S TurbV(0.0);
    if (A.vturb_on) {
        if (!have_s1) {
            a_rho_cell(g, Xpar, Ypar, S1.rc, fl);
            a_stage_2d(A, F, gi, g, S1);
        }
        TurbV = a_vturb(A, F, gi, S1, Zpar, kappa, pid, find, p, fl, w);
    }
    // new position and hand-off (ROMSPath.f90:821-836)
    const S newX = X + AdvectX + TurbHx;
    const S newY = Y + AdvectY + TurbHy;
    S tX = newX, tY = newY;
    bool ingrid = false, obound = false;
    for (int i = 1; i <= A.ngrid; i++) {
        tX = g.scl[i - 1][0] * newX + g.off[i - 1][0];
        tY = g.scl[i - 1][1] * newY + g.off[i - 1][1];
        rp_bounds(A.g[i - 1], aval(tX), aval(tY), ingrid, obound);
        if (ingrid) { gid = i; break; }
    }
    const RpGridDev& gn = A.g[gid - 1];
    ARho<S> rn;
    a_rho_cell(gn, tX, tY, rn, fl);
    const S tdepth = -a_dot4(gn.h, rn.o, rn.cb);
    const S P_zeta = a_polint(A.pi, a_dot4(F.f[gid - 1][0][0], rn.o, rn.ci), a_dot4(F.f[gid - 1][0][1], rn.o, rn.ci),
                              a_dot4(F.f[gid - 1][0][2], rn.o, rn.ci));
    bool hbot = false, htop = false;
    S newZ;
    if (A.nsb == 0) {                                     // ROMSPath.f90:852-872
        newZ = z0 + AdvectZ + TurbV;
        if (aval(newZ) < aval(tdepth)) { newZ = tdepth + aabs(newZ - tdepth); hbot = true; }
        if (aval(newZ) > aval(P_zeta)) { newZ = P_zeta - aabs(newZ - P_zeta); htop = true; }
    } else if (A.nsb == 1) {
        newZ = P_zeta - A.vertdist;
    } else {
        newZ = tdepth + A.vertdist;
    }
    if (ingrid) {                                         // 874-892
        a.isin = 1;
        X = tX;
        Y = tY;
        Z = newZ;
        double st = 1.0;
        if (htop) st = RP_F_1P1;
        if (hbot) st = RP_F_1P2;
        a.status = st;
        a.gid = gid;
    } else if (obound) {
        a.isin = 0;
        a.gid = A.ngrid;
        a.status = -8.0;
    } else {
        a.isin = 1;
        a.status = -9.0;
    }
}
