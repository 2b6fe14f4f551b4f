// rp_step.cuh -- the per-particle step of update_particles
// (ROMSPath.f90:662-905) on the device: RK4 advection, HTurb, VTurb with
// the PPPACK smoothing spline, nest hand-off, vertical update and status.
#pragma once

#include "rp_device.cuh"

// --------------------------------------------------------------- noise

// Normal deviate `d` of particle `pid` at this step: the noise hook when
// set, else Philox4x32-10 at counter (pid, step, d/2) with Box-Muller's
// cosine branch (pdf_module.f90:26-40) on the uniforms (r+0.5)/2^32.
__device__ __forceinline__ double rp_normal(const RpStepArgs& A, uint32_t pid, uint32_t d) {
    if (A.hook) return A.hook[(int64_t)(pid - A.pid_base) * A.ndraw + d];
    uint32_t c[4] = {pid, (uint32_t)A.step_index, (uint32_t)(A.step_index >> 32), d >> 1};
    rp_philox(c, (uint32_t)A.seed, (uint32_t)(A.seed >> 32));
    const uint32_t a = (d & 1u) ? c[2] : c[0];
    const uint32_t b = (d & 1u) ? c[3] : c[1];
    const double u1 = ((double)a + 0.5) / 4294967296.0;
    const double u2 = ((double)b + 0.5) / 4294967296.0;
    return sqrt(-2.0 * rp_log_pos(u1)) * rp_cos2pi(u2);
}

// Uniform k (0..4) of behave's draws: the hook's entry d0 + 2 + k (d0 =
// 2 + idt/deltat, after the HTurb and VTurb normals and behave's two), else
// Philox4x32-10 at counter (pid, step, 0x40000000 + k/4), word k%4.
__device__ __forceinline__ double rp_uniform(const RpStepArgs& A, uint32_t pid, uint32_t d0, uint32_t k) {
    if (A.hook) return A.hook[(int64_t)(pid - A.pid_base) * A.ndraw + d0 + 2 + k];
    uint32_t c[4] = {pid, (uint32_t)A.step_index, (uint32_t)(A.step_index >> 32), 0x40000000u + (k >> 2)};
    rp_philox(c, (uint32_t)A.seed, (uint32_t)(A.seed >> 32));
    return ((double)c[k & 3u] + 0.5) / 4294967296.0;
}

// laplace (pdf_module.f90:42-55) of one uniform: sign(dev2, dev1) with
// dev1 = u - 0.5, dev2 = -log(1 - 2|dev1|) / sqrt(2)
__device__ __forceinline__ double rp_laplace_of(double u) {
    const double dev1 = RP_SUB(u, 0.5);
    const double dev2 = RP_MUL(-1.0, rp_log(RP_SUB(1.0, RP_MUL(2.0, fabs(dev1))))) / sqrt(2.0);
    const double mag = fabs(dev2);
    return (dev1 >= 0.0) ? mag : -mag;
}

// ------------------------------------------------------- find_currents

struct StageState {
    RhoCell rc;
    double tdepth, zb, zc, zf, zeta;
};

// The u, v, w gathers of find_currents under WETDRY: each slot's value
// with that slot's wetdry masks (interpolation_module.f90:628-671, 710-757,
// 917-939).  Out of line: the step without WETDRY keeps its registers.
template <typename T>
__device__ __noinline__ void rp_gather_wd(const RpStepArgs& A, const RpGridDev& g, double X, double Y,
                                          const LevelPick& Lr, const LevelPick& Lw, const RhoCell& rc, double& Uad,
                                          double& Vad, double& Wad, uint32_t& fl) {
    const int N = g.N;
    const int ns = (A.ets == 1) ? 2 : 3;
    const int sl[3] = {g.sb, g.sc, g.sf};
    double u[3], v[3], w[3];
    for (int q = 0; q < ns; q++) {
        UVCell c;
        rp_u_cell(g, X, Y, c, fl, g.wd_u, RP_SLOTS, sl[q]);
        u[q] = rp_col_uv<T>(g.u, c, N, Lr, sl[q]);
        rp_v_cell(g, X, Y, c, fl, g.wd_v, RP_SLOTS, sl[q]);
        v[q] = rp_col_uv<T>(g.v, c, N, Lr, sl[q]);
        double cw[4];
        rp_rho_wd_weights(g, rc, sl[q], cw, fl);
        w[q] = rp_col_rho<T>(g.w, rc, cw, N + 1, Lw, sl[q]);
    }
    if (A.ets == 1) {                                      // advection_module.f90:277-287
        Uad = rp_polintd(A.pi, u[0], u[0], u[1]);
        Vad = rp_polintd(A.pi, v[0], v[0], v[1]);
        Wad = rp_polintd(A.pi, w[0], w[0], w[1]);
    } else {
        Uad = rp_polintd(A.pi, u[0], u[1], u[2]);
        Vad = rp_polintd(A.pi, v[0], v[1], v[2]);
        Wad = rp_polintd(A.pi, w[0], w[1], w[2]);
    }
}

// find_currents (advection_module.f90:129-350); Z is INOUT.
template <typename T>
__device__ __forceinline__ void rp_find_currents(const RpStepArgs& A, const RpGridDev& g, double X, double Y,
                                                 double& Z, double& Uad, double& Vad, double& Wad,
                                                 StageState& S, uint32_t& fl) {
    rp_rho_cell(g, X, Y, S.rc, fl);
    S.tdepth = -1.0 * rp_bil(g.h, S.rc);
    S.zb = rp_zeta_at<T>(g, S.rc, g.sb);
    S.zc = rp_zeta_at<T>(g, S.rc, g.sc);
    S.zf = rp_zeta_at<T>(g, S.rc, g.sf);
    if (Z < S.tdepth) Z = S.tdepth + RP_F_0P001;
    S.zeta = rp_polintd(A.pi, S.zb, S.zc, S.zf);
    if (Z > S.zeta) Z = S.zeta - RP_F_0P001;

    LevelPick Lr, Lw;
    rp_walk_rho(g, S.zeta, S.tdepth, Z, Lr);
    rp_walk_w(g, S.zeta, S.tdepth, Z, Lw, fl);
    if (A.wetdry) {
        rp_gather_wd<T>(A, g, X, Y, Lr, Lw, S.rc, Uad, Vad, Wad, fl);
        return;
    }
    const int N = g.N;
    {
        UVCell cu;
        rp_u_cell(g, X, Y, cu, fl);
        const double Ub = rp_col_uv<T>(g.u, cu, N, Lr, g.sb);
        const double Uc = rp_col_uv<T>(g.u, cu, N, Lr, g.sc);
        if (A.ets == 1) {
            Uad = rp_polintd(A.pi, Ub, Ub, Uc);
        } else {
            const double Uf = rp_col_uv<T>(g.u, cu, N, Lr, g.sf);
            Uad = rp_polintd(A.pi, Ub, Uc, Uf);
        }
    }
    {
        UVCell cv;
        rp_v_cell(g, X, Y, cv, fl);
        const double Vb = rp_col_uv<T>(g.v, cv, N, Lr, g.sb);
        const double Vc = rp_col_uv<T>(g.v, cv, N, Lr, g.sc);
        if (A.ets == 1) {
            Vad = rp_polintd(A.pi, Vb, Vb, Vc);
        } else {
            const double Vf = rp_col_uv<T>(g.v, cv, N, Lr, g.sf);
            Vad = rp_polintd(A.pi, Vb, Vc, Vf);
        }
    }
    {
        const double* cw = S.rc.wet4 ? S.rc.cb : S.rc.ci;
        const double Wb = rp_col_rho<T>(g.w, S.rc, cw, N + 1, Lw, g.sb);
        const double Wc = rp_col_rho<T>(g.w, S.rc, cw, N + 1, Lw, g.sc);
        if (A.ets == 1) {
            Wad = rp_polintd(A.pi, Wb, Wb, Wc);
        } else {
            const double Wf = rp_col_rho<T>(g.w, S.rc, cw, N + 1, Lw, g.sf);
            Wad = rp_polintd(A.pi, Wb, Wc, Wf);
        }
    }
}

// ----------------------------------------------------------- spline

// Workspace of one particle's smoothing-spline fit: six arrays of
// (NPMAX+1) doubles with 1-based element i of array a at
// base[(a*(NPMAX+1) + i) * S].  S = 1 for a private array, S = 32 for a
// warp's lane-interleaved shared-memory block (bank-conflict free).
constexpr int kSplineArrays = 6;

template <int NPMAX, int S>
struct SplineView {
    double* base;
    __device__ __forceinline__ double& at(int a, int i) const { return base[(a * (NPMAX + 1) + i) * S]; }
    __device__ __forceinline__ double& fitz(int i) const { return at(0, i); }  // breaks fitz(1..np)
    __device__ __forceinline__ double& y(int i) const { return at(1, i); }     // fitKH(1..np)
    __device__ __forceinline__ double& qty(int i) const { return at(2, i); }   // Q'y
    __device__ __forceinline__ double& r1(int i) const { return at(3, i); }    // v(i,2) after factorisation
    __device__ __forceinline__ double& r2(int i) const { return at(4, i); }    // v(i,3) after factorisation
    __device__ __forceinline__ double& u(int i) const { return at(5, i); }     // u(i)/v(i,1), then u(i)
};

// The breaks fitz(1..np) as VTurb's resampling forms them
// (ver_turb_module.f90:126-136): fitz(1) = z1, fitz(k) = fitz(k-1) + dz for
// k = 2..np-1, fitz(np) = zend.  The chol1d passes re-form them by the same
// additions, ascending, instead of reading them back from the workspace.
struct RpBreaks {
    double z1, dz, zend;
};

// chol1d (pppack.f90:1428-1566) for p.  The setupq bands are rebuilt on the
// fly: with all data weights dy(i) = serr, v(i,1) = r(i-1),
// v(i,2) = -r(i) - r(i-1), v(i,3) = r(i) where r(k) = serr / v(k,4) and
// v(k,4) = fitz(k+1) - fitz(k), each formed by the same operation as in
// setupq.  Factorisation and forward substitution run in one ascending
// sweep that stores v(i,2), v(i,3) and u(i)/v(i,1); back substitution runs
// descending; then Q u and sum_i qu(i)^2 dy(i)^2 are formed ascending (the
// reference's summation order), with utru (pppack.f90:5219-5223) on request.
template <class W>
__device__ __forceinline__ double rp_chol1d(const W& w, int np, const RpBreaks& B, double p, double serr,
                                            double dy2, double* utru_out) {
    const double six1mp = 6.0 * (1.0 - p);
    const double twop = 2.0 * p;
    double acc = B.z1;                           // the running sum of the breaks
    auto brk = [&](int k) -> double {            // fitz(k), k = 2, 3, ... in turn
        acc = acc + B.dz;
        return (k == np) ? B.zend : acc;
    };
    const double f2 = brk(2), f3 = brk(3), f4 = brk(4);
    double v4a = f2 - B.z1;                      // v4(1)
    double v4b = f3 - f2;                        // v4(2)
    double v4c = f4 - f3;                        // v4(3)
    double fprev = f4;                           // fitz(i+2)
    const double r1_ = serr / v4a;               // r(1)
    double ri = serr / v4b;                      // r(i),   i = 2
    double rn = serr / v4c;                      // r(i+1)
    double v4n = v4c;                            // v4(i+1)
    double a1, a2, b1;
    {
        const double v2s2 = -ri - r1_;
        const double v2s3 = -rn - ri;
        const double v5_2 = r1_ * r1_ + v2s2 * v2s2 + ri * ri;
        a1 = six1mp * v5_2 + twop * (v4a + v4b);                         // V1(2)
        const double v6_2 = (2 <= np - 2) ? (v2s2 * ri + ri * v2s3) : 0.0;
        a2 = six1mp * v6_2 + p * v4b;                                     // V2(2)
        const double v5_3 = ri * ri + v2s3 * v2s3 + rn * rn;
        b1 = six1mp * v5_3 + twop * (v4b + v4c);                         // V1(3)
    }
    double uprev = 0.0, ucur = w.qty(2), r2prev = 0.0;
    w.u(1) = 0.0;
    // The sweeps are written without branches on the element index (values
    // past the ends are formed from clamped in-range loads and discarded by
    // the selects), so that unrolled iterations issue their independent
    // workspace loads together.
#pragma unroll 4
    for (int i = 2; i <= np - 2; i++) {
        // r(i+2), v4(i+2) (used while i+2 <= np-1)
        const bool has2 = (i + 2 <= np - 1);
        double v4nn = v4n;                        // past the end: discarded by the selects
        if (has2) {
            const double f = brk(i + 3);
            v4nn = f - fprev;
            fprev = f;
        }
        const double rnn = serr / v4nn;
        const double qn = w.qty(i + 1);
        const double V3i = six1mp * ((i <= np - 3) ? (ri * rn) : 0.0);
        const double ratio1 = a2 / a1;
        b1 = b1 - ratio1 * a2;
        const double v2sn = -rn - ri;             // v(i+1,2) of setupq
        const double v2snn = -rnn - rn;           // v(i+2,2)
        const double v6n = (i + 1 <= np - 2) ? (v2sn * rn + rn * v2snn) : 0.0;
        const double c2 = (six1mp * v6n + p * v4n) - ratio1 * V3i;
        const double ratio2 = V3i / a1;
        const double v5nn = rn * rn + v2snn * v2snn + rnn * rnn;
        const double c1 = has2 ? ((six1mp * v5nn + twop * (v4n + v4nn)) - ratio2 * V3i) : 0.0;
        w.r1(i) = ratio1;
        w.r2(i) = ratio2;
        w.u(i) = ucur / a1;                       // u(i)/v(i,1)
        const double unext = qn - ratio1 * ucur - r2prev * uprev;
        uprev = ucur;
        ucur = unext;
        r2prev = ratio2;
        a1 = b1;
        a2 = c2;
        b1 = c1;
        ri = rn;
        rn = rnn;
        v4n = v4nn;
    }
    // back substitution
    const double unm1 = ucur / a1;                // u(np-1)/v(np-1,1)
    w.u(np - 1) = unm1;
    w.u(np) = 0.0;
    double up2 = 0.0, up1 = unm1;
#pragma unroll 4
    for (int i = np - 2; i >= 2; i--) {
        const double qi = w.u(i), s1 = w.r1(i), s2 = w.r2(i);
        const double ui = qi - up1 * s1 - up2 * s2;
        w.u(i) = ui;
        up2 = up1;
        up1 = ui;
    }
    // qu = Q u and the weighted sum of squares, i = 1..np in order
    double prev = 0.0, sum = 0.0, utru = 0.0;
    double ulast = 0.0;                           // u(1)
    double flast = B.z1;
    acc = B.z1;
#pragma unroll 4
    for (int i = 2; i <= np; i++) {
        const double ui = w.u(i);
        const double fi = brk(i);
        const double v4i = fi - flast;
        const double raw = (ui - ulast) / v4i;
        const double fin = raw - prev;
        sum = sum + (fin * fin) * dy2;
        if (utru_out) utru = utru + v4i * (ulast * (ulast + ui) + ui * ui);
        prev = raw;
        ulast = ui;
        flast = fi;
    }
    const double finn = -prev;
    sum = sum + (finn * finn) * dy2;
    if (utru_out) *utru_out = utru;
    return sum;
}

// smooth (pppack.f90:5108-5317) on fitz/y already in w; dy(i) = serr for
// all i.  Returns p; w.u holds the final u; passes = chol1d passes made.
template <class W>
__device__ __forceinline__ double rp_smooth(const W& w, int np, const RpBreaks& B, double serr, double s,
                                            int max_iter, uint32_t& fl, int& passes) {
    const double dy2 = serr * serr;
    // setupq's Q'y (pppack.f90:4816-4822)
    {
        double prev = (w.y(2) - w.y(1)) / (w.fitz(2) - w.fitz(1));
        for (int i = 2; i <= np - 1; i++) {
            const double diff = (w.y(i + 1) - w.y(i)) / (w.fitz(i + 1) - w.fitz(i));
            w.qty(i) = diff - prev;
            prev = diff;
        }
    }
    double p, q, sfq;
    passes = 1;
    if (s <= 0.0) {
        p = 1.0;
        rp_chol1d(w, np, B, p, serr, dy2, nullptr);
    } else {
        p = 0.0;
        double utru = 0.0;
        sfq = 36.0 * rp_chol1d(w, np, B, p, serr, dy2, &utru);
        if (s < sfq) {
            const double ooss = 1.0 / sqrt(s);
            double oosf = 1.0 / sqrt(sfq);
            q = -(oosf - ooss) * sfq / (6.0 * utru * oosf);
            double prevq = 0.0, prevsf = oosf;
            int it = 0;
            for (;;) {
                const double sum = rp_chol1d(w, np, B, q / (1.0 + q), serr, dy2, nullptr);
                sfq = 36.0 * sum / ((1.0 + q) * (1.0 + q));
                it++;
                passes++;
                if (fabs(sfq - s) <= 0.01 * s) break;
                if (it >= max_iter) { fl |= RP_FL_SPLINE; break; }
                oosf = 1.0 / sqrt(sfq);
                const double change = (q - prevq) / (oosf - prevsf) * (oosf - ooss);
                prevq = q;
                q = q - change;
                prevsf = oosf;
            }
            p = q / (1.0 + q);
        }
    }
    return p;
}

// ppvalu (pppack.f90:4246-4362) of the smoothing spline at x, with the
// coefficients of the one piece it needs formed from u and y exactly as
// smooth's epilogue forms a(:,1..4) (pppack.f90:5303-5316).
template <class W>
__device__ __forceinline__ double rp_ppvalu(const W& w, int np, double p, double serr, double x, int jderiv) {
    // interv (pppack.f90:3363-3576) for strictly increasing breaks
    int i;
    if (!(x >= w.fitz(1))) {
        i = 1;
    } else {
        int lo = 1, hi = np;   // fitz(lo) <= x; answer in [lo, hi-1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (w.fitz(mid) <= x) lo = mid; else hi = mid;
        }
        i = lo;
    }
    const double dy2 = serr * serr;
    const double K1 = 6.0 * (1.0 - p) * dy2;
    auto v4 = [&](int k) -> double { return w.fitz(k + 1) - w.fitz(k); };
    auto raw = [&](int k) -> double { return (w.u(k) - w.u(k - 1)) / v4(k - 1); };  // k >= 2
    auto fin = [&](int k) -> double {
        if (k == 1) return raw(2) - 0.0;
        if (k == np) return -raw(np);
        return raw(k + 1) - raw(k);
    };
    const double a1i = w.y(i) - K1 * fin(i);
    const double a1n = w.y(i + 1) - K1 * fin(i + 1);
    const double a3i = w.u(i) * 6.0 * p;
    const double a3n = w.u(i + 1) * 6.0 * p;
    const double h4 = v4(i);
    const double a4i = (a3n - a3i) / h4;
    const double a2i = (a1n - a1i) / h4 - (a3i + a4i / 3.0 * h4) / 2.0 * h4;
    // Horner loop of ppvalu with k = 4: value = (value/fmmjdr)*h + coef(m)
    const double h = x - w.fitz(i);
    double value = 0.0;
    if (jderiv == 0) {
        value = (value / 4.0) * h + a4i;
        value = (value / 3.0) * h + a3i;
        value = (value / 2.0) * h + a2i;
        value = (value / 1.0) * h + a1i;
    } else {
        value = (value / 3.0) * h + a4i;
        value = (value / 2.0) * h + a3i;
        value = (value / 1.0) * h + a2i;
    }
    return value;
}

// ----------------------------------------------------------------- VTurb

// VTurb (ver_turb_module.f90:31-329).  The 2-D quantities at (Xpar, Ypar)
// are those of RK stage 1 (identical operations and operands).
template <typename T, class W>
__device__ double rp_vturb(const RpStepArgs& A, const RpGridDev& g, const StageState& S, double Zpar,
                           uint32_t pid, uint32_t& fl, const W& w) {
    const int sw = g.N + 1;
    const int np = (int)((double)sw * A.sub);
    const double tdepth = S.tdepth, zeta = S.zeta;
    const double h = -1.0 * tdepth;
    const ZCtx zx = rp_zctx(g.vtransform, g.hc, h);
    // column z(k), KH(k) (ver_turb_module.f90:100-124), held in the r1/r2
    // arrays until the fit overwrites them
    auto zc = [&](int k) -> double& { return w.r1(k); };
    auto kh = [&](int k) -> double& { return w.r2(k); };
    const double* cw = S.rc.wet4 ? S.rc.cb : S.rc.ci;
    const int64_t o[4] = {S.rc.o00, S.rc.o10, S.rc.o11, S.rc.o01};
    for (int k = 1; k <= sw; k++) {
        const double s = __ldg(g.sw + k - 1), cs = __ldg(g.csw + k - 1);
        double zb, zcv, zf;
        if (g.vtransform == 2) {
            const double Sk = rp_div_by(g.hc * s + h * cs, zx.den, zx.yden);
            zb = S.zb + (S.zb + h) * Sk;
            zcv = S.zc + (S.zc + h) * Sk;
            zf = S.zf + (S.zf + h) * Sk;
        } else {
            zb = rp_zlevel_c(zx, s, cs, S.zb);
            zcv = rp_zlevel_c(zx, s, cs, S.zc);
            zf = rp_zlevel_c(zx, s, cs, S.zf);
        }
        zc(k) = rp_polintd(A.pi, zb, zcv, zf);
        double ab[4], ac[4], af[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int64_t base = (o[q] * sw + (k - 1)) * RP_SLOTS;
            ab[q] = rp_ld<T>(g.aks, base + g.sb);
            ac[q] = rp_ld<T>(g.aks, base + g.sc);
            af[q] = rp_ld<T>(g.aks, base + g.sf);
        }
        const double Kb = cw[0] * ab[0] + cw[1] * ab[1] + cw[2] * ab[2] + cw[3] * ab[3];
        const double Kc = cw[0] * ac[0] + cw[1] * ac[1] + cw[2] * ac[2] + cw[3] * ac[3];
        const double Kf = cw[0] * af[0] + cw[1] * af[1] + cw[2] * af[2] + cw[3] * af[3];
        kh(k) = rp_polintd(A.pi, Kb, Kc, Kf);
    }
    // resample to np points (ver_turb_module.f90:126-136), linint per point
    const double dz = (zc(sw) - zc(1)) / (double)(np - 1);
    w.fitz(1) = zc(1);
    w.fitz(np) = zc(sw);
    w.y(1) = kh(1);
    w.y(np) = kh(sw);
    double x = zc(1);
    for (int i = 2; i <= np - 1; i++) {
        x = x + dz;
        w.fitz(i) = x;
        int jlo = 1, jhi = sw;
        for (;;) {
            const int k = (jhi + jlo) / 2;
            if (zc(k) > x) jhi = k; else jlo = k;
            if (jhi - jlo == 1) break;
        }
        const double m = (kh(jlo) - kh(jhi)) / (zc(jlo) - zc(jhi));
        const double b = kh(jlo) - m * zc(jlo);
        w.y(i) = m * x + b;
    }
    int passes;
    const RpBreaks B{zc(1), dz, zc(sw)};
    const double p = rp_smooth(w, np, B, A.serr, A.smth, A.spline_max_iter, fl, passes);
    if (A.spl) rp_count_fit(A.spl, passes);

    // random displacement sub-steps (ver_turb_module.f90:231-293)
    const double deltat = A.deltat;
    double ParZc = Zpar;
    for (int i = 1; i <= A.loop; i++) {
        double Kprimec = 0.0;
        if (ParZc <= tdepth || ParZc >= zeta) Kprimec = 0.0;
        else Kprimec = rp_ppvalu(w, np, p, A.serr, ParZc, 1);
        const double KprimeZc = Kprimec * deltat;
        const double Z3rdc = ParZc + 0.5 * KprimeZc;
        double KH3rdc;
        if (Z3rdc < tdepth || Z3rdc > zeta) {
            KH3rdc = A.aksback;
        } else {
            KH3rdc = rp_ppvalu(w, np, p, A.serr, Z3rdc, 0);
            if (KH3rdc < A.aksback) KH3rdc = A.aksback;
        }
        const double DEV = rp_normal(A, pid, (uint32_t)(1 + i));
        const double r = 1.0;
        const double dTz = KprimeZc + DEV * sqrt(2.0 / r * KH3rdc * deltat);
        ParZc = ParZc + dTz;
        if (ParZc <= tdepth) ParZc = tdepth + fabs(ParZc - tdepth);
        if (ParZc >= zeta) ParZc = zeta - fabs(ParZc - zeta);
    }
    return ParZc - Zpar;
}

// ------------------------------------------------------------ one particle

// Skip tests of update_particles (ROMSPath.f90:672-690).
__device__ __forceinline__ bool rp_active(const RpStepArgs& A, int64_t n) {
    const RpParticlesDev& P = A.p;
    if (A.ix[2] <= P.dob[n]) return false;
    if (P.status[n] == 9.0) return false;
    if (A.oob && !P.isin[n]) return false;
    return true;
}

// VTurb of one particle on its own (the first kernel of the split step):
// the stage-1 z clamp of find_currents (advection_module.f90:171-183) is
// applied first when RK4 runs, exactly as RKAdvect hands Zpar to VTurb.
template <typename T, class W>
__device__ void rp_vturb_one(const RpStepArgs& A, int64_t n, const W& w, double* turbv) {
    const RpParticlesDev& P = A.p;
    if (!rp_active(A, n)) return;
    uint32_t fl = 0;
    const int gid = P.gid[n];
    const RpGridDev& g = A.g[gid - 1];
    const double Xpar = P.x[n], Ypar = P.y[n];
    double Zpar = P.z[n];
    StageState S1;
    rp_rho_cell(g, Xpar, Ypar, S1.rc, fl);
    S1.tdepth = -1.0 * rp_bil(g.h, S1.rc);
    S1.zb = rp_zeta_at<T>(g, S1.rc, g.sb);
    S1.zc = rp_zeta_at<T>(g, S1.rc, g.sc);
    S1.zf = rp_zeta_at<T>(g, S1.rc, g.sf);
    S1.zeta = rp_polintd(A.pi, S1.zb, S1.zc, S1.zf);
    if (A.scheme == 1) {
        if (Zpar < S1.tdepth) Zpar = S1.tdepth + RP_F_0P001;
        if (Zpar > S1.zeta) Zpar = S1.zeta - RP_F_0P001;
    }
    turbv[n] = rp_vturb<T>(A, g, S1, Zpar, P.pid[n], fl, w);
    if (fl) P.flags[n] |= fl;
}

// getInterpStr (interpolation_module.f90:964-1174) of one slot on the u or
// v corner set: the same edge and dry-corner rules as u and v in getInterp3D.
template <typename T>
__device__ __forceinline__ double rp_str_at(const void* f, const UVCell& c, int slot) {
    double v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = c.use[k] ? rp_ld<T>(f, c.o[k] * RP_SLOTS + slot) : 0.0;
    return c.cff[0] * v[0] + c.cff[1] * v[1] + c.cff[2] * v[2] + c.cff[3] * v[3];
}

// getInterp3D of salt or temp, ztype 1 (interpolation_module.f90:529-558,
// 769-809): the rho corner set (bilinear, inverse distance with a dry
// corner) on the rho levels of the slot's own zeta.
// wcf: under WETDRY the slot's weights from its wetdry_mask_rho
// (rp_rho_wd_weights, formed once per cell by the caller), else null.
template <typename T>
__device__ __forceinline__ double rp_tracer_at(const RpGridDev& g, const void* f, const RhoCell& c, double zeta,
                                               double depth, double zpar, int slot, const double* wcf) {
    LevelPick L;
    rp_walk_rho(g, zeta, depth, zpar, L);
    return rp_col_rho<T>(f, c, wcf ? wcf : (c.wet4 ? c.cb : c.ci), g.N, L, slot);
}

// The diagnostics that close update_particles' particle loop
// (ROMSPath.f90:935-986), at the particle's new position and grid, with
// the step's tdepth: height above bottom and, where it reaches a new
// minimum, the bottom stress (WriteBottom); salinity and temperature and
// their running sums (SaltTempOn, SaltTempMean).  Out of line: the step's
// registers are not spent on it when the diagnostics are off.
template <typename T>
__device__ __noinline__ void rp_diag_one(const RpStepArgs& A, int64_t n, double tdepth, uint32_t& fl) {
    const RpParticlesDev& P = A.p;
    const RpGridDev& g = A.g[P.gid[n] - 1];
    const double X = P.x[n], Y = P.y[n], Z = P.z[n];
    if (A.diag & RP_DIAG_BOTTOM_D) {                       // 935-952
        const double btemp = -1.0 * tdepth + Z;
        const double hob0 = P.hob[n];
        const double hob = (btemp < hob0) ? btemp : hob0;
        P.hob[n] = hob;
        if (btemp == hob) {
            const int sl[3] = {g.sb, g.sc, g.sf};
            double su[3], sv[3];
            UVCell c;
            if (A.wetdry) {                                // each slot's wetdry_mask_u / _v
                for (int q = 0; q < 3; q++) {
                    rp_u_cell(g, X, Y, c, fl, g.wd_u, RP_SLOTS, sl[q]);
                    su[q] = rp_str_at<T>(g.bustr, c, sl[q]);
                    rp_v_cell(g, X, Y, c, fl, g.wd_v, RP_SLOTS, sl[q]);
                    sv[q] = rp_str_at<T>(g.bvstr, c, sl[q]);
                }
            } else {
                rp_u_cell(g, X, Y, c, fl);
                for (int q = 0; q < 3; q++) su[q] = rp_str_at<T>(g.bustr, c, sl[q]);
                rp_v_cell(g, X, Y, c, fl);
                for (int q = 0; q < 3; q++) sv[q] = rp_str_at<T>(g.bvstr, c, sl[q]);
            }
            P.bustr[n] = rp_polintd(A.pi, su[0], su[1], su[2]);
            P.bvstr[n] = rp_polintd(A.pi, sv[0], sv[1], sv[2]);
        }
    }
    if (A.diag & RP_DIAG_SALTTEMP_D) {                     // 962-986
        RhoCell c;
        rp_rho_cell(g, X, Y, c, fl);
        const double zb = rp_zeta_at<T>(g, c, g.sb);
        const double zc = rp_zeta_at<T>(g, c, g.sc);
        const double zf = rp_zeta_at<T>(g, c, g.sf);
        double wcf[3][4];                                  // WETDRY: each slot's weights, once
        if (A.wetdry) {
            rp_rho_wd_weights(g, c, g.sb, wcf[0], fl);
            rp_rho_wd_weights(g, c, g.sc, wcf[1], fl);
            rp_rho_wd_weights(g, c, g.sf, wcf[2], fl);
        }
        const double* wb = A.wetdry ? wcf[0] : nullptr;
        const double* wc = A.wetdry ? wcf[1] : nullptr;
        const double* wf = A.wetdry ? wcf[2] : nullptr;
        const double s = rp_polintd(A.pi, rp_tracer_at<T>(g, g.salt, c, zb, tdepth, Z, g.sb, wb),
                                    rp_tracer_at<T>(g, g.salt, c, zc, tdepth, Z, g.sc, wc),
                                    rp_tracer_at<T>(g, g.salt, c, zf, tdepth, Z, g.sf, wf));
        const double t = rp_polintd(A.pi, rp_tracer_at<T>(g, g.temp, c, zb, tdepth, Z, g.sb, wb),
                                    rp_tracer_at<T>(g, g.temp, c, zc, tdepth, Z, g.sc, wc),
                                    rp_tracer_at<T>(g, g.temp, c, zf, tdepth, Z, g.sf, wf));
        P.salt[n] = s;
        P.temp[n] = t;
        if (A.diag & RP_DIAG_MEAN_D) {
            P.mean_salt[n] = P.mean_salt[n] + s;
            P.mean_temp[n] = P.mean_temp[n] + t;
        }
    }
}

// behave's response to the four standard deviations at the particle
// (behavior_module.f90:285-375): 4 laplace, 2 normal and 1 uniform draws,
// the Fuchs swim / sink choice into par(:,pAcc/pVort/pbehaveW/pSSF);
// returns the vertical velocity wb (cm/s).  Real powers are pinned as
// x**2.0D0 = x*x, r**3.0D0 = (r*r)*r, x**0.5D0 = sqrt(x); exp and log are
// this project's own.  Shared by both forms of the step.
__device__ __forceinline__ double rp_behave_swim(const RpStepArgs& A, int64_t n, uint32_t pid, double stdaccturbu,
                                                 double stdvortturb, double stdaccwaveu, double stdaccwavev) {
    const RpBehaviorDev& b = A.beh;
    const double G = 980.0, RHOF = 1.026, MU = 0.010260, RHOP = 1.06;   // ROMSPath.h:15-19
    double wb;
    const uint32_t d0 = 2u + (uint32_t)A.loop;
    const double vortturbu = RP_MUL(stdvortturb, rp_laplace_of(rp_uniform(A, pid, d0, 0)));
    const double vortturbv = RP_MUL(stdvortturb, rp_laplace_of(rp_uniform(A, pid, d0, 1)));
    const double vorttot = sqrt(RP_ADD(RP_MUL(vortturbu, vortturbu), RP_MUL(vortturbv, vortturbv)));
    const double accturbu = RP_MUL(stdaccturbu, rp_laplace_of(rp_uniform(A, pid, d0, 2)));
    const double accturbv = RP_MUL(stdaccturbu, rp_laplace_of(rp_uniform(A, pid, d0, 3)));
    const double accwaveu = RP_MUL(stdaccwaveu, rp_normal(A, pid, d0));
    const double accwavev = RP_MUL(stdaccwavev, rp_normal(A, pid, d0 + 1));
    const double au = RP_ADD(accturbu, accwaveu), av = RP_ADD(accturbv, accwavev);
    const double acctot = sqrt(RP_ADD(RP_MUL(au, au), RP_MUL(av, av)));
    const double c1v = 2.0 / rp_log(b.vort_cr / b.vort_sat);
    const double c2v = RP_MUL(c1v, rp_log(vorttot / sqrt(RP_MUL(b.vort_cr, b.vort_sat))));
    const double c1a = 2.0 / rp_log(b.acc_cr / b.acc_sat);
    const double c2a = RP_MUL(c1a, rp_log(acctot / sqrt(RP_MUL(b.acc_cr, b.acc_sat))));
    const double ev = rp_exp(RP_MUL(-2.0, c2v)), ea = rp_exp(RP_MUL(-2.0, c2a));
    const double pswimv = RP_ADD(RP_SUB(b.b1pv, b.b0pv) / RP_ADD(1.0, ev), b.b0pv);
    const double pswima = RP_ADD(RP_SUB(b.b1pa, b.b0pa) / RP_ADD(1.0, ea), b.b0pa);
    const double pswim = (b.va_flag == 1) ? pswimv : (b.va_flag == 2) ? pswima : ((pswima < pswimv) ? pswima : pswimv);
    const double wswimv = RP_ADD(RP_MUL(RP_SUB(b.b1w, b.b0wv), 1.0) / RP_ADD(1.0, ev), b.b0wv);
    const double wswima = RP_ADD(RP_MUL(RP_SUB(b.b1w, b.b0wa), 1.0) / RP_ADD(1.0, ea), b.b0wa);
    const double wswim = (b.va_flag == 1) ? wswimv : (b.va_flag == 2) ? wswima : RP_ADD(wswima, wswimv);
    const double r = b.initsize / 2.0e4;
    const double t1 = RP_MUL(RP_MUL(RP_MUL(RP_MUL(4.0 / 3.0, G), RP_MUL(RP_MUL(r, r), r)), RHOF), RHOP - RHOF);
    const double wsink = RP_SUB(RP_MUL(3.0, MU), sqrt(RP_ADD(t1, RP_MUL(9.0, RP_MUL(MU, MU))))) / RP_MUL(r, RHOF);
    double ssf;
    if (rp_uniform(A, pid, d0, 4) < pswim) {
        wb = wswim;
        ssf = 0.0;
    } else {
        wb = wsink;
        ssf = 1.0;
    }
    const RpParticlesDev& P = A.p;
    P.acc[n] = acctot / 100.0;
    P.vort[n] = vorttot;
    P.behavew[n] = wb;
    P.ssf[n] = ssf;
    return wb;
}

// ZBehav of behave (381-391) from the vertical velocity wb
__device__ __forceinline__ double rp_behave_z(const RpStepArgs& A, double wb) {
    if (A.beh.behavior == 1) return RP_MUL(A.beh.swimfast, (double)A.idt);
    if (A.beh.behavior == 10) return RP_MUL(wb, (double)A.idt) / 100.0;
    return 0.0;
}

// getInterp3D of a behave field, ztype 2 (the w levels) at one slot; wcf
// as for rp_tracer_at
template <typename T>
__device__ __forceinline__ double rp_wfield_at(const RpGridDev& g, const void* f, const RhoCell& c, double zeta,
                                               double depth, double zpar, int slot, const double* wcf, uint32_t& fl) {
    LevelPick L;
    rp_walk_w(g, zeta, depth, zpar, L, fl);
    return rp_col_rho<T>(f, c, wcf ? wcf : (c.wet4 ? c.cb : c.ci), g.N + 1, L, slot);
}

// behave (behavior_module.f90:186-393) at the step's (Xpar, Ypar, Zpar) in
// the particle's grid: with Process_VA / Process_WA the standard deviations
// of turbulent acceleration and vorticity and of wave acceleration at the
// particle (240-280), then the response; returns ZBehav.  Out of line: the
// passive step keeps its registers.
template <typename T>
__device__ __noinline__ double rp_behave(const RpStepArgs& A, int64_t n, const RpGridDev& g, double Xpar,
                                         double Ypar, double Zpar, uint32_t pid, uint32_t& fl) {
    const RpBehaviorDev& b = A.beh;
    double wb = 0.0;
    if (b.va || b.wa) {
        RhoCell c;
        rp_rho_cell(g, Xpar, Ypar, c, fl);
        const double depth = -1.0 * rp_bil(g.h, c);
        const double zt[3] = {rp_zeta_at<T>(g, c, g.sb), rp_zeta_at<T>(g, c, g.sc), rp_zeta_at<T>(g, c, g.sf)};
        const int sl[3] = {g.sb, g.sc, g.sf};
        double wcf[3][4];                                  // WETDRY: each slot's weights, once
        if (A.wetdry)
            for (int q = 0; q < 3; q++) rp_rho_wd_weights(g, c, sl[q], wcf[q], fl);
        auto wq = [&](int q) -> const double* { return A.wetdry ? wcf[q] : nullptr; };
        double ey[3], stdaccturbu = 0.0, stdvortturb = 0.0, stdaccwaveu = 0.0, stdaccwavev = 0.0;
        if (b.va) {
            for (int q = 0; q < 3; q++) ey[q] = rp_wfield_at<T>(g, g.turbaccel, c, zt[q], depth, Zpar, sl[q], wq(q), fl);
            stdaccturbu = rp_polintd(A.pi, ey[0], ey[1], ey[2]);
            for (int q = 0; q < 3; q++) ey[q] = rp_wfield_at<T>(g, g.turbvort, c, zt[q], depth, Zpar, sl[q], wq(q), fl);
            stdvortturb = rp_polintd(A.pi, ey[0], ey[1], ey[2]);
            stdaccturbu = RP_MUL(stdaccturbu, 100.0);
        }
        if (b.wa) {
            for (int q = 0; q < 3; q++) ey[q] = rp_wfield_at<T>(g, g.waveaccelu, c, zt[q], depth, Zpar, sl[q], wq(q), fl);
            stdaccwaveu = rp_polintd(A.pi, ey[0], ey[1], ey[2]);
            for (int q = 0; q < 3; q++) ey[q] = rp_wfield_at<T>(g, g.waveaccelv, c, zt[q], depth, Zpar, sl[q], wq(q), fl);
            stdaccwavev = rp_polintd(A.pi, ey[0], ey[1], ey[2]);
            stdaccwaveu = RP_MUL(stdaccwaveu, 100.0);
            stdaccwavev = RP_MUL(stdaccwavev, 100.0);
        }
        wb = rp_behave_swim(A, n, pid, stdaccturbu, stdvortturb, stdaccwaveu, stdaccwavev);
    }
    return rp_behave_z(A, wb);
}

// One particle of update_particles.  With turbv_in non-null the VTurb
// displacement comes from the split kernel instead of being computed here.
template <typename T, class W>
__device__ void rp_update_one(const RpStepArgs& A, int64_t n, const W& w, const double* turbv_in) {
    const RpParticlesDev& P = A.p;
    if (!rp_active(A, n)) return;                          // ROMSPath.f90:672-690
    P.age[n] = P.age[n] + (double)(float)A.idt;            // 693

    uint32_t fl = 0;
    int gid = P.gid[n];
    const RpGridDev& g = A.g[gid - 1];
    const uint32_t pid = P.pid[n];
    const double Xpar = P.x[n], Ypar = P.y[n], z0 = P.z[n];
    double Zpar = z0;

    double pm, pn;                                         // 727-728
    {
        const int I = rp_ifloor(Xpar), J = rp_ifloor(Ypar);
        const double X = Xpar - (double)I, Y = Ypar - (double)J;
        const int i0 = rp_clamp(I, 1, g.nx, fl), i1 = rp_clamp(I + 1, 1, g.nx, fl);
        const int j0 = rp_clamp(J, 1, g.ny, fl), j1 = rp_clamp(J + 1, 1, g.ny, fl);
        const int64_t o00 = (int64_t)(j0 - 1) * g.nx + (i0 - 1), o10 = (int64_t)(j0 - 1) * g.nx + (i1 - 1);
        const int64_t o11 = (int64_t)(j1 - 1) * g.nx + (i1 - 1), o01 = (int64_t)(j1 - 1) * g.nx + (i0 - 1);
        const double c0 = (1 - X) * (1 - Y), c1 = X * (1 - Y), c2 = X * Y, c3 = (1 - X) * Y;
        pm = c0 * __ldg(g.pm + o00) + c1 * __ldg(g.pm + o10) + c2 * __ldg(g.pm + o11) + c3 * __ldg(g.pm + o01);
        pn = c0 * __ldg(g.pn + o00) + c1 * __ldg(g.pn + o10) + c2 * __ldg(g.pn + o11) + c3 * __ldg(g.pn + o01);
    }

    double AdvectX = 0.0, AdvectY = 0.0, AdvectZ = 0.0;
    StageState S1;
    bool have_s1 = false;
    if (A.scheme == 1) {                                   // RKAdvect, advection_module.f90:20-125
        const double didt = (double)A.idt;
        double Uad, Vad, Wad;
        StageState St;
        rp_find_currents<T>(A, g, Xpar, Ypar, Zpar, Uad, Vad, Wad, S1, fl);
        have_s1 = true;
        const double kn1_u = Uad * pm, kn1_v = Vad * pn, kn1_w = Wad;
        double x1 = Xpar + Uad * pm * didt / 2.0;
        double y1 = Ypar + Vad * pn * didt / 2.0;
        double z1 = Zpar + Wad * didt / 2.0;
        rp_find_currents<T>(A, g, x1, y1, z1, Uad, Vad, Wad, St, fl);
        const double kn2_u = Uad * pm, kn2_v = Vad * pn, kn2_w = Wad;
        double x2 = Xpar + Uad * pm * didt / 2.0;
        double y2 = Ypar + Vad * pn * didt / 2.0;
        double z2 = Zpar + Wad * didt / 2.0;
        rp_find_currents<T>(A, g, x2, y2, z2, Uad, Vad, Wad, St, fl);
        const double kn3_u = Uad * pm, kn3_v = Vad * pn, kn3_w = Wad;
        double x3 = Xpar + Uad * pm * didt / 2.0;
        double y3 = Ypar + Vad * pn * didt / 2.0;
        double z3 = Zpar + Wad * didt / 2.0;
        rp_find_currents<T>(A, g, x3, y3, z3, Uad, Vad, Wad, St, fl);
        const double kn4_u = Uad * pm, kn4_v = Vad * pn, kn4_w = Wad;
        const double P_U = (kn1_u + 2.0 * kn2_u + 2.0 * kn3_u + kn4_u) / 6.0;
        const double P_V = (kn1_v + 2.0 * kn2_v + 2.0 * kn3_v + kn4_v) / 6.0;
        const double P_W = (kn1_w + 2.0 * kn2_w + 2.0 * kn3_w + kn4_w) / 6.0;
        AdvectX = didt * P_U;
        AdvectY = didt * P_V;
        AdvectZ = didt * P_W;
    }

    double TurbHx = 0.0, TurbHy = 0.0;
    if (A.hturb_on) {                                      // HTurb, hor_turb_module.f90:30-51
        const double r = 1.0;
        const double KM = A.khturb[gid - 1];
        const double devX = rp_normal(A, pid, 0u);
        const double devY = rp_normal(A, pid, 1u);
        TurbHx = devX * sqrt(2.0 / r * KM * (double)A.idt);
        TurbHy = devY * sqrt(2.0 / r * KM * (double)A.idt);
    }
    TurbHx = TurbHx * pm;
    TurbHy = TurbHy * pn;

    double TurbV = 0.0;
    if (A.vturb_on && turbv_in) {                          // VTurb, 783 (split kernel)
        TurbV = turbv_in[n];
    } else if (A.vturb_on) {                               // VTurb, 783
        if (!have_s1) {
            rp_rho_cell(g, Xpar, Ypar, S1.rc, fl);
            S1.tdepth = -1.0 * rp_bil(g.h, S1.rc);
            S1.zb = rp_zeta_at<T>(g, S1.rc, g.sb);
            S1.zc = rp_zeta_at<T>(g, S1.rc, g.sc);
            S1.zf = rp_zeta_at<T>(g, S1.rc, g.sf);
            S1.zeta = rp_polintd(A.pi, S1.zb, S1.zc, S1.zf);
        }
        TurbV = rp_vturb<T>(A, g, S1, Zpar, pid, fl, w);
    }
    double ZBehav = 0.0;                                   // behave(), 800-804
    if (A.beh.behavior || A.beh.va || A.beh.wa) ZBehav = rp_behave<T>(A, n, g, Xpar, Ypar, Zpar, pid, fl);

    // new position and nest hand-off (821-836)
    const double newXpos = P.x[n] + AdvectX + TurbHx;
    const double newYpos = P.y[n] + AdvectY + TurbHy;
    double tempX = newXpos, tempY = newYpos;
    bool ingrid = false, obound = false;
    for (int i = 1; i <= A.ngrid; i++) {
        tempX = g.scl[i - 1][0] * newXpos + g.off[i - 1][0];
        tempY = g.scl[i - 1][1] * newYpos + g.off[i - 1][1];
        rp_bounds(A.g[i - 1], tempX, tempY, ingrid, obound);
        if (ingrid) { gid = i; break; }
    }
    const RpGridDev& gn = A.g[gid - 1];
    RhoCell rn;
    rp_rho_cell(gn, tempX, tempY, rn, fl);
    const double tdepth = -1.0 * rp_bil(gn.h, rn);         // 837
    const double e0 = 1.0 * rp_zeta_at<T>(gn, rn, gn.sb);
    const double e1 = 1.0 * rp_zeta_at<T>(gn, rn, gn.sc);
    const double e2 = 1.0 * rp_zeta_at<T>(gn, rn, gn.sf);
    const double P_zeta = rp_polintd(A.pi, e0, e1, e2);    // 843
    P.wd[n] = (-1.0 * tdepth) + P_zeta;
    P.zeta[n] = P_zeta;
    P.bath[n] = -1.0 * tdepth;
    bool hbot = false, htop = false;
    double newZpos;
    if (A.nsb == 0) {                                      // 852-872
        newZpos = z0 + AdvectZ + TurbV + ZBehav;
        if (newZpos < tdepth) { newZpos = tdepth + fabs(newZpos - tdepth); hbot = true; }
        if (newZpos > P_zeta) { newZpos = P_zeta - fabs(newZpos - P_zeta); htop = true; }
    } else if (A.nsb == 1) {
        newZpos = P_zeta - A.vertdist;
    } else {
        newZpos = tdepth + A.vertdist;
    }
    if (ingrid) {                                          // 874-892
        P.isin[n] = 1;
        P.x[n] = tempX;
        P.y[n] = tempY;
        P.z[n] = newZpos;
        double st = 1.0;
        if (htop) st = RP_F_1P1;
        if (hbot) st = RP_F_1P2;
        P.status[n] = st;
        P.gid[n] = gid;
    } else if (obound) {
        P.isin[n] = 0;
        P.gid[n] = A.ngrid;
        P.status[n] = -8.0;
    } else {
        P.isin[n] = 1;
        P.status[n] = -9.0;
    }
    if (A.diag) rp_diag_one<T>(A, n, tdepth, fl);
    if (fl) P.flags[n] |= fl;
}
