// rp_mixed.cuh -- the mixed-precision form of the particle step.
//
// Same algorithm as the FP64 form (rp_step.cuh), with
//   * positions in FP32 with Kahan-compensated accumulation (p - c),
//   * u, v, w, AKs stored in FP16 with a scale per (ring slot, level),
//     zeta in FP32; interpolation, RK4 and reflections in FP32,
//   * age in FP64,
//   * the PPPACK smoothing-spline fit with its factor's leading rows, the
//     secant search and the random-displacement sub-steps in FP64 and the
//     substitution sweeps in FP32, the search for the smoothing parameter
//     started from the particle's values of the previous steps (one chol1d
//     pass when the guess meets smooth()'s 1 % criterion).
// The 16-bit storage is FP16 (RP_FIELD_MIXED) or int16 fixed point
// (RP_FIELD_MIXED_I16, |v| / scale <= 32767 with scale = level max / 32767).
// The four ring slots of one (point, level) are one 8-byte load (16 bytes
// for zeta), and polintd's time interpolation at ix(2) is applied as its
// Lagrange weights on the b/c/f slots (RpStepArgs::lw), summed on the host
// by the physical slot each sits in (RpGridDev::w4, the spare slot's
// weight 0) and combined with the level scales before the corner sum; the
// spare slot never holds a non-finite value there (finite quantisation,
// masked FP32 slots, cleared when an upload frees it).  polintd is linear
// in its values, so the s-level depths are formed once from the
// interpolated zeta.  Results differ from the exact form by rounding; the
// error is measured against the FP64 form on identical noise.
#pragma once

#include <cuda_fp16.h>

#include "rp_step.cuh"

// ------------------------------------------------------------ cells (FP32)

// Corner offsets (j * xi + i) in 32 bits: every field index of this form,
// offset * levels + level, stays below 2^31 (rp_create checks the grids).
using MOff = int32_t;

struct MRho {
    MOff o[4];
    float X, Y;
    float cb[4];
    float ci[4];
    float hb;                      // h, bilinear (getInterp2D's rule for h)
    bool wet4;
};

__device__ __forceinline__ int m_floor(float x) {
    const float f = floorf(x);
    if (!(f >= -1.0e9f)) return -1000000000;
    if (f > 1.0e9f) return 1000000000;
    return (int)f;
}

// getcoeff's inverse-distance weights; 1/dist from one reciprocal square
// root of dist^2 (dist = 0 exactly where dist^2 = 0)
__device__ __forceinline__ void m_getcoeff(float X, float Y, const float m[4], float cff[4], uint32_t& fl) {
    float d2[4], W[4];
    d2[0] = X * X + Y * Y;
    d2[1] = (1.f - X) * (1.f - X) + Y * Y;
    d2[2] = (1.f - X) * (1.f - X) + (1.f - Y) * (1.f - Y);
    d2[3] = X * X + (1.f - Y) * (1.f - Y);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (d2[k] == 0.f) {
            fl |= RP_FL_NODE;
            if (m[k] != 0.f) {
#pragma unroll
                for (int q = 0; q < 4; q++) cff[q] = (q == k) ? 1.f : 0.f;
                return;
            }
            W[k] = 0.f;
        } else {
            W[k] = m[k] * rsqrtf(d2[k]);
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
    c.o[0] = (j0 - 1) * g.nx + (i0 - 1);
    c.o[1] = (j0 - 1) * g.nx + (i1 - 1);
    c.o[2] = (j1 - 1) * g.nx + (i1 - 1);
    c.o[3] = (j1 - 1) * g.nx + (i0 - 1);
    const float X = c.X, Y = c.Y;
    c.cb[0] = (1.f - X) * (1.f - Y);
    c.cb[1] = X * (1.f - Y);
    c.cb[2] = X * Y;
    c.cb[3] = (1.f - X) * Y;
    float m[4], hk[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float2 a = __ldg(g.hm + c.o[k]);       // (h, mask_rho)
        hk[k] = a.x;
        m[k] = a.y;
    }
    c.hb = c.cb[0] * hk[0] + c.cb[1] * hk[1] + c.cb[2] * hk[2] + c.cb[3] * hk[3];
    c.wet4 = (m[0] + m[1] + m[2] + m[3]) >= 4.f;
    m_getcoeff(X, Y, m, c.ci, fl);
}

__device__ __forceinline__ float m_bil(const double* a, const MRho& c) {
    return c.cb[0] * (float)__ldg(a + c.o[0]) + c.cb[1] * (float)__ldg(a + c.o[1]) +
           c.cb[2] * (float)__ldg(a + c.o[2]) + c.cb[3] * (float)__ldg(a + c.o[3]);
}

// time weights of the b, c, f ring slots (polintd at ix(2) in Lagrange
// form) and the physical slots they sit in
struct MTime {
    float wb, wc, wf;
    int sb, sc, sf;
    float4 w4;                     // the same weights by physical slot (0 for the spare slot)
    uint4 m32;                     // bit masks of the three live slots of an FP32 float4
};

// The four FP32 slots of a value, the spare slot's bits cleared: the spare
// slot (the one an upload may be filling) can hold anything, NaN included,
// and its weight of 0 must not meet it.  (The 16-bit fields need no mask:
// their quantisation stores finite values only and finite scales.)
__device__ __forceinline__ float4 m_live4(const float4& v, const uint4& m) {
    return make_float4(__uint_as_float(__float_as_uint(v.x) & m.x), __uint_as_float(__float_as_uint(v.y) & m.y),
                       __uint_as_float(__float_as_uint(v.z) & m.z), __uint_as_float(__float_as_uint(v.w) & m.w));
}

__device__ __forceinline__ float m_pick4(const float4& v, int s) {
    return s == 0 ? v.x : (s == 1 ? v.y : (s == 2 ? v.z : v.w));
}

// time-interpolated zeta at the cell's corners, inverse-distance weights
// (getInterp2D's zeta rule, interpolation_module.f90:478-486)
__device__ __forceinline__ float m_zeta(const RpGridDev& g, const MRho& c, const MTime& t) {
    const float4* z = reinterpret_cast<const float4*>(g.zeta);
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float4 v = m_live4(__ldg(z + c.o[q]), t.m32);
        acc += c.ci[q] * fmaf(t.w4.w, v.w, fmaf(t.w4.z, v.z, fmaf(t.w4.y, v.y, t.w4.x * v.x)));
    }
    return acc;
}

struct MUV {
    MOff o[4];
    float cff[4];
    bool use[4];
};

// u / v corner sets with the reference's edge rules (interpolation_module.f90:608-767)
// The masks are mask_u / mask_v, or under WETDRY one ring slot's
// wetdry_mask_u / _v (mk = the ring, ms = RP_SLOTS, mo = the physical slot).
__device__ __forceinline__ void m_uv_cell(const RpGridDev& g, float ip, float jp, bool is_u, MUV& c, uint32_t& fl,
                                          const uint8_t* mk = nullptr, int ms = 1, int mo = 0) {
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
        for (int k = 0; k < 4; k++) c.o[k] = (cj[k] - 1) * xi_u + (ci[k] - 1);
        const uint8_t* mm = mk ? mk : g.mu;
#pragma unroll
        for (int k = 0; k < 4; k++) m[k] = (float)__ldg(mm + c.o[k] * ms + mo);
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
        for (int k = 0; k < 4; k++) c.o[k] = (cj[k] - 1) * xi_v + (ci[k] - 1);
        const uint8_t* mm = mk ? mk : g.mv;
#pragma unroll
        for (int k = 0; k < 4; k++) m[k] = (float)__ldg(mm + c.o[k] * ms + mo);
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

// The level brackets of getInterp3D for rho levels (ztype 1) and w levels
// (ztype 2) (interpolation_module.f90:529-582), with the reference's
// boundary cases (rho: constant outside; w: pinned as in the FP64 form).
// The first w level above zpar is found by bisection over the monotone
// levels; rho level k lies between w levels k and k+1, so one more depth
// decides the rho bracket.
__device__ __forceinline__ void m_walk2(const RpGridDev& g, float zeta, float depth, float zpar, MPick& Lr,
                                        MPick& Lw, uint32_t& fl) {
    const int N = g.N, vt = g.vtransform;
    const float hc = (float)g.hc;
    const float h = -depth;
    const float den_r = 1.f / (hc + h);
    auto zw = [&](int k) -> float {
        const float2 a = __ldg(g.scs_w + k - 1);
        return m_zlev(vt, hc, h, den_r, a.x, a.y, zeta);
    };
    auto zr = [&](int k) -> float {
        const float2 a = __ldg(g.scs_r + k - 1);
        return m_zlev(vt, hc, h, den_r, a.x, a.y, zeta);
    };
    int lo = 0, hi = N + 2;             // zw(lo) <= zpar < zw(hi) (virtual ends)
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (zw(mid) > zpar) hi = mid; else lo = mid;
    }
    const int iw = hi;                  // first w level above zpar, N+2 if none
    int ir;                             // first rho level above zpar, N+1 if none
    if (iw == 1) ir = 1;
    else if (iw > N + 1) ir = N + 1;
    else ir = (zr(iw - 1) > zpar) ? iw - 1 : iw;
    if (iw > N + 1) {
        fl |= RP_FL_WTOP;
        Lw.ibot = N + 1; Lw.itop = N + 1; Lw.z1 = 0.5f; Lw.z2 = 0.5f;
    } else if (iw == 1) {
        fl |= RP_FL_WBOT;
        Lw.ibot = 1; Lw.itop = 1; Lw.z1 = 0.5f; Lw.z2 = 0.5f;
    } else {
        const float za = zw(iw - 1), zb = zw(iw);
        const float Z = (zpar - za) / (zb - za);
        Lw.ibot = iw - 1; Lw.itop = iw; Lw.z1 = 1.f - Z; Lw.z2 = Z;
    }
    if (ir > N) {
        Lr.ibot = N; Lr.itop = N; Lr.z1 = 0.5f; Lr.z2 = 0.5f;
    } else if (ir == 1) {
        Lr.ibot = 1; Lr.itop = 1; Lr.z1 = 0.5f; Lr.z2 = 0.5f;
    } else {
        const float za = zr(ir - 1), zb = zr(ir);
        const float Z = (zpar - za) / (zb - za);
        Lr.ibot = ir - 1; Lr.itop = ir; Lr.z1 = 1.f - Z; Lr.z2 = Z;
    }
}

// one stored 16-bit value (before its level scale): FP16, or int16 fixed point
template <typename E>
__device__ __forceinline__ float m_dec(uint32_t bits);
template <>
__device__ __forceinline__ float m_dec<__half>(uint32_t bits) {
    return __half2float(__ushort_as_half((unsigned short)bits));
}
template <>
__device__ __forceinline__ float m_dec<int16_t>(uint32_t bits) {
    return (float)(int16_t)(uint16_t)bits;
}

// slot s (0..3, uniform) of the four 16-bit slots of one (point, level)
template <typename E>
__device__ __forceinline__ float m_slot(const uint2& v, int s) {
    const uint32_t word = (s < 2) ? v.x : v.y;
    return m_dec<E>((s & 1) ? (word >> 16) : (word & 0xffffu));
}

// the four 16-bit slots of one (point, level) dotted with per-slot weights
// (slot s is half s & 1 of word s >> 1)
template <typename E>
__device__ __forceinline__ float m_dot4(const uint2& v, const float4& w);
template <>
__device__ __forceinline__ float m_dot4<__half>(const uint2& v, const float4& w) {
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
    return fmaf(w.w, b.y, fmaf(w.z, b.x, fmaf(w.y, a.y, w.x * a.x)));
}
template <>
__device__ __forceinline__ float m_dot4<int16_t>(const uint2& v, const float4& w) {
    const float a0 = (float)(int16_t)(v.x & 0xffffu), a1 = (float)((int32_t)v.x >> 16);
    const float b0 = (float)(int16_t)(v.y & 0xffffu), b1 = (float)((int32_t)v.y >> 16);
    return fmaf(w.w, b1, fmaf(w.z, b0, fmaf(w.y, a1, w.x * a0)));
}

// the level scales folded into the slot weights
__device__ __forceinline__ float4 m_scaled_w4(const MTime& t, const float4& sc) {
    return make_float4(t.w4.x * sc.x, t.w4.y * sc.y, t.w4.z * sc.z, t.w4.w * sc.w);
}

// sum over corners of cff * (time-interpolated, scaled value) at level lev
template <typename E>
__device__ __forceinline__ float m_level(const uint2* f, const float4* qs, const MOff o[4], const float cff[4],
                                         const bool use[4], int nlev, int lev, const MTime& t) {
    const float4 ws = m_scaled_w4(t, __ldg(qs + lev - 1));   // level scales [k][slot4]
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (use[q]) {
            const uint2 v = __ldg(f + o[q] * nlev + lev - 1);
            acc += cff[q] * m_dot4<E>(v, ws);
        }
    }
    return acc;
}

// the same sum from a level's four corner words and scales already loaded
template <typename E>
__device__ __forceinline__ float m_level_of(const uint2 v[4], const float4& sc, const float cff[4],
                                            const bool use[4], const MTime& t) {
    const float4 ws = m_scaled_w4(t, sc);
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++)
        if (use[q]) acc += cff[q] * m_dot4<E>(v[q], ws);
    return acc;
}

// zcff1*zprof(Ibot) + zcff2*zprof(Itop), time-interpolated
template <typename E>
__device__ __forceinline__ float m_col(const void* fv, const float* qs, const MOff o[4], const float cff[4],
                                       const bool use[4], int nlev, const MPick& L, const MTime& t) {
    const uint2* f = reinterpret_cast<const uint2*>(fv);
    const float4* q4 = reinterpret_cast<const float4*>(qs);
    const float pb = m_level<E>(f, q4, o, cff, use, nlev, L.ibot, t);
    const float pt = (L.itop == L.ibot) ? pb : m_level<E>(f, q4, o, cff, use, nlev, L.itop, t);
    return L.z1 * pb + L.z2 * pt;
}

// ---------------------------------------------- WETDRY: one slot at a time
//
// Under WETDRY each ring slot has its own masks, so the corner weights
// differ by slot and the three slots cannot share one weighted gather:
// each slot's value is formed with its own weights, then the slot weights
// are applied (interpolation_module.f90:628-939).

// one slot's value at level lev of a 16-bit field
template <typename E>
__device__ __forceinline__ float m_level_slot(const uint2* f, const float4* qs, const MOff o[4],
                                              const float cff[4], const bool use[4], int nlev, int lev, int s) {
    const float sc = m_pick4(__ldg(qs + lev - 1), s);
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++)
        if (use[q]) acc += cff[q] * m_slot<E>(__ldg(f + o[q] * nlev + lev - 1), s);
    return acc * sc;
}

template <typename E>
__device__ __forceinline__ float m_col_slot(const void* fv, const float* qs, const MOff o[4], const float cff[4],
                                            const bool use[4], int nlev, const MPick& L, int s) {
    const uint2* f = reinterpret_cast<const uint2*>(fv);
    const float4* q4 = reinterpret_cast<const float4*>(qs);
    const float pb = m_level_slot<E>(f, q4, o, cff, use, nlev, L.ibot, s);
    const float pt = (L.itop == L.ibot) ? pb : m_level_slot<E>(f, q4, o, cff, use, nlev, L.itop, s);
    return L.z1 * pb + L.z2 * pt;
}

// rho-point weights of one slot: bilinear, or getcoeff's with that slot's
// wetdry_mask_rho when a corner is dry
__device__ __forceinline__ void m_rho_wd_cff(const RpGridDev& g, const MRho& c, int s, float cff[4], uint32_t& fl) {
    float m[4];
#pragma unroll
    for (int k = 0; k < 4; k++) m[k] = (float)__ldg(g.wd_rho + c.o[k] * RP_SLOTS + s);
    if (m[0] + m[1] + m[2] + m[3] < 4.f) {
        m_getcoeff(c.X, c.Y, m, cff, fl);
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) cff[k] = c.cb[k];
    }
}

// find_currents' u, v, w under WETDRY (out of line: the step keeps its
// registers when WETDRY is off)
template <typename E>
__device__ __noinline__ void m_gather_wd(const RpStepArgs& A, const RpGridDev& g, float X, float Y, const MRho& rc,
                                         const MPick& Lr, const MPick& Lw, float& U, float& V, float& Wv,
                                         uint32_t& fl) {
    const int N = g.N;
    const bool all[4] = {true, true, true, true};
    const float wt[3] = {A.lw[1][0], A.lw[1][1], A.lw[1][2]};   // (b, b, c) at ets == 1
    const int sl[3] = {g.sb, g.sc, g.sf};
    U = 0.f;
    V = 0.f;
    Wv = 0.f;
    for (int q = 0; q < 3; q++) {
        if (wt[q] == 0.f) continue;
        MUV c;
        m_uv_cell(g, X, Y, true, c, fl, g.wd_u, RP_SLOTS, sl[q]);
        U += wt[q] * m_col_slot<E>(g.u, g.qs_u, c.o, c.cff, c.use, N, Lr, sl[q]);
        m_uv_cell(g, X, Y, false, c, fl, g.wd_v, RP_SLOTS, sl[q]);
        V += wt[q] * m_col_slot<E>(g.v, g.qs_v, c.o, c.cff, c.use, N, Lr, sl[q]);
        float cw[4];
        m_rho_wd_cff(g, rc, sl[q], cw, fl);
        Wv += wt[q] * m_col_slot<E>(g.w, g.qs_w, rc.o, cw, all, N + 1, Lw, sl[q]);
    }
}

struct MStage {
    MRho rc;
    float tdepth, zeta;
};

// depth and time-interpolated zeta at the stage's cell S.rc
__device__ __forceinline__ void m_stage_2d(const MTime& tz, const RpGridDev& g, MStage& S) {
    S.tdepth = -S.rc.hb;
    S.zeta = m_zeta(g, S.rc, tz);
}

__device__ __forceinline__ MTime m_time(const RpStepArgs& A, const RpGridDev& g, int which) {
    MTime t;
    t.wb = A.lw[which][0];
    t.wc = A.lw[which][1];
    t.wf = A.lw[which][2];
    t.sb = g.sb;
    t.sc = g.sc;
    t.sf = g.sf;
    // by physical slot, and the live slots' masks (host-computed per step)
    t.w4 = g.w4[which];
    t.m32 = g.m32;
    return t;
}

// find_currents (advection_module.f90:129-350) in FP32 on 16-bit fields;
// Z is INOUT.  E is the 16-bit storage type of u, v, w; FEAT: a kernel
// built for the options beyond the passive step (here WETDRY).
template <typename E, bool FEAT>
__device__ __forceinline__ void m_find_currents(const RpStepArgs& A, const RpGridDev& g, float X, float Y, float& Z,
                                                float& U, float& V, float& Wv, uint32_t& fl) {
    MStage S;
    m_rho_cell(g, X, Y, S.rc, fl);
    m_stage_2d(m_time(A, g, 0), g, S);
    if (Z < S.tdepth) Z = S.tdepth + 0.001f;
    if (Z > S.zeta) Z = S.zeta - 0.001f;
    MPick Lr, Lw;
    m_walk2(g, S.zeta, S.tdepth, Z, Lr, Lw, fl);
    if (FEAT && A.wetdry) {
        m_gather_wd<E>(A, g, X, Y, S.rc, Lr, Lw, U, V, Wv, fl);
        return;
    }
    const int N = g.N;
    const MTime tv = m_time(A, g, 1);                  // (b, b, c) at ets == 1
    {
        MUV cu;
        m_uv_cell(g, X, Y, true, cu, fl);
        U = m_col<E>(g.u, g.qs_u, cu.o, cu.cff, cu.use, N, Lr, tv);
    }
    {
        MUV cv;
        m_uv_cell(g, X, Y, false, cv, fl);
        V = m_col<E>(g.v, g.qs_v, cv.o, cv.cff, cv.use, N, Lr, tv);
    }
    const bool all[4] = {true, true, true, true};
    const float* cw = S.rc.wet4 ? S.rc.cb : S.rc.ci;
    Wv = m_col<E>(g.w, g.qs_w, S.rc.o, cw, all, N + 1, Lw, tv);
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

// Workspace: the chol1d arrays (ratio1, ratio2 and u), then four FP32
// arrays for the data (the column and the resampled values carry FP32
// information only).  RP_MIXED_WS sets the chol1d arrays' storage: 0 all
// FP64, 1 the factor ratios FP32 and u FP64, 2 all FP32 (the default; the
// sweeps of m_chol1d compute in FP32 either way).  kMixedArrays (NPMAX+1)
// doubles in all.
#ifndef RP_MIXED_WS
#define RP_MIXED_WS 2
#endif
#if RP_MIXED_WS == 0
using MRatio = double;
using MU = double;
#elif RP_MIXED_WS == 1
using MRatio = float;
using MU = double;
#else
using MRatio = float;
using MU = float;
#endif
constexpr int kMixedBytesPerPoint = 2 * (int)sizeof(MRatio) + (int)sizeof(MU) + 4 * 4;
constexpr int kMixedArrays = (kMixedBytesPerPoint + 7) / 8;

struct MFit;

// The per-thread workspace in local memory (the fused step): every array
// of the fit, the resampled data y stored by the first pass.  PREF: the
// back substitution loads u four rows ahead (fewer stalls, more registers
// live; which is faster depends on the workload).
template <int NPMAX, bool PREF = true>
struct MSpline {
    static constexpr bool kStoreY = true;
    static constexpr int kColBatch = 2;
    static constexpr bool kLightCheck = false;
    static constexpr bool kPrefetch = PREF;
    double* base;
    __device__ __forceinline__ MU& u(int i) const { return reinterpret_cast<MU*>(base)[i]; }  // u(i)/v(i,1), then u(i)
    __device__ __forceinline__ MRatio* rb() const {
        return reinterpret_cast<MRatio*>(reinterpret_cast<char*>(base) + (NPMAX + 1) * sizeof(MU));
    }
    __device__ __forceinline__ MRatio& s1(int i) const { return rb()[i]; }                   // ratio1(i)
    __device__ __forceinline__ MRatio& s2(int i) const { return rb()[(NPMAX + 1) + i]; }     // ratio2(i)
    __device__ __forceinline__ float* fb() const {
        return reinterpret_cast<float*>(reinterpret_cast<char*>(base) + (NPMAX + 1) * (sizeof(MU) + 2 * sizeof(MRatio)));
    }
    __device__ __forceinline__ float& y(int i) const { return fb()[i]; }                     // resampled data y(i)
    __device__ __forceinline__ float& cz(int k) const { return fb()[(NPMAX + 1) + k]; }      // column z(k)
    __device__ __forceinline__ float& cm(int k) const { return fb()[2 * (NPMAX + 1) + k]; }  // slope on [z(k), z(k+1)]
    __device__ __forceinline__ float& cb(int k) const { return fb()[3 * (NPMAX + 1) + k]; }  // intercept
    __device__ __forceinline__ double yat(const MFit&, int i) const { return (double)y(i); }
};

struct MFit {
    int np, sw;
    double z1, h, rh;              // first break, spacing, 1/h
    double serr, dy2;
};

// The workspace in shared memory (the split step's VTurb kernel): u, the
// factor ratios of the rows before the factor turns stationary (rows
// 2..KSM+1; later rows, met only when it does not, in the thread's local
// array `ovf`), and the column's breaks, slopes and intercepts (sw <= CMAX).
// Element k of a thread sits at word k * B of its own column (threads of a
// block in consecutive banks).  The resampled data are not stored: ppvalu's
// two values per piece come from the column (the same m x + b the fit's
// sweep forms).
template <int NPMAX, int KSM, int CMAX, int B>
struct MSmemSpline {
    static_assert(sizeof(MU) == 4 && sizeof(MRatio) == 4, "shared-memory workspace holds FP32 arrays");
    static constexpr bool kStoreY = false;
    static constexpr int kColBatch = 8;
    static constexpr bool kLightCheck = true;
    static constexpr bool kPrefetch = true;
    static constexpr int kWords = NPMAX + 2 * KSM + 3 * CMAX;
    float* sm;                     // this thread's first word
    float* ovf;                    // 2 (NPMAX + 1) floats, local
    __device__ __forceinline__ float& u(int i) const { return sm[(i - 1) * B]; }
    __device__ __forceinline__ float& s1(int i) const {
        return (i <= KSM + 1) ? sm[(NPMAX + i - 2) * B] : ovf[i];
    }
    __device__ __forceinline__ float& s2(int i) const {
        return (i <= KSM + 1) ? sm[(NPMAX + KSM + i - 2) * B] : ovf[NPMAX + 1 + i];
    }
    __device__ __forceinline__ float& y(int) const { return ovf[0]; }        // never stored (kStoreY)
    __device__ __forceinline__ float& cz(int k) const { return sm[(NPMAX + 2 * KSM + k - 1) * B]; }
    __device__ __forceinline__ float& cm(int k) const { return sm[(NPMAX + 2 * KSM + CMAX + k - 1) * B]; }
    __device__ __forceinline__ float& cb(int k) const { return sm[(NPMAX + 2 * KSM + 2 * CMAX + k - 1) * B]; }
    // resampled value y(i) at z1 + (i-1) h: the column piece j with
    // cz(j) <= x (j in 1..sw-1; 1 below cz(2)), found by bisection
    __device__ __forceinline__ double yat(const MFit& f, int i) const;
};

// linint of the column at ascending points: the current piece j (slope,
// intercept and upper end) is held in registers and advanced as needed
template <class W>
struct MWalk {
    int j;
    double zn, m, b;               // cz(j+1), cm(j), cb(j)
    __device__ __forceinline__ void init(const W& w) {
        j = 1;
        zn = w.cz(2);
        m = w.cm(1);
        b = w.cb(1);
    }
    __device__ __forceinline__ double at(const W& w, int sw, double x) {
        while (j < sw - 1 && zn <= x) {
            j++;
            zn = w.cz(j + 1);
            m = w.cm(j);
            b = w.cb(j);
        }
        return m * x + b;
    }
};

template <int NPMAX, int KSM, int CMAX, int B>
__device__ __forceinline__ double MSmemSpline<NPMAX, KSM, CMAX, B>::yat(const MFit& f, int i) const {
    const double x = (i == 1) ? f.z1 : f.z1 + (double)(i - 1) * f.h;
    int lo = 1, hi = f.sw - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((double)cz(mid) <= x) lo = mid; else hi = mid - 1;
    }
    return (double)cm(lo) * x + (double)cb(lo);
}

// linint of the column at ascending points in FP32 (the column's breaks,
// slopes and intercepts are stored in FP32)
template <class W>
struct MWalkF {
    int j;
    float zn, m, b;                // cz(j+1), cm(j), cb(j)
    __device__ __forceinline__ void init(const W& w) {
        j = 1;
        zn = w.cz(2);
        m = w.cm(1);
        b = w.cb(1);
    }
    __device__ __forceinline__ float at(const W& w, int sw, float x) {
        while (j < sw - 1 && zn <= x) {
            j++;
            zn = w.cz(j + 1);
            m = w.cm(j);
            b = w.cb(j);
        }
        return fmaf(m, x, b);
    }
};

// One chol1d pass at p: factorise, solve for u, form qu = Q u; returns
// sum_i qu(i)^2 dy^2 and, on request, utru = sum v4 (u(i-1)(u(i-1)+u(i)) + u(i)^2).
// The factor's rows before it turns stationary are formed in FP64 and
// stored in FP32; the substitutions, qu and its sum run in FP32 (the data,
// the factor ratios and u are FP32 values).  With store_y the resampled
// values y(i) are also kept (for ppvalu); u is written back only with
// store_u (a pass whose u may be the fit's).
template <class W>
__device__ double m_chol1d(const W& w, const MFit& f, double p, double* utru_out, bool store_y,
                           bool store_u) {
    store_y = store_y && W::kStoreY;
    const int np = f.np;
    const double r = f.serr * f.rh;
    const double r2 = r * r;
    const double six1mp = 6.0 * (1.0 - p);
    const double D = six1mp * (6.0 * r2) + 4.0 * p * f.h;
    const double E = six1mp * (-4.0 * r2) + p * f.h;
    const double F = six1mp * r2;
    const float hf = (float)f.h, rhf = (float)f.rh, z1f = (float)f.z1;
    // Q'y on the fly: qty(i) = (y(i+1) - 2 y(i) + y(i-1)) / h, y at z1 + (i-1) h
    MWalkF<W> wk;
    wk.init(w);
    float ym = wk.at(w, f.sw, z1f);
    float y0 = wk.at(w, f.sw, z1f + hf);
    float yp = wk.at(w, f.sw, fmaf(2.f, hf, z1f));
    if (store_y) {
        w.y(1) = ym;
        w.y(2) = y0;
        w.y(3) = yp;
    }
    double a1 = D, a2 = E, b1 = D;
    float uprev = 0.f, ucur = (yp - 2.f * y0 + ym) * rhf, r2prev = 0.f;
    // The bands are constant (uniform breaks), so the factor converges to
    // a fixed point: once a row's ratios round to the previous row's in
    // FP32, rows ks..np-3 reuse them (no division, no store); the last row
    // (F = 0 there) is factorised from the held state.
    int ks = np - 1;                                 // first reused row (np-1: none)
    float hinv = 0.f, hr1 = 0.f, hr2 = 0.f;
    float pr1 = 0.f, pr2 = 0.f;
#pragma unroll 2
    for (int i = 2; i <= np - 2; i++) {
        float inv, ratio1, ratio2;
        if (i < ks || i == np - 2) {
            const double Fi = (i <= np - 3) ? F : 0.0;
            const double invd = 1.0 / a1;            // one division per row
            const double ratio1d = a2 * invd;
            const double b1n = b1 - ratio1d * a2;
            const double c2 = E - ratio1d * Fi;
            const double ratio2d = Fi * invd;
            const double c1 = D - ratio2d * Fi;
            inv = (float)invd;
            ratio1 = (float)ratio1d;
            ratio2 = (float)ratio2d;
            if (i > 2 && i < np - 2 && ratio1 == pr1 && ratio2 == pr2) {
                ks = i;
                hinv = inv;
                hr1 = ratio1;
                hr2 = ratio2;
            } else {
                w.s1(i) = ratio1;
                w.s2(i) = ratio2;
                a1 = b1n;
                a2 = c2;
                b1 = c1;
            }
            pr1 = ratio1;
            pr2 = ratio2;
        } else {
            inv = hinv;
            ratio1 = hr1;
            ratio2 = hr2;
        }
        w.u(i) = ucur * inv;
        ym = y0;
        y0 = yp;
        yp = wk.at(w, f.sw, fmaf((float)(i + 1), hf, z1f));   // y(i+2) at z1 + (i+1) h
        if (store_y) w.y(i + 2) = yp;
        const float qn = (yp - 2.f * y0 + ym) * rhf;          // qty(i+1)
        const float unext = qn - ratio1 * ucur - r2prev * uprev;
        uprev = ucur;
        ucur = unext;
        r2prev = ratio2;
    }
    // back substitution, descending, with qu and its sum of squares:
    // raw(k) = (u(k) - u(k-1))/h for 2 <= k <= np, raw(1) = raw(np+1) = 0,
    // qu(k) = raw(k+1) - raw(k)
    const bool want_utru = utru_out != nullptr;
    float up1 = 0.f;                                 // u(np)
    float up2 = 0.f;                                 // u(np+1), unused
    float rawp = 0.f;                                // raw(np+1)
    float sum = 0.f, utru = 0.f;                     // sum of qu^2 (times dy2 at the end)
    if (store_u) w.u(np) = 0.f;
    {
        const float ui = (float)((double)ucur / a1); // u(np-1)
        if (store_u) w.u(np - 1) = ui;
        const float raw = (up1 - ui) * rhf;          // raw(np)
        const float fin = rawp - raw;                // qu(np)
        sum = fmaf(fin, fin, sum);
        if (want_utru) utru = utru + hf * (ui * (ui + up1) + up1 * up1);
        rawp = raw;
        up2 = up1;
        up1 = ui;
    }
    const float h1 = hr1, h2 = hr2;                  // the held rows' ratios
    // with W::kPrefetch, u(i) is loaded four rows ahead of its use (index 1
    // stands in past the start; that value is never used)
    float q0 = w.u(np - 2), q1 = w.u(max(np - 3, 1)), q2 = w.u(max(np - 4, 1)), q3 = w.u(max(np - 5, 1));
#pragma unroll 2
    for (int i = np - 2; i >= 2; i--) {
        float uq;
        if constexpr (W::kPrefetch) {
            uq = q0;
            q0 = q1;
            q1 = q2;
            q2 = q3;
            q3 = w.u(max(i - 4, 1));
        } else {
            uq = w.u(i);
        }
        const bool held = (i >= ks && i <= np - 3);
        float s1v = h1, s2v = h2;
        if (!held) {
            s1v = w.s1(i);
            s2v = w.s2(i);
        }
        const float ui = uq - up1 * s1v - up2 * s2v;
        if (store_u) w.u(i) = ui;
        const float raw = (up1 - ui) * rhf;          // raw(i+1)
        const float fin = rawp - raw;                // qu(i+1)
        sum = fmaf(fin, fin, sum);
        if (want_utru) utru = utru + hf * (ui * (ui + up1) + up1 * up1);
        rawp = raw;
        up2 = up1;
        up1 = ui;
    }
    {
        const float raw = up1 * rhf;                 // raw(2), u(1) = 0
        const float fin2 = rawp - raw;               // qu(2)
        sum = sum + fin2 * fin2 + raw * raw;         // qu(1) = raw(2)
        if (want_utru) utru = utru + hf * (up1 * up1);
    }
    if (store_u) w.u(1) = 0.f;
    if (want_utru) *utru_out = (double)utru;
    return (double)sum * f.dy2;
}

// SF(q) = 36 sum qu^2 dy^2 / (1+q)^2 of one chol1d pass at p = q/(1+q)
template <class W>
__device__ __forceinline__ double m_sf(const W& w, const MFit& f, double q, bool store_y,
                                       bool store_u) {
    return 36.0 * m_chol1d(w, f, q / (1.0 + q), nullptr, store_y, store_u) / ((1.0 + q) * (1.0 + q));
}

// The same sum S(p) = sum qu^2 dy^2 = u'Tu (T = Q'D^2Q) from one forward
// sweep, with nothing stored and no back substitution.  With
// M(p) = 6(1-p) T + p R the matrix of chol1d and b = Q'y, let
// phi(p) = b'M^-1 b = sum_i w_i^2 / d_i over the forward-substituted values
// w = L^-1 b and the pivots d of M = L diag(d) L'.  Since u'Mu = phi and
// dphi/dp = -u'M'u = 6 u'Tu - u'Ru, phi + p phi' = 6 u'Tu, i.e.
//   S(p) = (phi(p) + p phi'(p)) / 6,
// and phi' is carried through the sweep as derivatives in p of the factor
// (D, E, F are linear in p) and of w.  The factor turns stationary as in
// m_chol1d (its ratios and their derivatives repeat in FP32); the last row
// is factorised from the held state.
template <class W>
__device__ double m_light_S(const W& w, const MFit& f, double p) {
    const int np = f.np;
    const double r = f.serr * f.rh;
    const double r2 = r * r;
    const double six1mp = 6.0 * (1.0 - p);
    const double D = six1mp * (6.0 * r2) + 4.0 * p * f.h;
    const double E = six1mp * (-4.0 * r2) + p * f.h;
    const double F = six1mp * r2;
    const double Dd = -36.0 * r2 + 4.0 * f.h;          // dD/dp, dE/dp, dF/dp
    const double Ed = 24.0 * r2 + f.h;
    const double Fd = -6.0 * r2;
    MWalk<W> wk;
    wk.init(w);
    double ym = wk.at(w, f.sw, f.z1);
    double y0 = wk.at(w, f.sw, f.z1 + f.h);
    double xn = f.z1 + 2.0 * f.h;
    double yp = wk.at(w, f.sw, xn);
    double a1 = D, a2 = E, b1 = D, a1d = Dd, a2d = Ed, b1d = Dd;
    double wc = (yp - 2.0 * y0 + ym) * f.rh, wcd = 0.0, wp = 0.0, wpd = 0.0;   // w(i), w(i-1) and d/dp
    double r2p = 0.0, r2pd = 0.0;                                               // ratio2(i-1)
    double phi = 0.0, phid = 0.0;
    bool held = false;
    double hinv = 0.0, hinvd = 0.0, hr1 = 0.0, hr1d = 0.0, hr2 = 0.0, hr2d = 0.0;
    float pr1 = 0.f, pr2 = 0.f, pr1d = 0.f, pr2d = 0.f;
#pragma unroll 2
    for (int i = 2; i <= np - 2; i++) {
        double inv, invd, ratio1, ratio1d, ratio2, ratio2d;
        if (!held || i == np - 2) {
            const double Fi = (i <= np - 3) ? F : 0.0, Fid = (i <= np - 3) ? Fd : 0.0;
            inv = 1.0 / a1;
            invd = -a1d * inv * inv;
            ratio1 = a2 * inv;
            ratio1d = a2d * inv + a2 * invd;
            ratio2 = Fi * inv;
            ratio2d = Fid * inv + Fi * invd;
            const float q1 = (float)ratio1, q2 = (float)ratio2, q1d = (float)ratio1d, q2d = (float)ratio2d;
            if (i > 2 && i < np - 2 && q1 == pr1 && q2 == pr2 && q1d == pr1d && q2d == pr2d) {
                held = true;
                hinv = inv; hinvd = invd; hr1 = ratio1; hr1d = ratio1d; hr2 = ratio2; hr2d = ratio2d;
            } else {
                const double b1n = b1 - ratio1 * a2, b1nd = b1d - ratio1d * a2 - ratio1 * a2d;
                const double c2 = E - ratio1 * Fi, c2d = Ed - ratio1d * Fi - ratio1 * Fid;
                const double c1 = D - ratio2 * Fi, c1d = Dd - ratio2d * Fi - ratio2 * Fid;
                a1 = b1n; a1d = b1nd;
                a2 = c2; a2d = c2d;
                b1 = c1; b1d = c1d;
            }
            pr1 = q1; pr2 = q2; pr1d = q1d; pr2d = q2d;
        } else {
            inv = hinv; invd = hinvd; ratio1 = hr1; ratio1d = hr1d; ratio2 = hr2; ratio2d = hr2d;
        }
        phi = phi + wc * wc * inv;
        phid = phid + (2.0 * wc * wcd) * inv + wc * wc * invd;
        ym = y0;
        y0 = yp;
        xn = xn + f.h;                               // z1 + (i+1) h, accumulated
        yp = wk.at(w, f.sw, xn);
        const double qn = (yp - 2.0 * y0 + ym) * f.rh;           // qty(i+1)
        const double wn = qn - ratio1 * wc - r2p * wp;
        const double wnd = -(ratio1d * wc + ratio1 * wcd + r2pd * wp + r2p * wpd);
        wp = wc; wpd = wcd;
        wc = wn; wcd = wnd;
        r2p = ratio2; r2pd = ratio2d;
    }
    {                                                              // row np-1
        const double inv = 1.0 / a1, invd = -a1d * inv * inv;
        phi = phi + wc * wc * inv;
        phid = phid + (2.0 * wc * wcd) * inv + wc * wc * invd;
    }
    return (phi + p * phid) * (1.0 / 6.0);
}

// True on the first internal step of an external step (ix(2) = ex(2)): the
// three frame times move on, so the time-interpolated fields jump here and
// the change of q over this step is no guide to the next one; the q history
// is then dropped (the next step starts from this step's q alone).
__device__ __forceinline__ bool m_stencil_moved(const RpStepArgs& A) { return A.ix[1] == A.ex[1]; }

// smooth() (pppack.f90:5108-5317): the secant search for q = p/(1-p) on
// 1/sqrt(SF) until |SF - s| <= 0.01 s.  Warm start: the particle's q of its
// previous step extrapolated with the one before (q2state), one pass when
// that meets the criterion, and the slope g of 1/sqrt(SF) in q found at an
// earlier step, which gives a Newton step when it does not; then secant
// steps.  Falls back to the reference's cold start (p = 0, utru) when that
// does not converge.  q and g are returned in qstate and gstate (q = 0 for
// p = 0; g <= 0 when unknown), the incoming q in q2state; passes = chol1d
// passes made.
template <class W>
__device__ double m_smooth(const W& w, const MFit& f, double s, int max_iter, double& qstate,
                           double& gstate, float& q2state, uint32_t& fl, int& passes) {
    // the first full pass of every path also stores y(i); the p = 0 pass
    // does not store u and is repeated as a full pass when p = 0 is the fit
    passes = 1;
    if (s <= 0.0) {
        m_chol1d(w, f, 1.0, nullptr, true, true);
        return 1.0;
    }
    const double ooss = 1.0 / sqrt(s);
    const double q_in = qstate;
    double q = q_in;
    const bool warm = q > 0.0;
    bool ys = false;                                 // y(i) stored by a pass already
    const double q2 = (double)q2state;               // the q of the step before the previous one
    q2state = (float)q_in;                           // the previous q, for the next step
    if (warm) {
        // first guess: this step's q extrapolated from the previous two
        // steps' (geometric, the ratio held to [1/2, 2]); the column changes
        // smoothly from step to step, so this guess usually meets the
        // criterion at once, where the previous q alone rarely does
        if (q2 > 0.0) q = q * fmin(fmax(q / q2, 0.5), 2.0);
        // the check: a full pass that stores u (the guess is usually the
        // fit), or where the view asks for it a light pass (one forward
        // sweep, nothing stored) followed by a full pass when it converged
        double sfq;
        bool us = false;
        if (W::kLightCheck) {
            sfq = 36.0 * m_light_S(w, f, q / (1.0 + q)) / ((1.0 + q) * (1.0 + q));
        } else {
            sfq = m_sf(w, f, q, true, true);
            ys = true;
            us = true;
        }
        if (fabs(sfq - s) <= 0.01 * s) {
            if (!us) {
                m_chol1d(w, f, q / (1.0 + q), nullptr, !ys, true);
                passes = 2;
            }
            // the history keeps the root estimate rather than the accepted
            // q (any q inside the 1 % band is accepted; the extrapolation
            // of such q's would carry the band's spread)
            const double qr = (gstate > 0.0) ? q - (1.0 / sqrt(sfq) - ooss) / gstate : q;
            qstate = (qr > 0.0) ? qr : q;
            return q / (1.0 + q);
        }
        double prevq = q, prevsf = 1.0 / sqrt(sfq);
        const double qn = (gstate > 0.0) ? q + (ooss - prevsf) / gstate : 0.0;
        q = (qn > 0.0) ? qn : q * sqrt(sfq / s);
        for (int it = 0; it < 6 && q > 0.0; it++) {
            sfq = m_sf(w, f, q, !ys, true);
            ys = true;
            passes++;
            const double oosf = 1.0 / sqrt(sfq);
            const double g = (oosf - prevsf) / (q - prevq);
            if (fabs(sfq - s) <= 0.01 * s) {
                const double qr = q - (oosf - ooss) / g;
                qstate = (g > 0.0 && qr > 0.0) ? qr : q;
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
    double sfq = 36.0 * m_chol1d(w, f, 0.0, &utru, !ys, false);
    passes += warm ? 1 : 0;
    if (!(s < sfq)) {
        m_chol1d(w, f, 0.0, nullptr, false, true);
        passes++;
        qstate = 0.0;
        gstate = 0.0;
        return 0.0;
    }
    double oosf = 1.0 / sqrt(sfq);
    q = -(oosf - ooss) * sfq / (6.0 * utru * oosf);
    double prevq = 0.0, prevsf = oosf;
    int it = 0;
    for (;;) {
        sfq = m_sf(w, f, q, false, true);
        oosf = 1.0 / sqrt(sfq);
        it++;
        passes++;
        const double g = (oosf - prevsf) / (q - prevq);
        if (fabs(sfq - s) <= 0.01 * s) {
            gstate = g;
            const double qr = q - (oosf - ooss) / g;
            qstate = (g > 0.0 && qr > 0.0) ? qr : q;
            return q / (1.0 + q);
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

// One piece of the fit: the coefficients a(i,1..4) smooth's epilogue forms
// (pppack.f90:5303-5316) for piece i, from u and y.
struct MPiece {
    int i;                          // 0: none yet
    double xi, c1, c2, c3, c4;
};

template <class W>
__device__ __forceinline__ void m_piece(const W& w, const MFit& f, double p, int i, MPiece& pc) {
    const int np = f.np;
    const double um = (i >= 2) ? (double)w.u(i - 1) : 0.0;
    const double u0 = (double)w.u(i), u1 = (double)w.u(i + 1);
    const double u2 = (i + 2 <= np) ? (double)w.u(i + 2) : 0.0;
    const double raw0 = (i >= 2) ? (u0 - um) * f.rh : 0.0;          // raw(i)
    const double raw1 = (u1 - u0) * f.rh;                            // raw(i+1)
    const double raw2 = (i + 2 <= np) ? (u2 - u1) * f.rh : 0.0;      // raw(i+2)
    const double K1 = 6.0 * (1.0 - p) * f.dy2;
    const double a1i = w.yat(f, i) - K1 * (raw1 - raw0);
    const double a1n = w.yat(f, i + 1) - K1 * (raw2 - raw1);
    const double a3i = u0 * 6.0 * p;
    const double a3n = u1 * 6.0 * p;
    const double a4i = (a3n - a3i) * f.rh;
    pc.i = i;
    pc.xi = f.z1 + (double)(i - 1) * f.h;
    pc.c1 = a1i;
    pc.c2 = (a1n - a1i) * f.rh - (a3i + a4i * (1.0 / 3.0) * f.h) * 0.5 * f.h;
    pc.c3 = a3i;
    pc.c4 = a4i;
}

// ppvalu (pppack.f90:4246-4362) of the fit at x; the piece is kept in
// registers between calls (consecutive sub-step positions mostly share it).
template <class W>
__device__ __forceinline__ double m_ppvalu(const W& w, const MFit& f, double p, double x, int jderiv,
                                           MPiece& pc) {
    const int np = f.np;
    // interv on uniform breaks: piece 1 below the first break, np-1 at or
    // above the last (also for a NaN x)
    const double t = floor((x - f.z1) * f.rh);
    const int i = (t >= 0.0 && t < (double)(np - 1)) ? (int)t + 1 : ((t >= (double)(np - 1)) ? np - 1 : 1);
    if (i != pc.i) m_piece(w, f, p, i, pc);
    const double hx = x - pc.xi;
    // Horner loop of ppvalu with k = 4: value = (value/fmmjdr)*h + coef(m)
    if (jderiv == 0) return ((pc.c4 * (1.0 / 3.0) * hx + pc.c3) * 0.5 * hx + pc.c2) * hx + pc.c1;
    return (pc.c4 * 0.5 * hx + pc.c3) * hx + pc.c2;
}

// Normal deviates d and d+1 (d even) of a particle-step: the noise hook's
// values when set, else the two Box-Muller deviates (cosine branch,
// pdf_module.f90:26-40) of one Philox4x32-10 call at counter (pid, step,
// d/2) -- the exact form's uniforms -- with the transform in FP32 (logf,
// cospif: the deviates agree with the exact form's to about 1e-6).
__device__ __forceinline__ void m_normal2(const RpStepArgs& A, uint32_t pid, uint32_t d, double& n0, double& n1) {
    if (A.hook) {
        const double* h = A.hook + (int64_t)(pid - A.pid_base) * A.ndraw + d;
        n0 = h[0];
        n1 = (d + 1 < (uint32_t)(2 + A.loop)) ? h[1] : 0.0;   // past the last sub-step: not read
        return;
    }
    uint32_t c[4] = {pid, (uint32_t)A.step_index, (uint32_t)(A.step_index >> 32), d >> 1};
    rp_philox(c, (uint32_t)A.seed, (uint32_t)(A.seed >> 32));
    const float k = 2.3283064365386963e-10f;     // 2^-32
    const float r0 = sqrtf(-2.f * logf(((float)c[0] + 0.5f) * k));
    const float r1 = sqrtf(-2.f * logf(((float)c[2] + 0.5f) * k));
    n0 = (double)(r0 * cospif(2.f * (((float)c[1] + 0.5f) * k)));
    n1 = (double)(r1 * cospif(2.f * (((float)c[3] + 0.5f) * k)));
}

// VTurb (ver_turb_module.f90:31-329): column in FP32 from the 16-bit AKs,
// the fit as m_smooth / m_chol1d form it, random-displacement sub-steps in
// FP64
template <typename E, class W>
__device__ float m_vturb(const RpStepArgs& A, const RpGridDev& g, const MStage& S, float Zpar,
                         uint32_t pid, double& qstate, double& gstate, float& q2state, uint32_t& fl, const W& w) {
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
    const uint2* aks = reinterpret_cast<const uint2*>(g.aks);
    const float4* qs = reinterpret_cast<const float4*>(g.qs_aks);
    const MTime tk = m_time(A, g, 0);
    const bool all[4] = {true, true, true, true};
    float zprev = 0.f, kprev = 0.f;
    // levels in batches of kColBatch: the batch's 4 kColBatch corner loads
    // are issued before any is used, so their latencies overlap (a
    // workspace view for a kernel with registers to spare asks for more)
    constexpr int kColBatch = W::kColBatch;
    for (int k0 = 1; k0 <= sw; k0 += kColBatch) {
        uint2 v[kColBatch][4];
        float4 sc[kColBatch];
#pragma unroll
        for (int b = 0; b < kColBatch; b++) {
            const int k = min(k0 + b, sw);
            sc[b] = __ldg(qs + k - 1);
#pragma unroll
            for (int q = 0; q < 4; q++) v[b][q] = __ldg(aks + S.rc.o[q] * sw + k - 1);
        }
#pragma unroll
        for (int b = 0; b < kColBatch; b++) {
            const int k = k0 + b;
            if (k > sw) break;
            // z_w(k) of the interpolated zeta (getWlevel is linear in zeta)
            const float2 scs = __ldg(g.scs_w + k - 1);
            const float zk = (k == sw) ? S.zeta : m_zlev(g.vtransform, hc, h, den_r, scs.x, scs.y, S.zeta);
            const float kk = m_level_of<E>(v[b], sc[b], cwt, all, tk);   // getInterpAKs
            w.cz(k) = zk;
            if (k >= 2) {
                const float m = (kk - kprev) / (zk - zprev);
                w.cm(k - 1) = m;
                w.cb(k - 1) = kprev - m * zprev;
            }
            zprev = zk;
            kprev = kk;
        }
    }
    f.z1 = w.cz(1);
    f.h = (zeta - f.z1) / (double)(f.np - 1);
    f.rh = 1.0 / f.h;
    int passes;
    const double p = m_smooth(w, f, A.smth, A.spline_max_iter, qstate, gstate, q2state, fl, passes);
    if (A.spl) rp_count_fit(A.spl, passes);
    const double deltat = A.deltat;
    double ParZc = (double)Zpar;
    MPiece pc;
    pc.i = 0;
    double dev_next = 0.0;
    for (int i = 1; i <= A.loop; i++) {
        double DEV;                                    // draw 1+i; pairs (2,3), (4,5), ...
        if (i & 1) m_normal2(A, pid, (uint32_t)(1 + i), DEV, dev_next);
        else DEV = dev_next;
        double Kprimec = 0.0;
        if (!(ParZc <= tdepth || ParZc >= zeta)) Kprimec = m_ppvalu(w, f, p, ParZc, 1, pc);
        const double KprimeZc = Kprimec * deltat;
        const double Z3rdc = ParZc + 0.5 * KprimeZc;
        double KH3rdc;
        if (Z3rdc < tdepth || Z3rdc > zeta) {
            KH3rdc = A.aksback;
        } else {
            KH3rdc = m_ppvalu(w, f, p, Z3rdc, 0, pc);
            if (KH3rdc < A.aksback) KH3rdc = A.aksback;
        }
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

// ------------------------------------------------------- diagnostics

// A field stored as FP32 for the four ring slots of each (point, level)
// (the diagnostics' fields in this form): value at level lev of the corner
// set, time-interpolated with the slot weights.
__device__ __forceinline__ float m_f32_level(const float4* f, const MOff o[4], const float cff[4],
                                             const bool use[4], int nlev, int lev, const MTime& t) {
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (use[q]) {
            const float4 v = m_live4(__ldg(f + o[q] * nlev + lev - 1), t.m32);
            acc += cff[q] * fmaf(t.w4.w, v.w, fmaf(t.w4.z, v.z, fmaf(t.w4.y, v.y, t.w4.x * v.x)));
        }
    }
    return acc;
}

// Each ring slot's rho weights of a cell under WETDRY, formed once for all
// the fields gathered there
struct MRhoWD {
    float cff[3][4];               // slots b, c, f
};

__device__ __forceinline__ void m_rho_wd_all(const RpGridDev& g, const MRho& c, const MTime& t, MRhoWD& wd,
                                             uint32_t& fl) {
    const int sl[3] = {t.sb, t.sc, t.sf};
    for (int q = 0; q < 3; q++) m_rho_wd_cff(g, c, sl[q], wd.cff[q], fl);
}

// A field held in FP32 on a rho corner set, levels L, time-interpolated;
// under WETDRY (wd set) each slot with its own weights
__device__ __forceinline__ float m_f32_col(const RpStepArgs& A, const RpGridDev& g, const void* fv, const MRho& c,
                                           int nlev, const MPick& L, const MTime& t, const MRhoWD* wd) {
    const float4* f = reinterpret_cast<const float4*>(fv);
    const bool all[4] = {true, true, true, true};
    if (!wd) {
        const float* cw = c.wet4 ? c.cb : c.ci;
        const float vb = m_f32_level(f, c.o, cw, all, nlev, L.ibot, t);
        const float vt = (L.itop == L.ibot) ? vb : m_f32_level(f, c.o, cw, all, nlev, L.itop, t);
        return L.z1 * vb + L.z2 * vt;
    }
    const float wt[3] = {t.wb, t.wc, t.wf};
    const int sl[3] = {t.sb, t.sc, t.sf};
    float acc = 0.f;
    for (int q = 0; q < 3; q++) {
        if (wt[q] == 0.f) continue;
        const float* cw = wd->cff[q];
        float lv[2];
        for (int h = 0; h < 2; h++) {
            const int lev = h ? L.itop : L.ibot;
            float a = 0.f;
#pragma unroll
            for (int k = 0; k < 4; k++) a += cw[k] * m_pick4(__ldg(f + c.o[k] * nlev + lev - 1), sl[q]);
            lv[h] = a;
        }
        acc += wt[q] * (L.z1 * lv[0] + L.z2 * lv[1]);
    }
    return acc;
}

// A field held in FP32 on the u or v corner set (one level), time-
// interpolated; under WETDRY each slot with its own masks
__device__ __forceinline__ float m_f32_uv(const RpStepArgs& A, const RpGridDev& g, const void* fv, float X, float Y,
                                          bool is_u, const MTime& t, uint32_t& fl) {
    const float4* f = reinterpret_cast<const float4*>(fv);
    MUV c;
    if (!A.wetdry) {
        m_uv_cell(g, X, Y, is_u, c, fl);
        return m_f32_level(f, c.o, c.cff, c.use, 1, 1, t);
    }
    const float wt[3] = {t.wb, t.wc, t.wf};
    const int sl[3] = {t.sb, t.sc, t.sf};
    float acc = 0.f;
    for (int q = 0; q < 3; q++) {
        if (wt[q] == 0.f) continue;
        m_uv_cell(g, X, Y, is_u, c, fl, is_u ? g.wd_u : g.wd_v, RP_SLOTS, sl[q]);
        float a = 0.f;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (c.use[k]) a += c.cff[k] * m_pick4(__ldg(f + c.o[k]), sl[q]);
        acc += wt[q] * a;
    }
    return acc;
}

// The diagnostics that close update_particles' particle loop
// (ROMSPath.f90:935-986) in this form: at the particle's new position and
// grid, with the step's tdepth; the bottom stress on the u / v corner sets
// (getInterpStr's rules) and salt / temp on the rho levels bracketing z at
// the time-interpolated zeta (as u and v are here), the b, c, f slots
// folded as Lagrange weights.  Out of line: the step keeps its registers
// when the diagnostics are off.
__device__ __noinline__ void m_diag_one(const RpStepArgs& A, int64_t n, float tdepth, uint32_t& fl) {
    const RpParticlesDev& P = A.p;
    const RpGridDev& g = A.g[P.gid[n] - 1];
    const float X = P.x32[n] - P.cx[n], Y = P.y32[n] - P.cy[n], Z = P.z32[n] - P.cz[n];
    const MTime t = m_time(A, g, 0);
    if (A.diag & RP_DIAG_BOTTOM_D) {                       // 935-952
        const double btemp = -1.0 * (double)tdepth + (double)Z;
        const double hob0 = P.hob[n];
        const double hob = (btemp < hob0) ? btemp : hob0;
        P.hob[n] = hob;
        if (btemp == hob) {
            P.bustr[n] = (double)m_f32_uv(A, g, g.bustr, X, Y, true, t, fl);
            P.bvstr[n] = (double)m_f32_uv(A, g, g.bvstr, X, Y, false, t, fl);
        }
    }
    if (A.diag & RP_DIAG_SALTTEMP_D) {                     // 962-986
        MRho c;
        m_rho_cell(g, X, Y, c, fl);
        const float zeta = m_zeta(g, c, t);
        MPick Lr, Lw;
        uint32_t wfl = 0;                                  // the w bracket is not used here
        m_walk2(g, zeta, tdepth, Z, Lr, Lw, wfl);
        MRhoWD wd;
        if (A.wetdry) m_rho_wd_all(g, c, t, wd, fl);
        const MRhoWD* pw = A.wetdry ? &wd : nullptr;
        const double s = (double)m_f32_col(A, g, g.salt, c, g.N, Lr, t, pw);
        const double tp = (double)m_f32_col(A, g, g.temp, c, g.N, Lr, t, pw);
        P.salt[n] = s;
        P.temp[n] = tp;
        if (A.diag & RP_DIAG_MEAN_D) {
            P.mean_salt[n] = P.mean_salt[n] + s;
            P.mean_temp[n] = P.mean_temp[n] + tp;
        }
    }
}

// behave (behavior_module.f90:186-393) in this form: its four fields held
// in FP32, gathered at the start position's rho cell on the w levels that
// bracket Zpar at the time-interpolated zeta (as w is here), the slots
// folded as Lagrange weights; then the response the exact form uses (FP64,
// own exp/log, the same draws).  Out of line, as the diagnostics.
__device__ __noinline__ double m_behave(const RpStepArgs& A, int64_t n, const RpGridDev& g, float Xpar, float Ypar,
                                        float Zpar, uint32_t pid, uint32_t& fl) {
    const RpBehaviorDev& b = A.beh;
    double wb = 0.0;
    if (b.va || b.wa) {
        MRho c;
        m_rho_cell(g, Xpar, Ypar, c, fl);
        const MTime t = m_time(A, g, 0);
        const float depth = -c.hb;
        const float zeta = m_zeta(g, c, t);
        MPick Lr, Lw;
        m_walk2(g, zeta, depth, Zpar, Lr, Lw, fl);
        const int nl = g.N + 1;
        MRhoWD wd;
        if (A.wetdry) m_rho_wd_all(g, c, t, wd, fl);
        const MRhoWD* pw = A.wetdry ? &wd : nullptr;
        auto col = [&](const void* f) -> double { return (double)m_f32_col(A, g, f, c, nl, Lw, t, pw); };
        double sa = 0.0, sv = 0.0, su = 0.0, sw = 0.0;
        if (b.va) {
            sa = RP_MUL(col(g.turbaccel), 100.0);
            sv = col(g.turbvort);
        }
        if (b.wa) {
            su = RP_MUL(col(g.waveaccelu), 100.0);
            sw = RP_MUL(col(g.waveaccelv), 100.0);
        }
        wb = rp_behave_swim(A, n, pid, sa, sv, su, sw);
    }
    return rp_behave_z(A, wb);
}

// ----------------------------------------------------------- one particle

// VTurb of one particle on its own (the first kernel of the split form),
// with the stage-1 z clamp of find_currents applied first when RK4 runs
// (advection_module.f90:171-183), as RKAdvect hands Zpar to VTurb.
template <typename E, class W>
__device__ void m_vturb_one(const RpStepArgs& A, int64_t n, const W& w, float* turbv) {
    const RpParticlesDev& Pt = A.p;
    if (!rp_active(A, n)) return;
    uint32_t fl = 0;
    const int gid = Pt.gid[n];
    const RpGridDev& g = A.g[gid - 1];
    const float Xpar = Pt.x32[n], Ypar = Pt.y32[n];
    float Zpar = Pt.z32[n] - Pt.cz[n];
    MStage S1;
    m_rho_cell(g, Xpar, Ypar, S1.rc, fl);
    m_stage_2d(m_time(A, g, 0), g, S1);
    if (A.scheme == 1) {
        if (Zpar < S1.tdepth) Zpar = S1.tdepth + 0.001f;
        if (Zpar > S1.zeta) Zpar = S1.zeta - 0.001f;
    }
    double q = Pt.qwarm[n], gs = Pt.gwarm[n];
    float q2 = Pt.qwarm2[n];
    turbv[n] = m_vturb<E>(A, g, S1, Zpar, Pt.pid[n], q, gs, q2, fl, w);
    Pt.qwarm[n] = q;
    Pt.gwarm[n] = gs;
    Pt.qwarm2[n] = m_stencil_moved(A) ? -1.f : q2;
    if (fl) Pt.flags[n] |= fl;
}

// One particle of update_particles in the mixed form.  With turbv_in
// non-null the VTurb displacement comes from the split form's first kernel.
// FEAT: the kernel variant with the options beyond the passive step (the
// diagnostics, WETDRY, behave); the passive variant carries none of their
// code.
template <typename E, bool FEAT, class W>
__device__ void m_update_one(const RpStepArgs& A, int64_t n, const W& w, const float* turbv_in) {
    const RpParticlesDev& Pt = A.p;
    if (!rp_active(A, n)) return;
    Pt.age[n] = Pt.age[n] + (double)(float)A.idt;
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
            float xs = Xpar, ys = Ypar, zs = Zpar;
            if (st > 0) {
                xs = Xpar + kx * half_dt;
                ys = Ypar + ky * half_dt;
                zs = Zpar + kz * half_dt;
            }
            m_find_currents<E, FEAT>(A, g, xs, ys, zs, U, V, Wv, fl);
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
    if (A.vturb_on && !turbv_in) {
        m_rho_cell(g, Xpar, Ypar, S1.rc, fl);
        m_stage_2d(m_time(A, g, 0), g, S1);
    }
    float TurbHx = 0.f, TurbHy = 0.f;
    if (A.hturb_on) {                                  // HTurb, hor_turb_module.f90:30-51
        const float sc = sqrtf(2.f * (float)A.khturb[gid - 1] * didt);
        double nx, ny;
        m_normal2(A, pid, 0u, nx, ny);
        TurbHx = (float)nx * sc;
        TurbHy = (float)ny * sc;
    }
    TurbHx *= pm;
    TurbHy *= pn;
    float TurbV = 0.f;
    if (A.vturb_on && turbv_in) {
        TurbV = turbv_in[n];
    } else if (A.vturb_on) {
        double q = Pt.qwarm[n], gs = Pt.gwarm[n];
        float q2 = Pt.qwarm2[n];
        TurbV = m_vturb<E>(A, g, S1, Zpar, pid, q, gs, q2, fl, w);
        Pt.qwarm[n] = q;
        Pt.gwarm[n] = gs;
        Pt.qwarm2[n] = m_stencil_moved(A) ? -1.f : q2;
    }
    float ZBehav = 0.f;                                // behave(), ROMSPath.f90:800-804
    if (FEAT && (A.beh.behavior || A.beh.va || A.beh.wa))
        ZBehav = A.beh_z[n];                           // from the behave pass before the step
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
    const float tdepth = -rn.hb;
    const float P_zeta = m_zeta(gn, rn, m_time(A, gn, 0));
    Pt.wd[n] = (double)(-tdepth + P_zeta);
    Pt.zeta[n] = (double)P_zeta;
    Pt.bath[n] = (double)(-tdepth);
    bool hbot = false, htop = false;
    float nz = z, ncz = cz;
    if (A.nsb == 0) {
        m_kahan_add(nz, ncz, AdvectZ + TurbV + ZBehav);
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
    if (FEAT && A.diag) A.diag_td[n] = tdepth;        // the diagnostics run in their own pass
    if (fl) Pt.flags[n] |= fl;
}
