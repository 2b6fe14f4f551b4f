/*
 * romspath_oracle.c -- CPU FP64 restatement of the ROMSPath particle step.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA path and the
 * timed CPU baseline.  Nothing in the product links or calls it.
 *
 * PARITY STATUS: parity unpinned against the reference binary (Fortran +
 * NetCDF, no tests, no compiler here).  Pinned by MT19937 known answers and
 * analytic invariants only; see romspath_oracle.h.
 *
 * Every function restates the reference routine whose file:line it cites
 * (paths relative to the ROMSPath source tree), keeping the reference's
 * evaluation order.  Where the reference reads out of bounds or divides
 * 0/0, the pinned behaviour is stated at the site and a flag bit is set.
 */
#include "romspath_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Fortran column-major, 1-based */
#define IX2(i, j, ni) ((int64_t)((i) - 1) + (int64_t)((j) - 1) * (int64_t)(ni))
#define IX3(i, j, k, ni, nj) \
    ((int64_t)((i) - 1) + (int64_t)(ni) * ((int64_t)((j) - 1) + (int64_t)(nj) * (int64_t)((k) - 1)))

/* Fortran single-precision literals widened to double by DBLE()/assignment:
 * DBLE(0.001) in advection_module.f90:174,182; ecut=0.1 in
 * boundary_module.f90:59; status 1.1 / 1.2 in ROMSPath.f90:882-883. */
#define F_0P001 ((double)0.001f)
#define F_0P1 ((double)0.1f)
#define F_1P1 ((double)1.1f)
#define F_1P2 ((double)1.2f)
#define PI_D 3.14159265358979323846 /* ROMSPath.h:11 */

static int64_t g_spline_calls, g_secant_iters;

void orc_last_stats(int64_t *spline_calls, int64_t *secant_iters)
{
    *spline_calls = g_spline_calls;
    *secant_iters = g_secant_iters;
}

/* floor() to int with NaN / overflow made defined (reference: floor() of a
 * finite in-range double). */
static inline int ifloor(double x)
{
    double f = floor(x);
    if (!(f >= -1.0e9)) return -1000000000;
    if (f > 1.0e9) return 1000000000;
    return (int)f;
}

/* Pinned out-of-range read: the index is clamped into the array and
 * ORC_FLAG_OOB is set (the reference reads past the array). */
static inline int clampi(int v, int lo, int hi, uint32_t *flags)
{
    if (v < lo) { *flags |= ORC_FLAG_OOB; return lo; }
    if (v > hi) { *flags |= ORC_FLAG_OOB; return hi; }
    return v;
}

/* ======================= random numbers ======================= */

/* init_genrand, random_module.f90:109-121 */
void orc_mt_init(orc_mt19937 *s, uint32_t seed)
{
    s->mt[0] = seed;
    for (int i = 1; i < 624; i++)
        s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->mti = 624;
}

/* genrand_int32, random_module.f90:167-198 (N=624, M=397) */
uint32_t orc_mt_int32(orc_mt19937 *s)
{
    const uint32_t UPPER = 0x80000000u, LOWER = 0x7fffffffu, MATA = 0x9908b0dfu;
    uint32_t y;
    if (s->mti >= 624) {
        int kk;
        for (kk = 0; kk < 624 - 397; kk++) {
            y = (s->mt[kk] & UPPER) | (s->mt[kk + 1] & LOWER);
            s->mt[kk] = s->mt[kk + 397] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
        }
        for (; kk < 623; kk++) {
            y = (s->mt[kk] & UPPER) | (s->mt[kk + 1] & LOWER);
            s->mt[kk] = s->mt[kk + (397 - 624)] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
        }
        y = (s->mt[623] & UPPER) | (s->mt[0] & LOWER);
        s->mt[623] = s->mt[396] ^ (y >> 1) ^ ((y & 1u) ? MATA : 0u);
        s->mti = 0;
    }
    y = s->mt[s->mti++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
}

/* genrand_real3, random_module.f90:240-247: (r + 0.5) / 2^32 in (0,1) */
double orc_mt_real3(orc_mt19937 *s)
{
    double r = (double)orc_mt_int32(s);
    return (r + 0.5) / 4294967296.0;
}

/* norm(), pdf_module.f90:26-40: Box-Muller, cosine branch only */
static double box_muller(double dev1, double dev2)
{
    return sqrt(-2.0 * log(dev1)) * cos(2.0 * PI_D * dev2);
}

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), the counter-based
 * generator that replaces the serial MT19937 stream on the device. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Natural log of a positive normal double and cos(2 pi u) on [0,1] from
 * their Taylor series with exact argument reductions (see
 * orc_log_pos / orc_cos2pi).  The device path uses the same operation
 * sequence, so Philox-driven normals are bit-identical on both sides. */
#define ORC_LN2_HI 0.6931471805599453
#define ORC_LN2_LO 2.3190468138462996e-17
#define ORC_SQRT2 1.4142135623730951
#define ORC_TWOPI_HI 6.283185307179586
#define ORC_TWOPI_LO 2.4492935982947064e-16

double orc_log_pos(double x)
{
    uint64_t b;
    memcpy(&b, &x, 8);
    int e = (int)((b >> 52) & 0x7ffu) - 1023;
    uint64_t mb = (b & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
    double m;
    memcpy(&m, &mb, 8);
    if (m > ORC_SQRT2) { m = m * 0.5; e = e + 1; }
    const double z = (m - 1.0) / (m + 1.0);
    const double z2 = z * z;
    double p = 1.0 / 23.0;
    p = p * z2 + 1.0 / 21.0;
    p = p * z2 + 1.0 / 19.0;
    p = p * z2 + 1.0 / 17.0;
    p = p * z2 + 1.0 / 15.0;
    p = p * z2 + 1.0 / 13.0;
    p = p * z2 + 1.0 / 11.0;
    p = p * z2 + 1.0 / 9.0;
    p = p * z2 + 1.0 / 7.0;
    p = p * z2 + 1.0 / 5.0;
    p = p * z2 + 1.0 / 3.0;
    p = p * z2 + 1.0;
    const double de = (double)e;
    return de * ORC_LN2_HI + (de * ORC_LN2_LO + 2.0 * z * p);
}

double orc_cos2pi(double u)
{
    double v = (u > 0.5) ? 1.0 - u : u;
    double sign = 1.0, r;
    if (v > 0.25) { v = 0.5 - v; sign = -1.0; }
    if (v <= 0.125) {
        const double x = v * ORC_TWOPI_HI + v * ORC_TWOPI_LO;
        const double x2 = x * x;
        double p = 1.0 / 2432902008176640000.0;
        p = p * x2 - 1.0 / 6402373705728000.0;
        p = p * x2 + 1.0 / 20922789888000.0;
        p = p * x2 - 1.0 / 87178291200.0;
        p = p * x2 + 1.0 / 479001600.0;
        p = p * x2 - 1.0 / 3628800.0;
        p = p * x2 + 1.0 / 40320.0;
        p = p * x2 - 1.0 / 720.0;
        p = p * x2 + 1.0 / 24.0;
        p = p * x2 - 0.5;
        r = p * x2 + 1.0;
    } else {
        const double w = 0.25 - v;
        const double x = w * ORC_TWOPI_HI + w * ORC_TWOPI_LO;
        const double x2 = x * x;
        double p = 1.0 / 121645100408832000.0;
        p = p * x2 - 1.0 / 355687428096000.0;
        p = p * x2 + 1.0 / 1307674368000.0;
        p = p * x2 - 1.0 / 6227020800.0;
        p = p * x2 + 1.0 / 39916800.0;
        p = p * x2 - 1.0 / 362880.0;
        p = p * x2 + 1.0 / 5040.0;
        p = p * x2 - 1.0 / 120.0;
        p = p * x2 + 1.0 / 6.0;
        p = p * x2;
        r = x - x * p;
    }
    return sign * r;
}

/* Normal deviate number `draw` of particle `pid` at internal step `step`:
 * counter (pid, step_lo, step_hi, draw/2), key = seed; two uniforms per
 * normal, mapped like genrand_real3, then norm()'s Box-Muller. */
double orc_philox_normal(uint64_t seed, uint32_t pid, uint64_t step, uint32_t draw)
{
    uint32_t ctr[4] = {pid, (uint32_t)step, (uint32_t)(step >> 32), draw >> 1};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    int w = (int)(draw & 1u) * 2;
    double u1 = ((double)o[w] + 0.5) / 4294967296.0;
    double u2 = ((double)o[w + 1] + 0.5) / 4294967296.0;
    return sqrt(-2.0 * orc_log_pos(u1)) * orc_cos2pi(u2);
}

/* exp: x = k ln2 + r with |r| <= ln2/2 (k ln2 split so k * hi is exact),
 * exp(r) by its Taylor series to r^13/13!, then 2^k in two factors. */
#define ORC_LN2E_HI 0x1.62e42fee00000p-1    /* ln2 truncated to 32 bits */
#define ORC_LN2E_LO 0x1.a39ef35793c76p-33   /* ln2 - ORC_LN2E_HI */
#define ORC_INV_LN2 1.4426950408889634

static double pow2i(int m)                  /* 2^m, -1022 <= m <= 1023 */
{
    uint64_t b = (uint64_t)(m + 1023) << 52;
    double r;
    memcpy(&r, &b, 8);
    return r;
}

double orc_exp(double x)
{
    if (x != x) return x;
    if (x > 709.782712893384) return INFINITY;
    if (x < -745.1332191019412) return 0.0;
    const double k = rint(x * ORC_INV_LN2);
    const double r = (x - k * ORC_LN2E_HI) - k * ORC_LN2E_LO;
    double p = 1.0 / 6227020800.0;                 /* 1/13! */
    p = p * r + 1.0 / 479001600.0;                 /* 1/12! */
    p = p * r + 1.0 / 39916800.0;
    p = p * r + 1.0 / 3628800.0;
    p = p * r + 1.0 / 362880.0;
    p = p * r + 1.0 / 40320.0;
    p = p * r + 1.0 / 5040.0;
    p = p * r + 1.0 / 720.0;
    p = p * r + 1.0 / 120.0;
    p = p * r + 1.0 / 24.0;
    p = p * r + 1.0 / 6.0;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    const int ki = (int)k, k1 = ki / 2, k2 = ki - k1;
    return (p * pow2i(k1)) * pow2i(k2);
}

double orc_log(double x)
{
    if (x != x || x < 0.0) return NAN;
    if (x == 0.0) return -INFINITY;
    if (x == INFINITY) return x;
    if (x < 0x1p-1022)                              /* subnormal: scale by 2^54 */
        return orc_log_pos(x * 0x1p54) - 54.0 * ORC_LN2_HI - 54.0 * ORC_LN2_LO;
    return orc_log_pos(x);
}

double orc_philox_uniform(uint64_t seed, uint32_t pid, uint64_t step, uint32_t k)
{
    uint32_t ctr[4] = {pid, (uint32_t)step, (uint32_t)(step >> 32), 0x40000000u + (k >> 2)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    return ((double)o[k & 3u] + 0.5) / 4294967296.0;
}

typedef struct {
    const orc_noise *nz;
    uint32_t pid;
} noise_ctx;

static double draw_normal(const noise_ctx *c, uint32_t d)
{
    const orc_noise *nz = c->nz;
    switch (nz->kind) {
    case ORC_NOISE_MT: {
        double dev1 = orc_mt_real3(nz->mt);
        double dev2 = orc_mt_real3(nz->mt);
        return box_muller(dev1, dev2);
    }
    case ORC_NOISE_PHILOX:
        return orc_philox_normal(nz->seed, c->pid, nz->step, d);
    default:
        return nz->hook[(int64_t)c->pid * nz->ndraw + d];
    }
}

/* Uniform k (0..4) of behave: genrand_real3 from the one stream, the
 * Philox uniform, or the hook's entry d0 + 2 + k (d0 = first behave draw). */
static double draw_uniform(const noise_ctx *c, uint32_t d0, uint32_t k)
{
    const orc_noise *nz = c->nz;
    switch (nz->kind) {
    case ORC_NOISE_MT:
        return orc_mt_real3(nz->mt);
    case ORC_NOISE_PHILOX:
        return orc_philox_uniform(nz->seed, c->pid, nz->step, k);
    default:
        return nz->hook[(int64_t)c->pid * nz->ndraw + d0 + 2 + k];
    }
}

/* laplace (pdf_module.f90:42-55) of one uniform */
static double laplace_of(double u)
{
    const double dev1 = u - 0.5;
    const double dev2 = -1.0 * orc_log(1.0 - (2.0 * fabs(dev1))) / sqrt(2.0);
    const double mag = fabs(dev2);
    return (dev1 >= 0.0) ? mag : -mag;                          /* sign(dev2, dev1) */
}

/* ======================= interpolation ======================= */

/* polintd, interpolation_module.f90:72-109 */
double orc_polintd(const double xa[3], const double ya[3], double x)
{
    int ns = 0;
    double dif = fabs(x - xa[0]);
    for (int i = 0; i < 3; i++) {
        double dift = fabs(x - xa[i]);
        if (dift < dif) { ns = i; dif = dift; }
    }
    double c = (xa[1] - x) * ((ya[2] - ya[1]) / (xa[1] - xa[2]));
    c = c - (xa[1] - x) * ((ya[1] - ya[0]) / (xa[0] - xa[1]));
    c = c / (xa[0] - xa[2]);
    double a, b;
    if (ns == 2) {
        a = (ya[2] - ya[1]) / (xa[1] - xa[2]);
        b = xa[2] - x;
    } else {
        a = (ya[1] - ya[0]) / (xa[0] - xa[1]);
        b = xa[0] - x;
    }
    return ya[ns] + (xa[ns] - x) * a + b * c;
}

/* linint, interpolation_module.f90:27-61 (xa, ya 1-based via pointer-1) */
void orc_linint(const double *xa, const double *ya, int n, double x, double *y, double *m)
{
    int jlo = 1, jhi = n, k;
    xa -= 1; ya -= 1;
    for (;;) {
        k = (jhi + jlo) / 2;
        if (xa[k] > x) jhi = k; else jlo = k;
        if (jhi - jlo == 1) break;
    }
    double mm = (ya[jlo] - ya[jhi]) / (xa[jlo] - xa[jhi]);
    double b = ya[jlo] - mm * xa[jlo];
    *y = mm * x + b;
    *m = mm;
}

/* getSlevel, grid_module.f90:513-555 */
double orc_getslevel(const orc_grid *g, double zeta, double depth, int k)
{
    double h = -1.0 * depth, S;
    double s = g->s_rho[k - 1], cs = g->cs_r[k - 1];
    switch (g->vtransform) {
    case 1:
        S = g->hc * s + (h - g->hc) * cs;
        return S + zeta * (1.0 + S / h);
    case 2:
        S = (g->hc * s + h * cs) / (g->hc + h);
        return zeta + (zeta + h) * S;
    default:
        return zeta * (1.0 + s) + g->hc * s + (h - g->hc) * cs;
    }
}

/* getWlevel, grid_module.f90:557-598 */
double orc_getwlevel(const orc_grid *g, double zeta, double depth, int k)
{
    double h = -1.0 * depth, S;
    double s = g->s_w[k - 1], cs = g->cs_w[k - 1];
    switch (g->vtransform) {
    case 1:
        S = g->hc * s + (h - g->hc) * cs;
        return S + zeta * (1.0 + S / h);
    case 2:
        S = (g->hc * s + h * cs) / (g->hc + h);
        return zeta + (zeta + h) * S;
    default:
        return zeta * (1.0 + s) + g->hc * s + (h - g->hc) * cs;
    }
}

/* getcoeff, interpolation_module.f90:1230-1273: inverse-distance weights
 * over wet corners.  Pinned: at an exact node (dist = 0) the reference
 * computes m/0 and 0/0 (NaN); here a wet node takes weight 1 and a dry node
 * weight 0 (the limit as the point approaches the node). */
static void getcoeff(double X, double Y, const double m[4], double cff[4], uint32_t *flags)
{
    double dist[4], W[4], WT;
    dist[0] = sqrt(X * X + Y * Y);
    dist[1] = sqrt((1 - X) * (1 - X) + Y * Y);
    dist[2] = sqrt((1 - X) * (1 - X) + (1 - Y) * (1 - Y));
    dist[3] = sqrt(X * X + (1 - Y) * (1 - Y));
    for (int k = 0; k < 4; k++) {
        if (dist[k] == 0.0) {
            *flags |= ORC_FLAG_NODE;
            if (m[k] != 0.0) {
                for (int q = 0; q < 4; q++) cff[q] = (q == k) ? 1.0 : 0.0;
                return;
            }
            W[k] = 0.0;
        } else {
            W[k] = m[k] / dist[k];
        }
    }
    WT = W[0] + W[1] + W[2] + W[3];
    if (WT == 0.0) {
        for (int k = 0; k < 4; k++) cff[k] = 0.0;
    } else {
        for (int k = 0; k < 4; k++) cff[k] = W[k] / WT;
    }
}

/* getInterp2D, interpolation_module.f90:421-507 (depth, pm, pn, zeta) */
double orc_getinterp2d(const orc_grid *g, int var, double ipar, double jpar, int t, uint32_t *flags)
{
    const int nx = g->xi_rho, ny = g->eta_rho;
    int I = ifloor(ipar), J = ifloor(jpar);
    double X = ipar - (double)I, Y = jpar - (double)J;
    int i0 = clampi(I, 1, nx, flags), i1 = clampi(I + 1, 1, nx, flags);
    int j0 = clampi(J, 1, ny, flags), j1 = clampi(J + 1, 1, ny, flags);
    double m[4], v[4], cff[4];
    m[0] = g->mask_rho[IX2(i0, j0, nx)];
    m[1] = g->mask_rho[IX2(i1, j0, nx)];
    m[2] = g->mask_rho[IX2(i1, j1, nx)];
    m[3] = g->mask_rho[IX2(i0, j1, nx)];
    cff[0] = (1 - X) * (1 - Y);
    cff[1] = X * (1 - Y);
    cff[2] = X * Y;
    cff[3] = (1 - X) * Y;
    const double *a;
    switch (var) {
    case ORC_V_DEPTH: a = g->h; break;
    case ORC_V_PM: a = g->pm; break;
    case ORC_V_PN: a = g->pn; break;
    case ORC_V_LON: a = g->lon_rho; break;                   /* 466-472 */
    case ORC_V_LAT: a = g->lat_rho; break;                   /* 473-477 */
    default: a = g->zeta[t - 1]; break;
    }
    v[0] = a[IX2(i0, j0, nx)];
    v[1] = a[IX2(i1, j0, nx)];
    v[2] = a[IX2(i1, j1, nx)];
    v[3] = a[IX2(i0, j1, nx)];
    if (var == ORC_V_ZETA) getcoeff(X, Y, m, cff, flags);
    return cff[0] * v[0] + cff[1] * v[1] + cff[2] * v[2] + cff[3] * v[3];
}

/* The mask getInterp3D / getInterpStr read: the frame's wetdry mask under
 * WETDRY (interpolation_module.f90:628-671 and the like), else the grid's. */
static double mk_u(const orc_grid *g, int t, int idx) { return g->wd_u[t - 1] ? g->wd_u[t - 1][idx] : (double)g->mask_u[idx]; }
static double mk_v(const orc_grid *g, int t, int idx) { return g->wd_v[t - 1] ? g->wd_v[t - 1][idx] : (double)g->mask_v[idx]; }
static double mk_r(const orc_grid *g, int t, int idx) { return g->wd_rho[t - 1] ? g->wd_rho[t - 1][idx] : (double)g->mask_rho[idx]; }

/* getInterp3D, interpolation_module.f90:509-962 (u, v, w, AKs).  The full
 * column profile is formed as in the reference, then two levels blended. */
double orc_getinterp3d(const orc_grid *g, int var, double ipar, double jpar, double zpar,
                       int t, int ztype, double zeta, double depth, uint32_t *flags)
{
    const int nx = g->xi_rho, ny = g->eta_rho, N = g->N;
    int nz, Itop, Ibot, i;
    double zlev1 = 0.0, zlev2 = 0.0, zcff1, zcff2, Z;

    if (ztype == 1) {
        /* interpolation_module.f90:529-558 */
        nz = N; Itop = nz; Ibot = nz;
        for (i = 1; i <= nz; i++) {
            zlev2 = orc_getslevel(g, zeta, depth, i);
            if (zlev2 > zpar) {
                Itop = i; Ibot = i - 1;
                zlev1 = (i == 1) ? depth : orc_getslevel(g, zeta, depth, i - 1);
                break;
            }
        }
        if (i > nz) {
            Itop = nz; Ibot = nz; zcff1 = 0.5; zcff2 = 0.5;
        } else if (Itop == 1) {
            Itop = 1; Ibot = 1; zcff1 = 0.5; zcff2 = 0.5;
        } else {
            Z = (zpar - zlev1) / (zlev2 - zlev1);
            zcff1 = 1.0 - Z; zcff2 = Z;
        }
    } else {
        /* interpolation_module.f90:559-582.  Pinned: the reference reads
         * getWlevel(...,0) (s_w(0), out of bounds) when z is below level 1
         * and leaves zlev(1) undefined when z is above level N+1; both
         * cases here take the boundary level's value. */
        nz = N + 1; Itop = nz; Ibot = nz;
        for (i = 1; i <= nz; i++) {
            zlev2 = orc_getwlevel(g, zeta, depth, i);
            if (zlev2 > zpar) {
                Itop = i; Ibot = i - 1;
                if (i > 1) zlev1 = orc_getwlevel(g, zeta, depth, i - 1);
                break;
            }
        }
        if (i > nz) {
            *flags |= ORC_FLAG_WTOP;
            Itop = nz; Ibot = nz; zcff1 = 0.5; zcff2 = 0.5;
        } else if (i == 1) {
            *flags |= ORC_FLAG_WBOT;
            Itop = 1; Ibot = 1; zcff1 = 0.5; zcff2 = 0.5;
        } else {
            Z = (zpar - zlev1) / (zlev2 - zlev1);
            zcff1 = 1.0 - Z; zcff2 = Z;
        }
    }

    int Inode = ifloor(ipar), Jnode = ifloor(jpar);
    double X = ipar - (double)Inode, Y = jpar - (double)Jnode;
    double cff[4], m[4];
    int ci[4], cj[4];
    const double *fld;
    int fni, fnj; /* field dims */
    int zero_dry = 0; /* u/v rule */

    if (var == ORC_V_U) {
        /* interpolation_module.f90:608-688 */
        const int xi_u = nx - 1, eta_u = ny;
        double uvI = ipar - 0.5;
        Inode = ifloor(uvI);
        X = uvI - (double)Inode;
        fld = g->u[t - 1]; fni = xi_u; fnj = eta_u;
        int j0 = clampi(Jnode, 1, eta_u, flags), j1 = clampi(Jnode + 1, 1, eta_u, flags);
        if (Inode >= xi_u) {
            ci[0] = ci[1] = ci[2] = ci[3] = xi_u;
            cj[0] = j0; cj[1] = j0; cj[2] = j1; cj[3] = j1;
            m[0] = mk_u(g, t, IX2(xi_u, j0, xi_u)); m[1] = 0; m[2] = 0;
            m[3] = mk_u(g, t, IX2(xi_u, j1, xi_u));
        } else if (Inode < 1) {
            ci[0] = ci[1] = ci[2] = ci[3] = 1;
            cj[0] = j0; cj[1] = j0; cj[2] = j1; cj[3] = j1;
            m[0] = 0; m[1] = mk_u(g, t, IX2(1, j0, xi_u));
            m[2] = mk_u(g, t, IX2(1, j1, xi_u)); m[3] = 0;
        } else {
            ci[0] = Inode; ci[1] = Inode + 1; ci[2] = Inode + 1; ci[3] = Inode;
            cj[0] = j0; cj[1] = j0; cj[2] = j1; cj[3] = j1;
            for (int k = 0; k < 4; k++) m[k] = mk_u(g, t, IX2(ci[k], cj[k], xi_u));
        }
        zero_dry = 1;
    } else if (var == ORC_V_V) {
        /* interpolation_module.f90:692-767, including the reference's
         * "if (Jnode > eta_v) Inode = eta_v" line (line 696) */
        const int xi_v = nx, eta_v = ny - 1;
        double uvJ = jpar - 0.5;
        Jnode = ifloor(uvJ);
        if (Jnode < 1) Jnode = 1;
        if (Jnode > eta_v) Inode = eta_v;
        Y = uvJ - (double)Jnode;
        fld = g->v[t - 1]; fni = xi_v; fnj = eta_v;
        int i0 = clampi(Inode, 1, xi_v, flags), i1 = clampi(Inode + 1, 1, xi_v, flags);
        if (Jnode >= eta_v) {
            ci[0] = i0; ci[1] = i1; ci[2] = i1; ci[3] = i0;
            cj[0] = cj[1] = cj[2] = cj[3] = eta_v;
            m[0] = mk_v(g, t, IX2(i0, eta_v, xi_v));
            m[1] = mk_v(g, t, IX2(i1, eta_v, xi_v));
            m[2] = 0; m[3] = 0;
        } else {
            ci[0] = i0; ci[1] = i1; ci[2] = i1; ci[3] = i0;
            cj[0] = Jnode; cj[1] = Jnode; cj[2] = Jnode + 1; cj[3] = Jnode + 1;
            for (int k = 0; k < 4; k++) m[k] = mk_v(g, t, IX2(ci[k], cj[k], xi_v));
        }
        zero_dry = 1;
    } else {
        /* w (interpolation_module.f90:917-939), AKs (810-829), salt and
         * temp (769-809): bilinear, inverse-distance when a corner is dry */
        fld = (var == ORC_V_W) ? g->w[t - 1]
            : (var == ORC_V_AKS) ? g->aks[t - 1]
            : (var == ORC_V_SALT) ? g->salt[t - 1]
            : (var == ORC_V_TEMP) ? g->temp[t - 1]
            : (var == ORC_V_TURBACCEL) ? g->turbaccel[t - 1]          /* 831-851 */
            : (var == ORC_V_TURBVORT) ? g->turbvort[t - 1]            /* 852-872 */
            : (var == ORC_V_WAVEACCELU) ? g->waveaccelu[t - 1]        /* 874-894 */
            : g->waveaccelv[t - 1];                                   /* 896-916 */
        fni = nx; fnj = ny;
        int i0 = clampi(Inode, 1, nx, flags), i1 = clampi(Inode + 1, 1, nx, flags);
        int j0 = clampi(Jnode, 1, ny, flags), j1 = clampi(Jnode + 1, 1, ny, flags);
        ci[0] = i0; ci[1] = i1; ci[2] = i1; ci[3] = i0;
        cj[0] = j0; cj[1] = j0; cj[2] = j1; cj[3] = j1;
        for (int k = 0; k < 4; k++) m[k] = mk_r(g, t, IX2(ci[k], cj[k], nx));
    }

    cff[0] = (1 - X) * (1 - Y);
    cff[1] = X * (1 - Y);
    cff[2] = X * Y;
    cff[3] = (1 - X) * Y;
    double nwater = m[0] + m[1] + m[2] + m[3];
    int use[4] = {1, 1, 1, 1};
    if (zero_dry) {
        if (nwater < 4.0 && nwater > 0.0) {
            for (int k = 0; k < 4; k++) if (m[k] == 0.0) use[k] = 0;
        } else if (nwater == 0.0) {
            for (int k = 0; k < 4; k++) { cff[k] = 0.0; use[k] = 0; }
        }
    } else if (nwater < 4.0) {
        getcoeff(X, Y, m, cff, flags);
    }

    /* zprof(i) for the whole column, as the reference forms it */
    double zprof[512];
    for (int k = 1; k <= nz; k++) {
        double v0 = use[0] ? fld[IX3(ci[0], cj[0], k, fni, fnj)] : 0.0;
        double v1 = use[1] ? fld[IX3(ci[1], cj[1], k, fni, fnj)] : 0.0;
        double v2 = use[2] ? fld[IX3(ci[2], cj[2], k, fni, fnj)] : 0.0;
        double v3 = use[3] ? fld[IX3(ci[3], cj[3], k, fni, fnj)] : 0.0;
        zprof[k] = cff[0] * v0 + cff[1] * v1 + cff[2] * v2 + cff[3] * v3;
    }
    return zcff1 * zprof[Ibot] + zcff2 * zprof[Itop];
}

/* getInterpStr, interpolation_module.f90:964-1174: bottom stress at a u
 * (bustr) or v (bvstr) point set, with the u/v edge rules and the
 * zero-the-dry-corners rule.  The rows Jnode+1 (bustr) and the columns
 * Inode+1 (bvstr) are read unclamped by the reference; here clamped and
 * flagged. */
double orc_getinterp_str(const orc_grid *g, int var, double ipar, double jpar, int t, uint32_t *flags)
{
    const int nx = g->xi_rho, ny = g->eta_rho;
    int Inode = ifloor(ipar), Jnode = ifloor(jpar);
    double X = ipar - (double)Inode, Y = jpar - (double)Jnode;
    double cff[4], v[4], m[4];
    if (var == ORC_V_BUSTR) {
        const int xi_u = nx - 1, eta_u = ny;
        const double *f = g->bustr[t - 1];
        double uvI = ipar - 0.5;
        Inode = ifloor(uvI);
        X = uvI - (double)Inode;
        cff[0] = (1 - X) * (1 - Y);
        cff[1] = X * (1 - Y);
        cff[2] = X * Y;
        cff[3] = (1 - X) * Y;
        int j0 = clampi(Jnode, 1, eta_u, flags), j1 = clampi(Jnode + 1, 1, eta_u, flags);
        if (Inode >= xi_u) {
            v[0] = f[IX2(xi_u, j0, xi_u)]; v[1] = f[IX2(xi_u, j0, xi_u)];
            v[2] = f[IX2(xi_u, j1, xi_u)]; v[3] = f[IX2(xi_u, j1, xi_u)];
            m[0] = mk_u(g, t, IX2(xi_u, j0, xi_u)); m[1] = 0; m[2] = 0; m[3] = mk_u(g, t, IX2(xi_u, j1, xi_u));
        } else if (Inode < 1) {
            v[0] = f[IX2(1, j0, xi_u)]; v[1] = f[IX2(1, j0, xi_u)];
            v[2] = f[IX2(1, j1, xi_u)]; v[3] = f[IX2(1, j1, xi_u)];
            m[0] = 0; m[1] = mk_u(g, t, IX2(1, j0, xi_u)); m[2] = mk_u(g, t, IX2(1, j1, xi_u)); m[3] = 0;
        } else {
            v[0] = f[IX2(Inode, j0, xi_u)]; v[1] = f[IX2(Inode + 1, j0, xi_u)];
            v[2] = f[IX2(Inode + 1, j1, xi_u)]; v[3] = f[IX2(Inode, j1, xi_u)];
            m[0] = mk_u(g, t, IX2(Inode, j0, xi_u)); m[1] = mk_u(g, t, IX2(Inode + 1, j0, xi_u));
            m[2] = mk_u(g, t, IX2(Inode + 1, j1, xi_u)); m[3] = mk_u(g, t, IX2(Inode, j1, xi_u));
        }
    } else {
        const int xi_v = nx, eta_v = ny - 1;
        const double *f = g->bvstr[t - 1];
        double uvJ = jpar - 0.5;
        Jnode = ifloor(uvJ);
        if (Jnode < 1) Jnode = 1;
        if (Jnode > eta_v) Inode = eta_v;                       /* the reference's line, as getInterp3D */
        Y = uvJ - (double)Jnode;
        cff[0] = (1 - X) * (1 - Y);
        cff[1] = X * (1 - Y);
        cff[2] = X * Y;
        cff[3] = (1 - X) * Y;
        int i0 = clampi(Inode, 1, xi_v, flags), i1 = clampi(Inode + 1, 1, xi_v, flags);
        if (Jnode >= eta_v) {
            v[0] = f[IX2(i0, eta_v, xi_v)]; v[1] = f[IX2(i1, eta_v, xi_v)];
            v[2] = f[IX2(i1, eta_v, xi_v)]; v[3] = f[IX2(i0, eta_v, xi_v)];
            m[0] = mk_v(g, t, IX2(i0, eta_v, xi_v)); m[1] = mk_v(g, t, IX2(i1, eta_v, xi_v)); m[2] = 0; m[3] = 0;
        } else {
            v[0] = f[IX2(i0, Jnode, xi_v)]; v[1] = f[IX2(i1, Jnode, xi_v)];
            v[2] = f[IX2(i1, Jnode + 1, xi_v)]; v[3] = f[IX2(i0, Jnode + 1, xi_v)];
            m[0] = mk_v(g, t, IX2(i0, Jnode, xi_v)); m[1] = mk_v(g, t, IX2(i1, Jnode, xi_v));
            m[2] = mk_v(g, t, IX2(i1, Jnode + 1, xi_v)); m[3] = mk_v(g, t, IX2(i0, Jnode + 1, xi_v));
        }
    }
    double nwater = m[0] + m[1] + m[2] + m[3];
    if (nwater < 4.0 && nwater > 0.0) {
        for (int k = 0; k < 4; k++) if (m[k] == 0.0) v[k] = 0.0;
    } else if (nwater == 0.0) {
        for (int k = 0; k < 4; k++) { cff[k] = 0.0; v[k] = 0.0; }
    }
    return cff[0] * v[0] + cff[1] * v[1] + cff[2] * v[2] + cff[3] * v[3];
}

/* getInterpAKs, interpolation_module.f90:1175-1229 (one w level) */
static double getinterp_aks(const orc_grid *g, double ipar, double jpar, int t, int lev, uint32_t *flags)
{
    const int nx = g->xi_rho, ny = g->eta_rho;
    int I = ifloor(ipar), J = ifloor(jpar);
    double X = ipar - (double)I, Y = jpar - (double)J;
    int i0 = clampi(I, 1, nx, flags), i1 = clampi(I + 1, 1, nx, flags);
    int j0 = clampi(J, 1, ny, flags), j1 = clampi(J + 1, 1, ny, flags);
    double cff[4], v[4], m[4];
    cff[0] = (1 - X) * (1 - Y);
    cff[1] = X * (1 - Y);
    cff[2] = X * Y;
    cff[3] = (1 - X) * Y;
    const double *a = g->aks[t - 1];
    v[0] = a[IX3(i0, j0, lev, nx, ny)];
    v[1] = a[IX3(i1, j0, lev, nx, ny)];
    v[2] = a[IX3(i1, j1, lev, nx, ny)];
    v[3] = a[IX3(i0, j1, lev, nx, ny)];
    m[0] = g->mask_rho[IX2(i0, j0, nx)];
    m[1] = g->mask_rho[IX2(i1, j0, nx)];
    m[2] = g->mask_rho[IX2(i1, j1, nx)];
    m[3] = g->mask_rho[IX2(i0, j1, nx)];
    double nwater = m[0] + m[1] + m[2] + m[3];
    if (nwater < 4.0) getcoeff(X, Y, m, cff, flags);
    return cff[0] * v[0] + cff[1] * v[1] + cff[2] * v[2] + cff[3] * v[3];
}

/* ======================= boundaries ======================= */

/* inside, interpolation_module.f90:269-420 (crossing count, Reid 1969).
 * xb, yb must have room for nb+1 entries. */
int orc_inside(int nb, double *xb, double *yb, double xo, double yo)
{
    int crossings = 0;
    xb[nb] = xb[0];
    yb[nb] = yb[0];
    for (int k = 0; k < nb; k++) {
        if (((xb[k + 1] - xo) * (xo - xb[k]) >= 0.0) && (xb[k] != xb[k + 1])) {
            double dx1 = xo - xb[k];
            double dx2 = xb[k + 1] - xo;
            double dxy = dx2 * (yo - yb[k]) - dx1 * (yb[k + 1] - yo);
            int inc = 0;
            if ((xb[k] == xo) && (yb[k] == yo)) {
                return 1;
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

/* bounds, boundary_module.f90:43-143 */
void orc_bounds(const orc_grid *g, double ipar, double jpar, int *nmask, int *ingrid, int *obound)
{
    const double ecut = F_0P1;
    const double fcut = 1.0 - ecut;
    const int nx = g->xi_rho, ny = g->eta_rho;
    *ingrid = 0;
    *obound = 0;
    *nmask = 0;
    int I = ifloor(ipar), J = ifloor(jpar);
    double X = ipar - (double)I, Y = jpar - (double)J;
    double tX[4] = {0, 0, 0, 0}, tY[4] = {0, 0, 0, 0};
    if ((I > 1) && (J > 1) && (I < nx - 1) && (J < ny - 1)) {
        double m11 = g->mask_rho[IX2(I, J, nx)];
        double m21 = g->mask_rho[IX2(I + 1, J, nx)];
        double m22 = g->mask_rho[IX2(I + 1, J + 1, nx)];
        double m12 = g->mask_rho[IX2(I, J + 1, nx)];
        int nm = (int)(m11 + m21 + m22 + m12);
        *nmask = nm;
        if (nm == 4) *ingrid = 1;
        if (nm == 3) {
            double mm[2][2] = {{m11, m12}, {m21, m22}}; /* mm[it-1][jt-1] */
            int n = 0;
            for (int it = 1; it <= 2; it++)
                for (int jt = 1; jt <= 2; jt++)
                    if (mm[it - 1][jt - 1] == 1) {
                        tX[n] = (double)it - 1.0;
                        tY[n] = (double)jt - 1.0;
                        n++;
                    }
            if (orc_inside(3, tX, tY, X, Y)) *ingrid = 1;
        }
        if (nm == 2) {
            if (m11 == 1 && (X < ecut) && (Y < ecut)) *ingrid = 1;
            if (m21 == 1 && (X > fcut) && (Y < ecut)) *ingrid = 1;
            if (m22 == 1 && (X > fcut) && (Y > fcut)) *ingrid = 1;
            if (m12 == 1 && (X < ecut) && (Y > fcut)) *ingrid = 1;
        }
        if ((I <= 1) || (J <= 1) || (I >= nx - 1) || (J >= ny - 1)) *obound = 1;
    } else {
        *obound = 1;
    }
}

/* zbounds, boundary_module.f90:145-179 */
static void zbounds(const orc_grid *g, double ipar, double jpar, double *zpar, int *ingrid, int t, uint32_t *flags)
{
    *ingrid = 0;
    int I = ifloor(ipar);
    if (I > 0) {
        double tdepth = -1.0 * orc_getinterp2d(g, ORC_V_DEPTH, ipar, jpar, 1, flags);
        double tzeta = orc_getinterp2d(g, ORC_V_ZETA, ipar, jpar, t, flags);
        if ((*zpar < tzeta) && (*zpar > tdepth)) *ingrid = 1;
        if (*zpar >= tzeta) {
            *zpar = tzeta - 0.01;
            *ingrid = 1;
        }
    }
}

/* ======================= PPPACK smoothing spline ======================= */

#define V_(i, j) v[((i) - 1) + ((j) - 1) * (int64_t)np]
#define A_(i, j) a[((i) - 1) + ((j) - 1) * (int64_t)np]

/* setupq, pppack.f90:4726-4825 */
static void setupq(const double *x, const double *dx, const double *y, int np, double *v, double *qty)
{
    x -= 1; dx -= 1; y -= 1; qty -= 1;
    for (int i = 1; i <= np - 1; i++) V_(i, 4) = x[i + 1] - x[i];
    for (int i = 2; i <= np - 1; i++) V_(i, 1) = dx[i - 1] / V_(i - 1, 4);
    V_(np, 1) = 0.0;
    for (int i = 2; i <= np - 1; i++) V_(i, 2) = -dx[i] / V_(i, 4) - dx[i] / V_(i - 1, 4);
    for (int i = 2; i <= np - 1; i++) V_(i, 3) = dx[i + 1] / V_(i, 4);
    for (int i = 2; i <= np - 1; i++)
        V_(i, 5) = V_(i, 1) * V_(i, 1) + V_(i, 2) * V_(i, 2) + V_(i, 3) * V_(i, 3);
    for (int i = 2; i <= np - 2; i++) V_(i, 6) = V_(i, 2) * V_(i + 1, 1) + V_(i, 3) * V_(i + 1, 2);
    V_(np - 1, 6) = 0.0;
    for (int i = 2; i <= np - 3; i++) V_(i, 7) = V_(i, 3) * V_(i + 2, 1);
    V_(np - 2, 7) = 0.0;
    V_(np - 1, 7) = 0.0;
    double prev = (y[2] - y[1]) / V_(1, 4);
    for (int i = 2; i <= np - 1; i++) {
        double diff = (y[i + 1] - y[i]) / V_(i, 4);
        qty[i] = diff - prev;
        prev = diff;
    }
}

/* chol1d, pppack.f90:1428-1566 */
static void chol1d(double p, double *v, const double *qty, int np, double *u, double *qu)
{
    qty -= 1; u -= 1; qu -= 1;
    double six1mp = 6.0 * (1.0 - p);
    double twop = 2.0 * p;
    for (int i = 2; i <= np - 1; i++) {
        V_(i, 1) = six1mp * V_(i, 5) + twop * (V_(i - 1, 4) + V_(i, 4));
        V_(i, 2) = six1mp * V_(i, 6) + p * V_(i, 4);
        V_(i, 3) = six1mp * V_(i, 7);
    }
    if (np < 4) {
        u[1] = 0.0;
        u[2] = qty[2] / V_(2, 1);
        u[3] = 0.0;
    } else {
        for (int i = 2; i <= np - 2; i++) {
            double ratio = V_(i, 2) / V_(i, 1);
            V_(i + 1, 1) = V_(i + 1, 1) - ratio * V_(i, 2);
            V_(i + 1, 2) = V_(i + 1, 2) - ratio * V_(i, 3);
            V_(i, 2) = ratio;
            ratio = V_(i, 3) / V_(i, 1);
            V_(i + 2, 1) = V_(i + 2, 1) - ratio * V_(i, 3);
            V_(i, 3) = ratio;
        }
        u[1] = 0.0;
        V_(1, 3) = 0.0;
        u[2] = qty[2];
        for (int i = 2; i <= np - 2; i++)
            u[i + 1] = qty[i + 1] - V_(i, 2) * u[i] - V_(i - 1, 3) * u[i - 1];
        u[np] = 0.0;
        u[np - 1] = u[np - 1] / V_(np - 1, 1);
        for (int i = np - 2; i >= 2; i--)
            u[i] = u[i] / V_(i, 1) - u[i + 1] * V_(i, 2) - u[i + 2] * V_(i, 3);
    }
    double prev = 0.0;
    for (int i = 2; i <= np; i++) {
        qu[i] = (u[i] - u[i - 1]) / V_(i - 1, 4);
        qu[i - 1] = qu[i] - prev;
        prev = qu[i];
    }
    qu[np] = -qu[np];
}

static double dot_sq(const double *a, const double *dy, int np)
{
    double s = 0.0;
    for (int i = 0; i < np; i++) s = s + (a[i] * a[i]) * (dy[i] * dy[i]);
    return s;
}

/* smooth, pppack.f90:5108-5317.  The reference's secant loop has no
 * iteration cap; here it stops after max_iter passes (ORC_FLAG_SPLINE). */
double orc_smooth(const double *x, const double *y, const double *dy, int np, double s,
                  double *v, double *a, int max_iter, int *iters)
{
    double p, q, sfq, utru, ooss, oosf, prevq, prevsf, change;
    int it = 0;
    setupq(x, dy, y, np, v, &A_(1, 4));
    if (s <= 0.0) {
        p = 1.0;
        chol1d(p, v, &A_(1, 4), np, &A_(1, 3), &A_(1, 1));
        sfq = 0.0;
    } else {
        p = 0.0;
        chol1d(p, v, &A_(1, 4), np, &A_(1, 3), &A_(1, 1));
        sfq = 36.0 * dot_sq(&A_(1, 1), dy, np);
        if (s < sfq) {
            utru = 0.0;
            for (int i = 2; i <= np; i++)
                utru = utru + V_(i - 1, 4) * (A_(i - 1, 3) * (A_(i - 1, 3) + A_(i, 3)) + A_(i, 3) * A_(i, 3));
            ooss = 1.0 / sqrt(s);
            oosf = 1.0 / sqrt(sfq);
            q = -(oosf - ooss) * sfq / (6.0 * utru * oosf);
            prevq = 0.0;
            prevsf = oosf;
            for (;;) {
                chol1d(q / (1.0 + q), v, &A_(1, 4), np, &A_(1, 3), &A_(1, 1));
                sfq = 36.0 * dot_sq(&A_(1, 1), dy, np) / ((1.0 + q) * (1.0 + q));
                it++;
                if (fabs(sfq - s) <= 0.01 * s) break;
                if (it >= max_iter) { it = -it; break; }
                oosf = 1.0 / sqrt(sfq);
                change = (q - prevq) / (oosf - prevsf) * (oosf - ooss);
                prevq = q;
                q = q - change;
                prevsf = oosf;
            }
            p = q / (1.0 + q);
        }
    }
    for (int i = 1; i <= np; i++)
        A_(i, 1) = y[i - 1] - 6.0 * (1.0 - p) * (dy[i - 1] * dy[i - 1]) * A_(i, 1);
    for (int i = 1; i <= np; i++) A_(i, 3) = A_(i, 3) * 6.0 * p;
    for (int i = 1; i <= np - 1; i++) {
        A_(i, 4) = (A_(i + 1, 3) - A_(i, 3)) / V_(i, 4);
        A_(i, 2) = (A_(i + 1, 1) - A_(i, 1)) / V_(i, 4) - (A_(i, 3) + A_(i, 4) / 3.0 * V_(i, 4)) / 2.0 * V_(i, 4);
    }
    if (iters) *iters = it;
    return sfq;
}

/* interv, pppack.f90:3363-3576.  The reference keeps its start hint ILO in a
 * SAVE variable; the result does not depend on the hint, which is kept per
 * thread here. */
static _Thread_local int interv_ilo = 1;
static int interv(const double *xt, int lxt, double x)
{
    int ilo = interv_ilo, ihi, istep, middle, left;
    xt -= 1;
    ihi = ilo + 1;
    if (lxt <= ihi) {
        if (xt[lxt] <= x) goto L110;
        if (lxt <= 1) { interv_ilo = ilo; return 1; }
        ilo = lxt - 1;
        ihi = lxt;
    }
    if (xt[ihi] <= x) goto L20;
    if (xt[ilo] <= x) { interv_ilo = ilo; return ilo; }
    istep = 1;
L10:
    ihi = ilo;
    ilo = ihi - istep;
    if (1 < ilo) {
        if (xt[ilo] <= x) goto L50;
        istep = istep * 2;
        goto L10;
    }
    ilo = 1;
    if (x < xt[1]) { interv_ilo = ilo; return 1; }
    goto L50;
L20:
    istep = 1;
L30:
    ilo = ihi;
    ihi = ilo + istep;
    if (ihi < lxt) {
        if (x < xt[ihi]) goto L50;
        istep = istep * 2;
        goto L30;
    }
    if (xt[lxt] <= x) goto L110;
    ihi = lxt;
L50:
    for (;;) {
        middle = (ilo + ihi) / 2;
        if (middle == ilo) { interv_ilo = ilo; return ilo; }
        if (xt[middle] <= x) ilo = middle; else ihi = middle;
    }
L110:
    interv_ilo = ilo;
    for (left = lxt - 1; left >= 1; left--)
        if (xt[left] < xt[lxt]) return left;
    return 0;
}

/* ppvalu, pppack.f90:4246-4362; coef is (k, l) column-major */
double orc_ppvalu(const double *brk, const double *coef, int l, int k, double x, int jderiv)
{
    double value = 0.0;
    double fmmjdr = (double)(k - jderiv);
    if (k <= jderiv) return value;
    int i = interv(brk, l + 1, x);
    double h = x - brk[i - 1];
    int m = k;
    for (;;) {
        value = (value / fmmjdr) * h + coef[(m - 1) + (int64_t)(i - 1) * k];
        m = m - 1;
        fmmjdr = fmmjdr - 1.0;
        if (fmmjdr <= 0.0) break;
    }
    return value;
}

/* ======================= particle physics ======================= */

typedef struct {
    const orc_params *prm;
    const orc_grid *g;
    const double *ex, *ix;
    int ets, tb, tc, tf;
} step_env;

/* find_currents, advection_module.f90:129-350 (version=2: all stages at
 * ix(2); ets==1 uses (b,b,c) for u,v,w only). zpar is INOUT. */
static void find_currents(const step_env *e, double X, double Y, double *zpar,
                          double *Uad, double *Vad, double *Wad, uint32_t *fl)
{
    const orc_grid *g = e->g;
    double tdepth = -1.0 * orc_getinterp2d(g, ORC_V_DEPTH, X, Y, e->tc, fl);
    double zetab = orc_getinterp2d(g, ORC_V_ZETA, X, Y, e->tb, fl);
    double zetac = orc_getinterp2d(g, ORC_V_ZETA, X, Y, e->tc, fl);
    double zetaf = orc_getinterp2d(g, ORC_V_ZETA, X, Y, e->tf, fl);
    if (*zpar < tdepth) *zpar = tdepth + F_0P001;
    double ey[3] = {zetab, zetac, zetaf};
    double zeta = orc_polintd(e->ex, ey, e->ix[1]);
    if (*zpar > zeta) *zpar = zeta - F_0P001;
    double Z = *zpar;
    double Uc = orc_getinterp3d(g, ORC_V_U, X, Y, Z, e->tc, 1, zeta, tdepth, fl);
    double Uf = orc_getinterp3d(g, ORC_V_U, X, Y, Z, e->tf, 1, zeta, tdepth, fl);
    double Ub = orc_getinterp3d(g, ORC_V_U, X, Y, Z, e->tb, 1, zeta, tdepth, fl);
    double Vb = orc_getinterp3d(g, ORC_V_V, X, Y, Z, e->tb, 1, zeta, tdepth, fl);
    double Vc = orc_getinterp3d(g, ORC_V_V, X, Y, Z, e->tc, 1, zeta, tdepth, fl);
    double Vf = orc_getinterp3d(g, ORC_V_V, X, Y, Z, e->tf, 1, zeta, tdepth, fl);
    double Wb = orc_getinterp3d(g, ORC_V_W, X, Y, Z, e->tb, 2, zeta, tdepth, fl);
    double Wc = orc_getinterp3d(g, ORC_V_W, X, Y, Z, e->tc, 2, zeta, tdepth, fl);
    double Wf = orc_getinterp3d(g, ORC_V_W, X, Y, Z, e->tf, 2, zeta, tdepth, fl);
    if (e->ets == 1) {
        ey[0] = Ub; ey[1] = Ub; ey[2] = Uc; *Uad = orc_polintd(e->ex, ey, e->ix[1]);
        ey[0] = Vb; ey[1] = Vb; ey[2] = Vc; *Vad = orc_polintd(e->ex, ey, e->ix[1]);
        ey[0] = Wb; ey[1] = Wb; ey[2] = Wc; *Wad = orc_polintd(e->ex, ey, e->ix[1]);
    } else {
        ey[0] = Ub; ey[1] = Uc; ey[2] = Uf; *Uad = orc_polintd(e->ex, ey, e->ix[1]);
        ey[0] = Vb; ey[1] = Vc; ey[2] = Vf; *Vad = orc_polintd(e->ex, ey, e->ix[1]);
        ey[0] = Wb; ey[1] = Wc; ey[2] = Wf; *Wad = orc_polintd(e->ex, ey, e->ix[1]);
    }
}

/* RKAdvect, advection_module.f90:20-125.  All three intermediate positions
 * use idt/2 (lines 54-56, 75-77, 96-98); Zpar is modified by the first
 * find_currents call and the modification is visible to the caller. */
static void rk_advect(const step_env *e, double Xpar, double Ypar, double *Zpar, double pm, double pn,
                      double *AdvectX, double *AdvectY, double *AdvectZ, uint32_t *fl)
{
    const double didt = (double)e->prm->idt;
    double Uad, Vad, Wad;
    double kn1_u, kn1_v, kn1_w, kn2_u, kn2_v, kn2_w, kn3_u, kn3_v, kn3_w, kn4_u, kn4_v, kn4_w;
    find_currents(e, Xpar, Ypar, Zpar, &Uad, &Vad, &Wad, fl);
    kn1_u = Uad * pm; kn1_v = Vad * pn; kn1_w = Wad;
    double x1 = Xpar + Uad * pm * didt / 2.0;
    double y1 = Ypar + Vad * pn * didt / 2.0;
    double z1 = *Zpar + Wad * didt / 2.0;
    find_currents(e, x1, y1, &z1, &Uad, &Vad, &Wad, fl);
    kn2_u = Uad * pm; kn2_v = Vad * pn; kn2_w = Wad;
    double x2 = Xpar + Uad * pm * didt / 2.0;
    double y2 = Ypar + Vad * pn * didt / 2.0;
    double z2 = *Zpar + Wad * didt / 2.0;
    find_currents(e, x2, y2, &z2, &Uad, &Vad, &Wad, fl);
    kn3_u = Uad * pm; kn3_v = Vad * pn; kn3_w = Wad;
    double x3 = Xpar + Uad * pm * didt / 2.0;
    double y3 = Ypar + Vad * pn * didt / 2.0;
    double z3 = *Zpar + Wad * didt / 2.0;
    find_currents(e, x3, y3, &z3, &Uad, &Vad, &Wad, fl);
    kn4_u = Uad * pm; kn4_v = Vad * pn; kn4_w = Wad;
    double P_U = (kn1_u + 2.0 * kn2_u + 2.0 * kn3_u + kn4_u) / 6.0;
    double P_V = (kn1_v + 2.0 * kn2_v + 2.0 * kn3_v + kn4_v) / 6.0;
    double P_W = (kn1_w + 2.0 * kn2_w + 2.0 * kn3_w + kn4_w) / 6.0;
    *AdvectX = didt * P_U;
    *AdvectY = didt * P_V;
    *AdvectZ = didt * P_W;
}

/* HTurb, hor_turb_module.f90:30-51 ((...)**0.5 evaluated as sqrt) */
static void hturb(const step_env *e, int ng, const noise_ctx *nc, double *TurbHx, double *TurbHy)
{
    double r = 1.0;
    double KM = e->prm->constant_hturb[ng - 1];
    double devX = draw_normal(nc, 0);
    double devY = draw_normal(nc, 1);
    *TurbHx = devX * sqrt(2.0 / r * KM * (double)e->prm->idt);
    *TurbHy = devY * sqrt(2.0 / r * KM * (double)e->prm->idt);
}

typedef struct {
    double *z, *kh, *fitz, *fitkh, *dy, *v, *a, *coefsm;
    int cap_sw, cap_np;
} vt_work;

static int vt_work_alloc(vt_work *w, int sw, int np)
{
    w->cap_sw = sw; w->cap_np = np;
    w->z = malloc(sizeof(double) * sw);
    w->kh = malloc(sizeof(double) * sw);
    w->fitz = malloc(sizeof(double) * np);
    w->fitkh = malloc(sizeof(double) * np);
    w->dy = malloc(sizeof(double) * np);
    w->v = malloc(sizeof(double) * np * 7);
    w->a = malloc(sizeof(double) * np * 4);
    w->coefsm = malloc(sizeof(double) * np * 4);
    return w->z && w->kh && w->fitz && w->fitkh && w->dy && w->v && w->a && w->coefsm;
}

static void vt_work_free(vt_work *w)
{
    free(w->z); free(w->kh); free(w->fitz); free(w->fitkh);
    free(w->dy); free(w->v); free(w->a); free(w->coefsm);
}

/* VTurb, ver_turb_module.f90:31-329 */
static double vturb(const step_env *e, double Xpar, double Ypar, double Zpar, const noise_ctx *nc,
                    vt_work *w, uint32_t *fl, int64_t *n_iter)
{
    const orc_params *prm = e->prm;
    const orc_grid *g = e->g;
    const int sw = g->N + 1;
    const int np = (int)((double)sw * prm->sub);
    double *z = w->z - 1, *kh = w->kh - 1, *fitz = w->fitz - 1, *fitkh = w->fitkh - 1, *dy = w->dy - 1;
    double ey[3];

    memset(w->v, 0, sizeof(double) * np * 7);
    memset(w->a, 0, sizeof(double) * np * 4);
    double tdepth = -1.0 * orc_getinterp2d(g, ORC_V_DEPTH, Xpar, Ypar, e->tc, fl);
    double zetab = orc_getinterp2d(g, ORC_V_ZETA, Xpar, Ypar, e->tb, fl);
    double zetac = orc_getinterp2d(g, ORC_V_ZETA, Xpar, Ypar, e->tc, fl);
    double zetaf = orc_getinterp2d(g, ORC_V_ZETA, Xpar, Ypar, e->tf, fl);
    ey[0] = zetab; ey[1] = zetac; ey[2] = zetaf;
    double zeta = orc_polintd(e->ex, ey, e->ix[1]);
    for (int i = 1; i <= sw; i++) {
        ey[0] = orc_getwlevel(g, zetab, tdepth, i);
        ey[1] = orc_getwlevel(g, zetac, tdepth, i);
        ey[2] = orc_getwlevel(g, zetaf, tdepth, i);
        z[i] = orc_polintd(e->ex, ey, e->ix[1]);
        ey[0] = getinterp_aks(g, Xpar, Ypar, e->tb, i, fl);
        ey[1] = getinterp_aks(g, Xpar, Ypar, e->tc, i, fl);
        ey[2] = getinterp_aks(g, Xpar, Ypar, e->tf, i, fl);
        kh[i] = orc_polintd(e->ex, ey, e->ix[1]);
    }
    double dz = (z[sw] - z[1]) / (double)(np - 1);
    fitz[1] = z[1];
    fitz[np] = z[sw];
    fitkh[1] = kh[1];
    fitkh[np] = kh[sw];
    for (int i = 2; i <= np - 1; i++) {
        double mm;
        fitz[i] = fitz[i - 1] + dz;
        orc_linint(&z[1], &kh[1], sw, fitz[i], &fitkh[i], &mm);
        dy[i] = prm->serr;
    }
    /* Pinned: dy(1) and dy(np) are never set in the reference
     * (ver_turb_module.f90:131-136); they are taken as serr. */
    dy[1] = prm->serr;
    dy[np] = prm->serr;
    if (prm->vt_dy_end == prm->vt_dy_end) { dy[1] = prm->vt_dy_end; dy[np] = prm->vt_dy_end; }
    /* experiment variant 1: K = c 4 xi (1 - xi) fitted to the column */
    double pc = 0.0;
    const double hcol = zeta - tdepth;
    if (prm->vt_variant == 1) {
        double num = 0.0, den = 0.0;
        for (int k = 1; k <= sw; k++) {
            const double xi = (z[k] - tdepth) / hcol;
            const double phi = 4.0 * xi * (1.0 - xi);
            num += kh[k] * phi;
            den += phi * phi;
        }
        pc = den > 0.0 ? num / den : 0.0;
    } else {
        int iters = 0;
        orc_smooth(&fitz[1], &fitkh[1], &dy[1], np, prm->smth, w->v, w->a, prm->spline_max_iter, &iters);
        if (iters < 0) { *fl |= ORC_FLAG_SPLINE; iters = -iters; }
        *n_iter += iters;
        for (int i = 1; i <= np; i++)
            for (int j = 1; j <= 4; j++)
                w->coefsm[(j - 1) + (int64_t)(i - 1) * 4] = w->a[(i - 1) + (int64_t)(j - 1) * np];
    }

    const double deltat = prm->deltat;
    const int loop = prm->idt / (int)deltat;
    double ParZc = Zpar;
    for (int i = 1; i <= loop; i++) {
        double Kprimec = 0.0, KprimeZc, Z3rdc, KH3rdc, DEV, r, dTz, newZc;
        if (ParZc <= tdepth || ParZc >= zeta) Kprimec = 0.0;
        else if (prm->vt_variant == 1) Kprimec = pc * 4.0 * (1.0 - 2.0 * ((ParZc - tdepth) / hcol)) / hcol;
        else Kprimec = orc_ppvalu(&fitz[1], w->coefsm, np - 1, 4, ParZc, 1);
        KprimeZc = Kprimec * deltat;
        Z3rdc = ParZc + 0.5 * KprimeZc;
        if (Z3rdc < tdepth || Z3rdc > zeta) {
            KH3rdc = prm->aksback;
        } else {
            if (prm->vt_variant == 1) {
                const double xi = (Z3rdc - tdepth) / hcol;
                KH3rdc = pc * 4.0 * xi * (1.0 - xi);
            } else {
                KH3rdc = orc_ppvalu(&fitz[1], w->coefsm, np - 1, 4, Z3rdc, 0);
            }
            if (KH3rdc < prm->aksback) KH3rdc = prm->aksback;
        }
        DEV = draw_normal(nc, (uint32_t)(1 + i));
        r = 1.0;
        dTz = KprimeZc + DEV * sqrt(2.0 / r * KH3rdc * deltat);
        newZc = ParZc + dTz;
        ParZc = newZc;
        if (ParZc <= tdepth) ParZc = tdepth + fabs(ParZc - tdepth);
        if (ParZc >= zeta) ParZc = zeta - fabs(ParZc - zeta);
    }
    return ParZc - Zpar;
}

/* One particle of update_particles, ROMSPath.f90:662-905 */
/* behave, behavior_module.f90:186-393, at the step's (Xpar, Ypar, Zpar)
 * (Zpar after find_currents' clamp) in the particle's grid.  Draws, in
 * the reference's order, 4 laplace, 2 norm and 1 genrand_real3 whenever
 * Process_VA or Process_WA; writes behout (par(:,pAcc/pVort/pbehaveW/pSSF),
 * ROMSPath.f90:800-804) and returns ZBehav.  Real powers are pinned:
 * x**2.0D0 = x*x, r**3.0D0 = (r*r)*r, x**0.5D0 = sqrt(x). */
static double behave(const step_env *e, const orc_grid *g, double Xpar, double Ypar, double Zpar,
                     const noise_ctx *nc, double behout[4], uint32_t *fl)
{
    const orc_params *b = e->prm;
    const double G = 980.0, RHOF = 1.026, MU = 0.010260, RHOP = 1.06;   /* ROMSPath.h:15-19 */
    double wb = 0.0;
    behout[0] = behout[1] = behout[2] = behout[3] = 0.0;
    if (b->process_va || b->process_wa) {                       /* 240 */
        const double depth = -1.0 * orc_getinterp2d(g, ORC_V_DEPTH, Xpar, Ypar, e->tc, fl);
        const double zt[3] = {orc_getinterp2d(g, ORC_V_ZETA, Xpar, Ypar, e->tb, fl),
                              orc_getinterp2d(g, ORC_V_ZETA, Xpar, Ypar, e->tc, fl),
                              orc_getinterp2d(g, ORC_V_ZETA, Xpar, Ypar, e->tf, fl)};
        const int sl[3] = {e->tb, e->tc, e->tf};
        double ey[3], stdaccturbu, stdvortturb, stdaccwaveu, stdaccwavev;
        if (b->process_va) {                                    /* 249-264 */
            for (int q = 0; q < 3; q++)
                ey[q] = orc_getinterp3d(g, ORC_V_TURBACCEL, Xpar, Ypar, Zpar, sl[q], 2, zt[q], depth, fl);
            stdaccturbu = orc_polintd(e->ex, ey, e->ix[1]);
            for (int q = 0; q < 3; q++)
                ey[q] = orc_getinterp3d(g, ORC_V_TURBVORT, Xpar, Ypar, Zpar, sl[q], 2, zt[q], depth, fl);
            stdvortturb = orc_polintd(e->ex, ey, e->ix[1]);
            stdaccturbu = stdaccturbu * 100.0;
        } else {
            stdaccturbu = 0.0;
            stdvortturb = 0.0;
        }
        if (b->process_wa) {                                    /* 269-280 */
            for (int q = 0; q < 3; q++)
                ey[q] = orc_getinterp3d(g, ORC_V_WAVEACCELU, Xpar, Ypar, Zpar, sl[q], 2, zt[q], depth, fl);
            stdaccwaveu = orc_polintd(e->ex, ey, e->ix[1]);
            for (int q = 0; q < 3; q++)
                ey[q] = orc_getinterp3d(g, ORC_V_WAVEACCELV, Xpar, Ypar, Zpar, sl[q], 2, zt[q], depth, fl);
            stdaccwavev = orc_polintd(e->ex, ey, e->ix[1]);
            stdaccwaveu = stdaccwaveu * 100.0;
            stdaccwavev = stdaccwavev * 100.0;
        } else {
            stdaccwaveu = 0.0;
            stdaccwavev = 0.0;
        }
        const uint32_t d0 = 2u + (uint32_t)(b->idt / (int)b->deltat);
        const double vortturbu = stdvortturb * laplace_of(draw_uniform(nc, d0, 0));   /* 285-292 */
        const double vortturbv = stdvortturb * laplace_of(draw_uniform(nc, d0, 1));
        const double vorttot = sqrt(vortturbu * vortturbu + vortturbv * vortturbv);
        const double accturbu = stdaccturbu * laplace_of(draw_uniform(nc, d0, 2));    /* 298-302 */
        const double accturbv = stdaccturbu * laplace_of(draw_uniform(nc, d0, 3));
        const double accwaveu = stdaccwaveu * draw_normal(nc, d0);                  /* 307-311 */
        const double accwavev = stdaccwavev * draw_normal(nc, d0 + 1);
        const double au = accturbu + accwaveu, av = accturbv + accwavev;
        const double acctot = sqrt(au * au + av * av);
        const double c1v = 2.0 / orc_log(b->vort_cr / b->vort_sat);                /* 322-326 */
        const double c2v = c1v * orc_log(vorttot / sqrt(b->vort_cr * b->vort_sat));
        const double c1a = 2.0 / orc_log(b->acc_cr / b->acc_sat);
        const double c2a = c1a * orc_log(acctot / sqrt(b->acc_cr * b->acc_sat));
        const double ev = orc_exp(-2.0 * c2v), ea = orc_exp(-2.0 * c2a);
        const double pswimv = (b->b1pv - b->b0pv) / (1.0 + ev) + b->b0pv;          /* 329-330 */
        const double pswima = (b->b1pa - b->b0pa) / (1.0 + ea) + b->b0pa;
        double pswim;
        if (b->va_flag == 1) pswim = pswimv;
        else if (b->va_flag == 2) pswim = pswima;
        else pswim = (pswima < pswimv) ? pswima : pswimv;                          /* min(pswima,pswimv) */
        const double wswimv = ((b->b1w - b->b0wv) * 1.0 / (1.0 + ev)) + b->b0wv;   /* 341 */
        const double wswima = ((b->b1w - b->b0wa) * 1.0 / (1.0 + ea)) + b->b0wa;   /* 344 */
        double wswim;
        if (b->va_flag == 1) wswim = wswimv;
        else if (b->va_flag == 2) wswim = wswima;
        else wswim = wswima + wswimv;
        const double r = b->initsize / 2.0e4;                                       /* 359-360 */
        const double wsink = ((3.0 * MU) - sqrt((4.0 / 3.0) * G * ((r * r) * r) * RHOF * (RHOP - RHOF) +
                                                (9.0 * (MU * MU)))) / (r * RHOF);
        behout[0] = acctot / 100.0;
        behout[1] = vorttot;
        if (draw_uniform(nc, d0, 4) < pswim) {                                     /* 366-375 */
            wb = wswim;
            behout[3] = 0.0;
        } else {
            wb = wsink;
            behout[3] = 1.0;
        }
        behout[2] = wb;
    }
    if (b->behavior == 1) return b->swimfast * (double)b->idt;                    /* 381-391 */
    if (b->behavior == 10) return wb * (double)b->idt / 100.0;
    return 0.0;
}

static void update_one(const step_env *e0, const orc_grid *grids, orc_particles *p, int64_t n,
                       const orc_noise *noise, vt_work *w, int64_t *n_spline, int64_t *n_iter)
{
    const orc_params *prm = e0->prm;
    if (e0->ix[2] <= p->dob[n]) return;                          /* 672 */
    if (p->status[n] == 9.0) return;                             /* 676 */
    if (prm->open_ocean_boundary && !p->isin[n]) return;         /* 688 */
    p->age[n] = p->age[n] + (double)(float)prm->idt;             /* 693 */

    uint32_t fl = 0;
    int gid = p->gid[n];
    step_env e = *e0;
    e.g = &grids[gid - 1];
    noise_ctx nc = {noise, p->pid ? p->pid[n] : (uint32_t)n};

    double Xpar = p->x[n], Ypar = p->y[n], Zpar = p->z[n];
    double pm = orc_getinterp2d(e.g, ORC_V_PM, Xpar, Ypar, 1, &fl);  /* 727 */
    double pn = orc_getinterp2d(e.g, ORC_V_PN, Xpar, Ypar, 1, &fl);
    double AdvectX = 0.0, AdvectY = 0.0, AdvectZ = 0.0;
    double TurbHx = 0.0, TurbHy = 0.0, TurbV = 0.0, ZBehav = 0.0;
    if (prm->scheme == 1)
        rk_advect(&e, Xpar, Ypar, &Zpar, pm, pn, &AdvectX, &AdvectY, &AdvectZ, &fl);
    if (prm->hturb_on) hturb(&e, gid, &nc, &TurbHx, &TurbHy);  /* 766 */
    TurbHx = TurbHx * pm;
    TurbHy = TurbHy * pn;
    if (prm->vturb_on) {                                         /* 783 */
        TurbV = vturb(&e, Xpar, Ypar, Zpar, &nc, w, &fl, n_iter);
        (*n_spline)++;
    }
    if (prm->behavior || prm->process_va || prm->process_wa) {     /* 800-804 */
        double behout[4];
        ZBehav = behave(&e, e.g, Xpar, Ypar, Zpar, &nc, behout, &fl);
        if (p->p_acc) {
            p->p_acc[n] = behout[0];
            p->p_vort[n] = behout[1];
            p->p_behavew[n] = behout[2];
            p->p_ssf[n] = behout[3];
        }
    }

    double newXpos = p->x[n] + AdvectX + TurbHx;                 /* 821 */
    double newYpos = p->y[n] + AdvectY + TurbHy;
    const orc_grid *gcur = &grids[gid - 1];
    double tempX = newXpos, tempY = newYpos;
    int ingrid = 0, obound = 0, nmask;
    for (int i = 1; i <= prm->ngrid; i++) {                     /* 828-836 */
        tempX = gcur->scl[i - 1][0] * newXpos + gcur->off[i - 1][0];
        tempY = gcur->scl[i - 1][1] * newYpos + gcur->off[i - 1][1];
        orc_bounds(&grids[i - 1], tempX, tempY, &nmask, &ingrid, &obound);
        if (ingrid) { gid = i; break; }
    }
    const orc_grid *gn = &grids[gid - 1];
    double tdepth = -1.0 * orc_getinterp2d(gn, ORC_V_DEPTH, tempX, tempY, e.tc, &fl);
    double ey[3];
    ey[0] = 1.0 * orc_getinterp2d(gn, ORC_V_ZETA, tempX, tempY, e.tb, &fl);
    ey[1] = 1.0 * orc_getinterp2d(gn, ORC_V_ZETA, tempX, tempY, e.tc, &fl);
    ey[2] = 1.0 * orc_getinterp2d(gn, ORC_V_ZETA, tempX, tempY, e.tf, &fl);
    double P_zeta = orc_polintd(e.ex, ey, e.ix[1]);              /* 843 */
    p->wd[n] = (-1.0 * tdepth) + P_zeta;
    p->zeta[n] = P_zeta;
    p->bath[n] = -1.0 * tdepth;
    int hbot = 0, htop = 0;
    double newZpos;
    switch (prm->nsb) {                                          /* 852-872 */
    case 0:
        newZpos = p->z[n] + AdvectZ + TurbV + ZBehav;
        if (newZpos < tdepth) { newZpos = tdepth + fabs(newZpos - tdepth); hbot = 1; }
        if (newZpos > P_zeta) { newZpos = P_zeta - fabs(newZpos - P_zeta); htop = 1; }
        break;
    case 1: newZpos = P_zeta - prm->vertdist; break;
    default: newZpos = tdepth + prm->vertdist; break;
    }
    if (ingrid) {                                                /* 874-892 */
        p->isin[n] = 1;
        p->x[n] = tempX;
        p->y[n] = tempY;
        p->z[n] = newZpos;
        p->status[n] = 1.0;
        if (htop) p->status[n] = F_1P1;
        if (hbot) p->status[n] = F_1P2;
        p->gid[n] = gid;
    } else if (obound) {
        p->isin[n] = 0;
        p->gid[n] = prm->ngrid;
        p->status[n] = -8.0;
    } else {
        p->isin[n] = 1;
        p->status[n] = -9.0;
    }
    if (prm->write_bottom) {                                     /* 935-952 */
        const orc_grid *gd = &grids[p->gid[n] - 1];
        double btemp = -1.0 * tdepth + p->z[n];
        p->p_hob[n] = (btemp < p->p_hob[n]) ? btemp : p->p_hob[n];
        if (btemp == p->p_hob[n]) {
            double eb[3];
            eb[0] = orc_getinterp_str(gd, ORC_V_BUSTR, p->x[n], p->y[n], e.tb, &fl);
            eb[1] = orc_getinterp_str(gd, ORC_V_BUSTR, p->x[n], p->y[n], e.tc, &fl);
            eb[2] = orc_getinterp_str(gd, ORC_V_BUSTR, p->x[n], p->y[n], e.tf, &fl);
            p->p_bustr[n] = orc_polintd(e.ex, eb, e.ix[1]);
            eb[0] = orc_getinterp_str(gd, ORC_V_BVSTR, p->x[n], p->y[n], e.tb, &fl);
            eb[1] = orc_getinterp_str(gd, ORC_V_BVSTR, p->x[n], p->y[n], e.tc, &fl);
            eb[2] = orc_getinterp_str(gd, ORC_V_BVSTR, p->x[n], p->y[n], e.tf, &fl);
            p->p_bvstr[n] = orc_polintd(e.ex, eb, e.ix[1]);
        }
    }
    if (prm->salttemp_on) {                                      /* 962-986 */
        const orc_grid *gd = &grids[p->gid[n] - 1];
        const double X = p->x[n], Y = p->y[n], Z = p->z[n];
        double zetab = orc_getinterp2d(gd, ORC_V_ZETA, X, Y, e.tb, &fl);
        double zetac = orc_getinterp2d(gd, ORC_V_ZETA, X, Y, e.tc, &fl);
        double zetaf = orc_getinterp2d(gd, ORC_V_ZETA, X, Y, e.tf, &fl);
        double es[3];
        es[0] = orc_getinterp3d(gd, ORC_V_SALT, X, Y, Z, e.tb, 1, zetab, tdepth, &fl);
        es[1] = orc_getinterp3d(gd, ORC_V_SALT, X, Y, Z, e.tc, 1, zetac, tdepth, &fl);
        es[2] = orc_getinterp3d(gd, ORC_V_SALT, X, Y, Z, e.tf, 1, zetaf, tdepth, &fl);
        p->p_salt[n] = orc_polintd(e.ex, es, e.ix[1]);
        es[0] = orc_getinterp3d(gd, ORC_V_TEMP, X, Y, Z, e.tb, 1, zetab, tdepth, &fl);
        es[1] = orc_getinterp3d(gd, ORC_V_TEMP, X, Y, Z, e.tc, 1, zetac, tdepth, &fl);
        es[2] = orc_getinterp3d(gd, ORC_V_TEMP, X, Y, Z, e.tf, 1, zetaf, tdepth, &fl);
        p->p_temp[n] = orc_polintd(e.ex, es, e.ix[1]);
        if (prm->salttemp_mean) {
            p->mean_salt[n] = p->mean_salt[n] + p->p_salt[n];
            p->mean_temp[n] = p->mean_temp[n] + p->p_temp[n];
        }
    }
    if (p->flags) p->flags[n] |= fl;
}

int orc_update_particles(const orc_params *prm, const orc_grid *grids, orc_particles *p,
                         const double ex[3], const double ix[3], int ets, int tb, int tc, int tf,
                         const orc_noise *noise, int nthreads)
{
    step_env e = {prm, grids, ex, ix, ets, tb, tc, tf};
    int maxsw = 0;
    for (int g = 0; g < prm->ngrid; g++) if (grids[g].N + 1 > maxsw) maxsw = grids[g].N + 1;
    int maxnp = (int)((double)maxsw * prm->sub) + 1;
    int64_t tot_spline = 0, tot_iter = 0;
    int err = 0;
    if (noise->kind == ORC_NOISE_MT || nthreads <= 1) {
        vt_work w;
        if (!vt_work_alloc(&w, maxsw, maxnp)) { vt_work_free(&w); return -1; }
        for (int64_t n = 0; n < p->n; n++) update_one(&e, grids, p, n, noise, &w, &tot_spline, &tot_iter);
        vt_work_free(&w);
    } else {
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads) reduction(+ : tot_spline, tot_iter) reduction(| : err)
        {
            vt_work w;
            if (!vt_work_alloc(&w, maxsw, maxnp)) err |= 1;
            else {
#pragma omp for schedule(dynamic, 64)
                for (int64_t n = 0; n < p->n; n++) update_one(&e, grids, p, n, noise, &w, &tot_spline, &tot_iter);
            }
            vt_work_free(&w);
        }
#else
        vt_work w;
        if (!vt_work_alloc(&w, maxsw, maxnp)) { vt_work_free(&w); return -1; }
        for (int64_t n = 0; n < p->n; n++) update_one(&e, grids, p, n, noise, &w, &tot_spline, &tot_iter);
        vt_work_free(&w);
#endif
    }
    g_spline_calls = tot_spline;
    g_secant_iters = tot_iter;
    return err ? -1 : 0;
}

/* ini_ROMSPath ownership loop, ROMSPath.f90:319-432 (positions already in
 * each grid's index space; LL2ij itself is init-time host work). */
int orc_init_particles(const orc_params *prm, const orc_grid *grids, orc_particles *p,
                       const double *ipos, const double *jpos, int tb, int tc)
{
    for (int64_t n = 0; n < p->n; n++) {
        p->status[n] = 9.0;
        p->age[n] = 0.0;
        p->gid[n] = prm->ngrid;
        p->isin[n] = 0;
        p->wd[n] = 9999.0;
        p->bath[n] = 9999.0;
        p->zeta[n] = 9999.0;
        p->x[n] = 1.0;
        p->y[n] = 1.0;
        if (p->flags) p->flags[n] = 0;
        if (prm->write_bottom) { p->p_hob[n] = 9999.0; p->p_bustr[n] = 0.0; p->p_bvstr[n] = 0.0; }  /* 260-264, 353-355 */
        if (prm->salttemp_on) {                                                                  /* 247-257 */
            p->p_salt[n] = 0.0; p->p_temp[n] = 0.0;
            if (prm->salttemp_mean) { p->mean_salt[n] = 0.0; p->mean_temp[n] = 0.0; }
        }
    }
    for (int ng = 1; ng <= prm->ngrid; ng++) {
        for (int64_t n = 0; n < p->n; n++) {
            double I = ipos[(int64_t)(ng - 1) * p->n + n], J = jpos[(int64_t)(ng - 1) * p->n + n];
            int nmask, ingrid, obound, inz;
            orc_bounds(&grids[ng - 1], I, J, &nmask, &ingrid, &obound);
            if (!p->isin[n] && ingrid) {
                uint32_t fl = 0;
                p->x[n] = I;
                p->y[n] = J;
                p->gid[n] = ng;
                p->status[n] = 0.0;
                p->isin[n] = 1;
                zbounds(&grids[ng - 1], I, J, &p->z[n], &inz, tb, &fl);
                if (!inz) p->status[n] = 9.0;
                if (p->flags) p->flags[n] |= fl;
            }
        }
    }
    if (prm->salttemp_on) {                                      /* 408-427 */
        for (int64_t n = 0; n < p->n; n++) {
            if (!p->isin[n]) continue;
            uint32_t fl = 0;
            const orc_grid *gd = &grids[p->gid[n] - 1];
            double tdepth = -1.0 * orc_getinterp2d(gd, ORC_V_DEPTH, p->x[n], p->y[n], tc, &fl);
            double zeta = orc_getinterp2d(gd, ORC_V_ZETA, p->x[n], p->y[n], tc, &fl);
            p->p_salt[n] = orc_getinterp3d(gd, ORC_V_SALT, p->x[n], p->y[n], p->z[n], tc, 1, zeta, tdepth, &fl);
            p->p_temp[n] = orc_getinterp3d(gd, ORC_V_TEMP, p->x[n], p->y[n], p->z[n], tc, 1, zeta, tdepth, &fl);
            p->wd[n] = (-1.0 * tdepth) + zeta;
            p->zeta[n] = zeta;
            p->bath[n] = -1.0 * tdepth;
            if (prm->salttemp_mean) { p->mean_salt[n] = p->p_salt[n]; p->mean_temp[n] = p->p_temp[n]; }
            if (p->flags) p->flags[n] |= fl;
        }
    }
    return 0;
}

/* dataOutput, ROMSPath.f90:1012-1024 */
void orc_output_lonlat(const orc_grid *grids, const orc_particles *p, double *lon, double *lat)
{
    for (int64_t n = 0; n < p->n; n++) {
        uint32_t fl = 0;
        const orc_grid *g = &grids[p->gid[n] - 1];
        lon[n] = orc_getinterp2d(g, ORC_V_LON, p->x[n], p->y[n], 1, &fl);
        lat[n] = orc_getinterp2d(g, ORC_V_LAT, p->x[n], p->y[n], 1, &fl);
    }
}

/* ======================= init lookup (LL2ij) ======================= */

#define ORC_PIO2_1 0x1.921fb54400000p+0     /* pi/2 in three parts; k * part */
#define ORC_PIO2_2 0x1.0b4611a600000p-34    /* is exact for |k| < 2^19      */
#define ORC_PIO2_3 0x1.3198a2e037073p-69
#define ORC_PIO2_HI 0x1.921fb54442d18p+0    /* pi/2 = HI + LO                */
#define ORC_PIO2_LO 0x1.1a62633145c07p-54
#define ORC_2_OVER_PI 0.6366197723675814

void orc_sincos(double x, double *s, double *c)
{
    const double k = rint(x * ORC_2_OVER_PI);
    const double r = ((x - k * ORC_PIO2_1) - k * ORC_PIO2_2) - k * ORC_PIO2_3;
    const double r2 = r * r;
    double p = -1.0 / 121645100408832000.0;        /* -1/19! */
    p = p * r2 + 1.0 / 355687428096000.0;           /*  1/17! */
    p = p * r2 - 1.0 / 1307674368000.0;
    p = p * r2 + 1.0 / 6227020800.0;
    p = p * r2 - 1.0 / 39916800.0;
    p = p * r2 + 1.0 / 362880.0;
    p = p * r2 - 1.0 / 5040.0;
    p = p * r2 + 1.0 / 120.0;
    p = p * r2 - 1.0 / 6.0;
    const double sr = r + (r * r2) * p;
    double q = 1.0 / 2432902008176640000.0;        /*  1/20! */
    q = q * r2 - 1.0 / 6402373705728000.0;
    q = q * r2 + 1.0 / 20922789888000.0;
    q = q * r2 - 1.0 / 87178291200.0;
    q = q * r2 + 1.0 / 479001600.0;
    q = q * r2 - 1.0 / 3628800.0;
    q = q * r2 + 1.0 / 40320.0;
    q = q * r2 - 1.0 / 720.0;
    q = q * r2 + 1.0 / 24.0;
    q = q * r2 - 0.5;
    const double cr = 1.0 + r2 * q;
    switch (((int)k) & 3) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
    }
}

/* asin t for 0 <= t <= 0.5 by its series sum c_n t^(2n+1), n <= 25 */
static double asin_series(double t)
{
    const double z = t * t;
    double p = 5267108601573.0 / 2392537302040576.0;
    p = p * z + 8061900920775.0 / 3448068464705536.0;
    p = p * z + 514589420475.0 / 206708186021888.0;
    p = p * z + 17534158031.0 / 6597069766656.0;
    p = p * z + 67282234305.0 / 23639499997184.0;
    p = p * z + 34461632205.0 / 11269994184704.0;
    p = p * z + 1472719325.0 / 446676598784.0;
    p = p * z + 2268783825.0 / 635655159808.0;
    p = p * z + 116680311.0 / 30064771072.0;
    p = p * z + 100180065.0 / 23622320128.0;
    p = p * z + 9694845.0 / 2080374784.0;
    p = p * z + 5014575.0 / 973078528.0;
    p = p * z + 1300075.0 / 226492416.0;
    p = p * z + 676039.0 / 104857600.0;
    p = p * z + 88179.0 / 12058624.0;
    p = p * z + 46189.0 / 5505024.0;
    p = p * z + 12155.0 / 1245184.0;
    p = p * z + 6435.0 / 557056.0;
    p = p * z + 143.0 / 10240.0;
    p = p * z + 231.0 / 13312.0;
    p = p * z + 63.0 / 2816.0;
    p = p * z + 35.0 / 1152.0;
    p = p * z + 5.0 / 112.0;
    p = p * z + 3.0 / 40.0;
    p = p * z + 1.0 / 6.0;
    return t + t * (z * p);
}

double orc_asin(double x)
{
    const double a = fabs(x);
    if (!(a <= 1.0)) return NAN;
    double r;
    if (a <= 0.5) {
        r = asin_series(a);
    } else {                                          /* asin a = pi/2 - 2 asin sqrt((1-a)/2) */
        const double t = sqrt((1.0 - a) * 0.5);
        r = (ORC_PIO2_HI - 2.0 * asin_series(t)) + ORC_PIO2_LO;
    }
    return (x < 0.0) ? -r : r;
}

/* inbox, interpolation_module.f90:232-268: the box's boundary polygon,
 * then inside() */
static int inbox(const orc_grid *g, int Li, int Ui, int Lj, int Uj, double inlon, double inlat, double *lonb,
                 double *latb)
{
    const int nx = g->xi_rho;
    const int Nb = 2 * (Uj - Lj + Ui - Li);
    int shft = 1 - Li;
    for (int i = Li; i <= Ui - 1; i++) {
        lonb[i + shft - 1] = g->lon_rho[IX2(i, Lj, nx)];
        latb[i + shft - 1] = g->lat_rho[IX2(i, Lj, nx)];
    }
    shft = 1 - Lj + Ui - Li;
    for (int j = Lj; j <= Uj - 1; j++) {
        lonb[j + shft - 1] = g->lon_rho[IX2(Ui, j, nx)];
        latb[j + shft - 1] = g->lat_rho[IX2(Ui, j, nx)];
    }
    shft = 1 + Uj - Lj + 2 * Ui - Li;
    for (int i = Ui; i >= Li + 1; i--) {
        lonb[shft - i - 1] = g->lon_rho[IX2(i, Uj, nx)];
        latb[shft - i - 1] = g->lat_rho[IX2(i, Uj, nx)];
    }
    shft = 1 + 2 * Uj - Lj + 2 * (Ui - Li);
    for (int j = Uj; j >= Lj + 1; j--) {
        lonb[shft - j - 1] = g->lon_rho[IX2(Li, j, nx)];
        latb[shft - j - 1] = g->lat_rho[IX2(Li, j, nx)];
    }
    return orc_inside(Nb, lonb, latb, inlon, inlat);
}

void orc_ll2ij(const orc_grid *g, int spherical, const double *inlon, const double *inlat, int64_t n,
               double *ipar, double *jpar)
{
    const int nx = g->xi_rho, ny = g->eta_rho;
    const double Eradius = 6371315.0, deg2rad = 3.14159265358979323846 / 180.0;   /* ROMSPath.h:11-13 */
    const size_t nbmax = 2 * (size_t)(nx + ny) + 2;
    double *lonb = (double *)malloc(nbmax * sizeof(double));
    double *latb = (double *)malloc(nbmax * sizeof(double));
    for (int64_t k = 0; k < n; k++) {
        const double lo = inlon[k], la = inlat[k];
        int Imin = 1, Imax = nx, Jmin = 1, Jmax = ny;
        int found = inbox(g, Imin, Imax, Jmin, Jmax, lo, la, lonb, latb);
        if (found) {                                             /* 138-159 */
            while (((Imax - Imin) > 1) || ((Jmax - Jmin) > 1)) {
                if ((Imax - Imin) > 1) {
                    const int i0 = (Imin + Imax) / 2;
                    if (inbox(g, Imin, i0, Jmin, Jmax, lo, la, lonb, latb)) Imax = i0;
                    else Imin = i0;
                }
                if ((Jmax - Jmin) > 1) {
                    const int j0 = (Jmin + Jmax) / 2;
                    if (inbox(g, Imin, Imax, Jmin, j0, lo, la, lonb, latb)) Jmax = j0;
                    else Jmin = j0;
                }
            }
        }
        found = inbox(g, Imin, Imax, Jmin, Jmax, lo, la, lonb, latb);   /* 166-168 */
        if (spherical == 0) {                                    /* 173-183 */
            const double xmin = g->lon_rho[IX2(Imin, Jmin, nx)], xmax = g->lon_rho[IX2(Imax, Jmax, nx)];
            const double ymin = g->lat_rho[IX2(Imin, Jmin, nx)], ymax = g->lat_rho[IX2(Imax, Jmax, nx)];
            const double xfac = ((double)Imax - (double)Imin) / (xmax - xmin);
            const double yfac = ((double)Jmax - (double)Jmin) / (ymax - ymin);
            const double dx = (lo - xmin) * xfac;
            const double dy = (la - ymin) * yfac;
            ipar[k] = (double)Imin + dx;
            jpar[k] = (double)Jmin + dy;
        } else if (found) {                                      /* 184-214 */
            const double yfac = Eradius * deg2rad;
            double sl, cl;
            orc_sincos(la * deg2rad, &sl, &cl);
            const double xfac = yfac * cl;
            const double l00 = g->lon_rho[IX2(Imin, Jmin, nx)], t00 = g->lat_rho[IX2(Imin, Jmin, nx)];
            const double l10 = g->lon_rho[IX2(Imin + 1, Jmin, nx)], t10 = g->lat_rho[IX2(Imin + 1, Jmin, nx)];
            const double l01 = g->lon_rho[IX2(Imin, Jmin + 1, nx)], t01 = g->lat_rho[IX2(Imin, Jmin + 1, nx)];
            const double xpp = (lo - l00) * xfac;
            const double ypp = (la - t00) * yfac;
            const double d1 = (l10 - l01) * xfac, d2 = (t10 - t01) * yfac;
            const double diag2 = d1 * d1 + d2 * d2;
            const double a1 = (l00 - l10) * xfac, a2 = (t00 - t10) * yfac;
            const double aa2 = a1 * a1 + a2 * a2;
            const double b1 = (l00 - l01) * xfac, b2 = (t00 - t01) * yfac;
            const double bb2 = b1 * b1 + b2 * b2;
            const double phi = orc_asin((diag2 - aa2 - bb2) / (2.0 * sqrt(aa2 * bb2)));
            const double ang = g->angle[IX2(Imin, Jmin, nx)];
            double sa, ca, sp, cp;
            orc_sincos(ang, &sa, &ca);
            orc_sincos(phi, &sp, &cp);
            double dx = xpp * ca + ypp * sa;
            double dy = ypp * ca - xpp * sa;
            dx = dx + dy * (sp / cp);                            /* TAN(phi) */
            dy = dy / cp;
            dx = dx / sqrt(aa2);
            dx = (dx > 0.0) ? dx : 0.0;                          /* MIN(MAX(0.0, .), 1.0) */
            dx = (dx < 1.0) ? dx : 1.0;
            dy = dy / sqrt(bb2);
            dy = (dy > 0.0) ? dy : 0.0;
            dy = (dy < 1.0) ? dy : 1.0;
            ipar[k] = (double)Imin + dx;
            jpar[k] = (double)Jmin + dy;
        } else {
            ipar[k] = -1.0;
            jpar[k] = -1.0;
        }
    }
    free(lonb);
    free(latb);
}

void orc_nest_maps(int ngrid, const orc_grid *grids, const double *refine, double *scl, double *off)
{
    double grefine[ORC_MAXNGRID][ORC_MAXNGRID];
    for (int a = 0; a < ngrid; a++)                              /* 437-450 */
        for (int b = 0; b < ngrid; b++) {
            grefine[a][b] = 1.0;
            const int dng = abs(a - b);
            for (int r = 1; r <= dng; r++) grefine[a][b] = refine[dng - 1] * grefine[a][b];
        }
    for (int k = 0; k < ngrid * 2 * ngrid; k++) { scl[k] = 1.0; off[k] = 0.0; }
#define SCL(ng, c, i) scl[((ng) * 2 + (c)) * ngrid + (i)]
#define OFF(ng, c, i) off[((ng) * 2 + (c)) * ngrid + (i)]
    for (int ng2 = 0; ng2 < ngrid; ng2++) {                      /* 454-481 */
        for (int ng = 0; ng < ngrid; ng++) {
            const orc_grid *A = &grids[ng], *B = &grids[ng2];
            int i, j = 1, ii = 1, jj = 1, hit = 0;
            for (i = 1; i <= A->xi_rho && !hit; i++) {
                for (j = 1; j <= A->eta_rho && !hit; j++) {
                    for (ii = 1; ii <= B->xi_rho && !hit; ii++) {
                        for (jj = 1; jj <= B->eta_rho; jj++) {
                            if (A->lon_rho[IX2(i, j, A->xi_rho)] == B->lon_rho[IX2(ii, jj, B->xi_rho)] &&
                                A->lat_rho[IX2(i, j, A->xi_rho)] == B->lat_rho[IX2(ii, jj, B->xi_rho)]) {
                                hit = 1;
                                break;
                            }
                        }
                        if (hit) break;
                    }
                    if (hit) break;
                }
                if (hit) break;
            }
            /* no coincident point: the indices past the loops' ends, as
             * Fortran leaves them after complete DO loops */
            for (int c = 0; c < 2; c++) {
                SCL(ng, c, ng2) = 1.0 / grefine[ng][ng2];
                SCL(ng2, c, ng) = grefine[ng2][ng];
            }
            OFF(ng, 0, ng2) = (double)ii - SCL(ng, 0, ng2) * (double)i;
            OFF(ng, 1, ng2) = (double)jj - SCL(ng, 1, ng2) * (double)j;
            OFF(ng2, 0, ng) = (double)i - SCL(ng2, 0, ng) * (double)ii;
            OFF(ng2, 1, ng) = (double)j - SCL(ng2, 1, ng) * (double)jj;
        }
    }
#undef SCL
#undef OFF
}
