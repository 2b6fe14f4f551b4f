// rp_geo.cuh -- the init lookup on the device: LL2ij (interpolation_module.
// f90:110-231) with inbox (232-268) and inside (269-420), and the sin, cos
// and asin it needs.  The series and reductions are this project's own and
// run the same operations as the oracle's orc_sincos / orc_asin /
// orc_ll2ij, so the fractional indices are bit-identical.
#pragma once

#include "rp_device.cuh"

#define RP_PIO2_1 0x1.921fb54400000p+0     // pi/2 in three parts; k * part
#define RP_PIO2_2 0x1.0b4611a600000p-34    // is exact for |k| < 2^19
#define RP_PIO2_3 0x1.3198a2e037073p-69
#define RP_PIO2_HI 0x1.921fb54442d18p+0    // pi/2 = HI + LO
#define RP_PIO2_LO 0x1.1a62633145c07p-54
#define RP_2_OVER_PI 0.6366197723675814

// sin and cos: x = k pi/2 + r, Taylor series of sin r to r^19 and of cos r
// to r^20, then the quadrant of k.
__device__ __forceinline__ void rp_sincos(double x, double& s, double& c) {
    const double k = rint(RP_MUL(x, RP_2_OVER_PI));
    const double r = RP_SUB(RP_SUB(RP_SUB(x, RP_MUL(k, RP_PIO2_1)), RP_MUL(k, RP_PIO2_2)), RP_MUL(k, RP_PIO2_3));
    const double r2 = RP_MUL(r, r);
    double p = -1.0 / 121645100408832000.0;       // -1/19!
    p = RP_ADD(RP_MUL(p, r2), 1.0 / 355687428096000.0);
    p = RP_SUB(RP_MUL(p, r2), 1.0 / 1307674368000.0);
    p = RP_ADD(RP_MUL(p, r2), 1.0 / 6227020800.0);
    p = RP_SUB(RP_MUL(p, r2), 1.0 / 39916800.0);
    p = RP_ADD(RP_MUL(p, r2), 1.0 / 362880.0);
    p = RP_SUB(RP_MUL(p, r2), 1.0 / 5040.0);
    p = RP_ADD(RP_MUL(p, r2), 1.0 / 120.0);
    p = RP_SUB(RP_MUL(p, r2), 1.0 / 6.0);
    const double sr = RP_ADD(r, RP_MUL(RP_MUL(r, r2), p));
    double q = 1.0 / 2432902008176640000.0;       // 1/20!
    q = RP_SUB(RP_MUL(q, r2), 1.0 / 6402373705728000.0);
    q = RP_ADD(RP_MUL(q, r2), 1.0 / 20922789888000.0);
    q = RP_SUB(RP_MUL(q, r2), 1.0 / 87178291200.0);
    q = RP_ADD(RP_MUL(q, r2), 1.0 / 479001600.0);
    q = RP_SUB(RP_MUL(q, r2), 1.0 / 3628800.0);
    q = RP_ADD(RP_MUL(q, r2), 1.0 / 40320.0);
    q = RP_SUB(RP_MUL(q, r2), 1.0 / 720.0);
    q = RP_ADD(RP_MUL(q, r2), 1.0 / 24.0);
    q = RP_SUB(RP_MUL(q, r2), 0.5);
    const double cr = RP_ADD(1.0, RP_MUL(r2, q));
    switch (((int)k) & 3) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = -sr; break;
        case 2: s = -sr; c = -cr; break;
        default: s = -cr; c = sr; break;
    }
}

// asin t for 0 <= t <= 0.5: sum of c_n t^(2n+1), c_n = (2n)! / (4^n (n!)^2
// (2n+1)), n <= 25, each coefficient the rounded quotient of its exact
// numerator and denominator
__device__ __forceinline__ double rp_asin_series(double t) {
    const double z = RP_MUL(t, t);
    double p = 5267108601573.0 / 2392537302040576.0;
    p = RP_ADD(RP_MUL(p, z), 8061900920775.0 / 3448068464705536.0);
    p = RP_ADD(RP_MUL(p, z), 514589420475.0 / 206708186021888.0);
    p = RP_ADD(RP_MUL(p, z), 17534158031.0 / 6597069766656.0);
    p = RP_ADD(RP_MUL(p, z), 67282234305.0 / 23639499997184.0);
    p = RP_ADD(RP_MUL(p, z), 34461632205.0 / 11269994184704.0);
    p = RP_ADD(RP_MUL(p, z), 1472719325.0 / 446676598784.0);
    p = RP_ADD(RP_MUL(p, z), 2268783825.0 / 635655159808.0);
    p = RP_ADD(RP_MUL(p, z), 116680311.0 / 30064771072.0);
    p = RP_ADD(RP_MUL(p, z), 100180065.0 / 23622320128.0);
    p = RP_ADD(RP_MUL(p, z), 9694845.0 / 2080374784.0);
    p = RP_ADD(RP_MUL(p, z), 5014575.0 / 973078528.0);
    p = RP_ADD(RP_MUL(p, z), 1300075.0 / 226492416.0);
    p = RP_ADD(RP_MUL(p, z), 676039.0 / 104857600.0);
    p = RP_ADD(RP_MUL(p, z), 88179.0 / 12058624.0);
    p = RP_ADD(RP_MUL(p, z), 46189.0 / 5505024.0);
    p = RP_ADD(RP_MUL(p, z), 12155.0 / 1245184.0);
    p = RP_ADD(RP_MUL(p, z), 6435.0 / 557056.0);
    p = RP_ADD(RP_MUL(p, z), 143.0 / 10240.0);
    p = RP_ADD(RP_MUL(p, z), 231.0 / 13312.0);
    p = RP_ADD(RP_MUL(p, z), 63.0 / 2816.0);
    p = RP_ADD(RP_MUL(p, z), 35.0 / 1152.0);
    p = RP_ADD(RP_MUL(p, z), 5.0 / 112.0);
    p = RP_ADD(RP_MUL(p, z), 3.0 / 40.0);
    p = RP_ADD(RP_MUL(p, z), 1.0 / 6.0);
    return RP_ADD(t, RP_MUL(t, RP_MUL(z, p)));
}

// asin x = pi/2 - 2 asin sqrt((1 - |x|) / 2) above |x| = 0.5
__device__ __forceinline__ double rp_asin(double x) {
    const double a = fabs(x);
    if (!(a <= 1.0)) return __longlong_as_double(0x7ff8000000000000ll);
    double r;
    if (a <= 0.5) {
        r = rp_asin_series(a);
    } else {
        const double t = sqrt(RP_MUL(RP_SUB(1.0, a), 0.5));
        r = RP_ADD(RP_SUB(RP_PIO2_HI, RP_MUL(2.0, rp_asin_series(t))), RP_PIO2_LO);
    }
    return (x < 0.0) ? -r : r;
}

// Vertex k (1..Nb) of inbox's boundary polygon of the box [Li,Ui]x[Lj,Uj]:
// the bottom row left to right, the right column upwards, the top row
// right to left, the left column downwards (interpolation_module.f90:244-264).
__device__ __forceinline__ void rp_box_vertex(const double* lon, const double* lat, int nx, int Li, int Ui, int Lj,
                                              int Uj, int k, double& x, double& y) {
    const int a = Ui - Li, b = Uj - Lj;
    int i, j;
    if (k <= a) {
        i = Li + k - 1; j = Lj;
    } else if (k <= a + b) {
        i = Ui; j = Lj + (k - a) - 1;
    } else if (k <= 2 * a + b) {
        i = Ui - (k - a - b) + 1; j = Uj;
    } else {
        i = Li; j = Uj - (k - 2 * a - b) + 1;
    }
    const int64_t o = (int64_t)(j - 1) * nx + (i - 1);
    x = __ldg(lon + o);
    y = __ldg(lat + o);
}

// inbox: inside() over the box's boundary, the vertices generated in turn
__device__ __forceinline__ bool rp_inbox(const double* lon, const double* lat, int nx, int Li, int Ui, int Lj, int Uj,
                                         double xo, double yo) {
    const int nb = 2 * (Uj - Lj + Ui - Li);
    double x0, y0;
    rp_box_vertex(lon, lat, nx, Li, Ui, Lj, Uj, 1, x0, y0);
    const double xs = x0, ys = y0;
    int crossings = 0;
    for (int k = 1; k <= nb; k++) {
        double x1, y1;
        if (k < nb) {
            rp_box_vertex(lon, lat, nx, Li, Ui, Lj, Uj, k + 1, x1, y1);
        } else {
            x1 = xs;
            y1 = ys;
        }
        if ((RP_MUL(RP_SUB(x1, xo), RP_SUB(xo, x0)) >= 0.0) && (x0 != x1)) {
            const double dx1 = RP_SUB(xo, x0);
            const double dx2 = RP_SUB(x1, xo);
            const double dxy = RP_SUB(RP_MUL(dx2, RP_SUB(yo, y0)), RP_MUL(dx1, RP_SUB(y1, yo)));
            int inc = 0;
            if ((x0 == xo) && (y0 == yo)) {
                return true;
            } else if (((dx1 == 0.0) && (yo >= y0)) || ((dx2 == 0.0) && (yo >= y1))) {
                inc = 1;
            } else if ((RP_MUL(dx1, dx2) > 0.0) && (RP_MUL(RP_SUB(x1, x0), dxy) >= 0.0)) {
                inc = 2;
            }
            if (x1 > x0) crossings += inc;
            else crossings -= inc;
        }
        x0 = x1;
        y0 = y1;
    }
    return crossings != 0;
}

// LL2ij of one particle in one grid (spherical: GRIDS(1)%spherical)
__device__ __forceinline__ void rp_ll2ij_one(const double* lon, const double* lat, const double* angle, int nx,
                                             int ny, int spherical, double lo, double la, double& ip, double& jp) {
    const double Eradius = 6371315.0, deg2rad = 3.14159265358979323846 / 180.0;   // ROMSPath.h:11-13
    int Imin = 1, Imax = nx, Jmin = 1, Jmax = ny;
    bool found = rp_inbox(lon, lat, nx, Imin, Imax, Jmin, Jmax, lo, la);
    if (found) {                                           // 138-159
        while (((Imax - Imin) > 1) || ((Jmax - Jmin) > 1)) {
            if ((Imax - Imin) > 1) {
                const int i0 = (Imin + Imax) / 2;
                if (rp_inbox(lon, lat, nx, Imin, i0, Jmin, Jmax, lo, la)) Imax = i0;
                else Imin = i0;
            }
            if ((Jmax - Jmin) > 1) {
                const int j0 = (Jmin + Jmax) / 2;
                if (rp_inbox(lon, lat, nx, Imin, Imax, Jmin, j0, lo, la)) Jmax = j0;
                else Jmin = j0;
            }
        }
    }
    found = rp_inbox(lon, lat, nx, Imin, Imax, Jmin, Jmax, lo, la);   // 166-168
    auto at = [&](const double* a, int i, int j) { return __ldg(a + (int64_t)(j - 1) * nx + (i - 1)); };
    if (spherical == 0) {                                  // 173-183
        const double xmin = at(lon, Imin, Jmin), xmax = at(lon, Imax, Jmax);
        const double ymin = at(lat, Imin, Jmin), ymax = at(lat, Imax, Jmax);
        const double xfac = RP_SUB((double)Imax, (double)Imin) / RP_SUB(xmax, xmin);
        const double yfac = RP_SUB((double)Jmax, (double)Jmin) / RP_SUB(ymax, ymin);
        ip = RP_ADD((double)Imin, RP_MUL(RP_SUB(lo, xmin), xfac));
        jp = RP_ADD((double)Jmin, RP_MUL(RP_SUB(la, ymin), yfac));
    } else if (found) {                                    // 184-214
        const double yfac = RP_MUL(Eradius, deg2rad);
        double sl, cl;
        rp_sincos(RP_MUL(la, deg2rad), sl, cl);
        const double xfac = RP_MUL(yfac, cl);
        const double l00 = at(lon, Imin, Jmin), t00 = at(lat, Imin, Jmin);
        const double l10 = at(lon, Imin + 1, Jmin), t10 = at(lat, Imin + 1, Jmin);
        const double l01 = at(lon, Imin, Jmin + 1), t01 = at(lat, Imin, Jmin + 1);
        const double xpp = RP_MUL(RP_SUB(lo, l00), xfac);
        const double ypp = RP_MUL(RP_SUB(la, t00), yfac);
        const double d1 = RP_MUL(RP_SUB(l10, l01), xfac), d2 = RP_MUL(RP_SUB(t10, t01), yfac);
        const double diag2 = RP_ADD(RP_MUL(d1, d1), RP_MUL(d2, d2));
        const double a1 = RP_MUL(RP_SUB(l00, l10), xfac), a2 = RP_MUL(RP_SUB(t00, t10), yfac);
        const double aa2 = RP_ADD(RP_MUL(a1, a1), RP_MUL(a2, a2));
        const double b1 = RP_MUL(RP_SUB(l00, l01), xfac), b2 = RP_MUL(RP_SUB(t00, t01), yfac);
        const double bb2 = RP_ADD(RP_MUL(b1, b1), RP_MUL(b2, b2));
        const double phi = rp_asin(RP_SUB(RP_SUB(diag2, aa2), bb2) / RP_MUL(2.0, sqrt(RP_MUL(aa2, bb2))));
        double sa, ca, sp, cp;
        rp_sincos(at(angle, Imin, Jmin), sa, ca);
        rp_sincos(phi, sp, cp);
        double dx = RP_ADD(RP_MUL(xpp, ca), RP_MUL(ypp, sa));
        double dy = RP_SUB(RP_MUL(ypp, ca), RP_MUL(xpp, sa));
        dx = RP_ADD(dx, RP_MUL(dy, sp / cp));              // TAN(phi)
        dy = dy / cp;
        dx = dx / sqrt(aa2);
        dx = (dx > 0.0) ? dx : 0.0;                        // MIN(MAX(0.0, .), 1.0)
        dx = (dx < 1.0) ? dx : 1.0;
        dy = dy / sqrt(bb2);
        dy = (dy > 0.0) ? dy : 0.0;
        dy = (dy < 1.0) ? dy : 1.0;
        ip = RP_ADD((double)Imin, dx);
        jp = RP_ADD((double)Jmin, dy);
    } else {
        ip = -1.0;
        jp = -1.0;
    }
}
