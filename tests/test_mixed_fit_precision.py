"""Precision margin of the mixed form's smoothing-spline pass (CPU).

The mixed form's chol1d pass (romspath_b200/csrc/rp_mixed.cuh, m_chol1d;
pppack.f90:1428-1566 on uniform breaks) factorises the pentadiagonal matrix
of smooth() in FP64 until its ratios repeat in FP32, stores the ratios in
FP32, and runs the forward and back substitutions and the sum of squares in
FP32.  This test restates that arithmetic in numpy (float32 for the sweeps)
and compares it with an FP64 solve of the same system over column spacings
h from 0.02 to 20 m and smoothing parameters q from 1e-16 to 100 on rough
AKs-like columns: the SF that smooth()'s secant search compares against
its 1 % band must stay well inside that band, and u (the fit's second
derivatives, which ppvalu evaluates) must stay close.
"""
import numpy as np

F32 = np.float32
SERR = 1e-4


def _bands(h, p):
    r = SERR / h
    r2 = r * r
    six = 6.0 * (1.0 - p)
    return six * 6.0 * r2 + 4.0 * p * h, six * (-4.0 * r2) + p * h, six * r2


def _sf(uu, h):
    raw = np.diff(uu) / h
    qu = np.diff(np.concatenate([[0.0], raw, [0.0]]))
    return float(np.sum(qu * qu) * SERR * SERR)


def _solve_fp64(y, h, p):
    n = len(y) - 2
    D, E, F = _bands(h, p)
    M = (np.diag(np.full(n, D)) + np.diag(np.full(n - 1, E), 1) + np.diag(np.full(n - 1, E), -1)
         + np.diag(np.full(n - 2, F), 2) + np.diag(np.full(n - 2, F), -2))
    u = np.linalg.solve(M, (y[2:] - 2.0 * y[1:-1] + y[:-2]) / h)
    uu = np.concatenate([[0.0], u, [0.0]])
    return uu, _sf(uu, h)


def _solve_mixed(y, h, p):
    """m_chol1d's scheme: FP64 leading factor rows rounded to FP32 until
    they repeat, then held; FP32 data, substitutions and u."""
    npt = len(y)
    D, E, F = _bands(h, p)
    rhf = F32(1.0 / h)
    yf = y.astype(F32)
    a1, a2, b1 = D, E, D
    ks, prev, held = npt - 1, None, None
    s1, s2, uq = {}, {}, {}
    ucur, uprev, r2prev = (yf[2] - F32(2) * yf[1] + yf[0]) * rhf, F32(0), F32(0)
    for i in range(2, npt - 1):                       # rows 2..np-2 (1-based)
        if i < ks or i == npt - 2:
            Fi = F if i <= npt - 3 else 0.0
            inv = 1.0 / a1
            ra1, ra2 = a2 * inv, Fi * inv
            q = (F32(ra1), F32(ra2))
            if 2 < i < npt - 2 and q == prev:
                ks, held = i, (F32(inv), q[0], q[1])
                invf, r1f, r2f = held
            else:
                s1[i], s2[i] = q
                a1, a2, b1 = b1 - ra1 * a2, E - ra1 * Fi, D - ra2 * Fi
                invf, r1f, r2f = F32(inv), q[0], q[1]
            prev = q
        else:
            invf, r1f, r2f = held
        uq[i] = ucur * invf
        qn = (yf[i + 1] - F32(2) * yf[i] + yf[i - 1]) * rhf
        uprev, ucur, r2prev = ucur, qn - r1f * ucur - r2prev * uprev, r2f
    u = np.zeros(npt + 1, dtype=F32)
    u[npt - 1] = F32(float(ucur) / a1)
    up1, up2 = u[npt - 1], F32(0)
    for i in range(npt - 2, 1, -1):
        r1f, r2f = (held[1], held[2]) if ks <= i <= npt - 3 else (s1[i], s2[i])
        ui = uq[i] - up1 * r1f - up2 * r2f
        u[i] = ui
        up2, up1 = up1, ui
    uu = u[1:npt + 1].astype(np.float64)
    return uu, _sf(uu, h)


def test_fp32_sweeps_stay_inside_the_secant_band():
    rng = np.random.default_rng(7)
    worst_sf = worst_u = 0.0
    for h in (0.02, 0.1, 0.5, 1.6, 5.0, 20.0):
        for q in (1e-16, 1e-13, 1e-10, 1e-8, 1e-6, 1e-3, 1.0, 100.0):
            p = q / (1.0 + q)
            for trial in range(3):
                z = np.linspace(0.0, 1.0, 124)
                y = 1e-3 + 1e-2 * np.abs(np.sin(3.0 * z + trial)) * (1.0 + 0.3 * rng.standard_normal(124))
                y = np.clip(y, 0.0, None)
                u64, sf64 = _solve_fp64(y, h, p)
                u32, sf32 = _solve_mixed(y, h, p)
                worst_sf = max(worst_sf, abs(sf32 - sf64) / sf64)
                worst_u = max(worst_u, float(np.max(np.abs(u32 - u64)) / np.max(np.abs(u64))))
    print("worst SF relative error %.2e, worst u relative error %.2e" % (worst_sf, worst_u))
    assert worst_sf < 1e-3        # smooth() accepts |SF - s| <= 1e-2 s
    assert worst_u < 1e-2
