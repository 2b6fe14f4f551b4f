"""Well-mixed-condition study of the random displacement model (VTurb).

Visser (1997; cited at ver_turb_module.f90:19): particles spread uniformly
over the water column must stay uniform under the random displacement
model with a non-uniform diffusivity.  This script runs the oracle's
restatement of the reference's VTurb (ver_turb_module.f90:31-329) with
advection and horizontal turbulence off, on the analytic frames of the
test grids, under variants that change one ingredient at a time, and prints
the chi-square of the final distribution over 20 equal bins of the
water-column fraction (z + h) / (h + zeta) (19 degrees of freedom: 43.8 is
the p = 0.001 point):

  reference     the reference's algorithm (dy(1) = dy(np) = serr pinned)
  dy_end=0      dy(1) = dy(np) = 0 (the value uninitialised memory often holds)
  dy_end=1e-2   dy(1) = dy(np) = 100 serr
  analytic      the smoothing-spline fit replaced by the exact parabola
                K = c 4 xi (1 - xi) fitted to the column, and its K'
  deltat=3      sub-step 3 s instead of 30 s (100 sub-steps per step)
  analytic, deltat=3
  steady        a steady column: no tide (zeta = 0) and a constant peak
                diffusivity, so the water column neither moves nor changes
  steady, analytic, deltat=3

The oracle is test infrastructure; this script only drives it.  Usage:

    python oracle/wmc_study.py [--grid tiny|cfg1] [--n 20000] [--days 2] [--only NAME]
                               [--release test|full]
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import harness  # noqa: E402
from romspath_b200 import synth  # noqa: E402

VARIANTS = {
    "reference": ({}, False),
    "dy_end=0": ({"vt_dy_end": 0.0}, False),
    "dy_end=1e-2": ({"vt_dy_end": 1e-2}, False),
    "analytic": ({"vt_variant": 1}, False),
    "deltat=3": ({"deltat": 3.0}, False),
    "analytic, deltat=3": ({"vt_variant": 1, "deltat": 3.0}, False),
    "steady": ({}, True),
    "steady, analytic": ({"vt_variant": 1}, True),
    "steady, deltat=3": ({"deltat": 3.0}, True),
    "steady, analytic, deltat=3": ({"vt_variant": 1, "deltat": 3.0}, True),
}


def steady_frame(spec, grid, t):
    """The analytic frame at time t with zeta = 0 and AKs = 1e-2 4 xi (1 - xi)."""
    f = dict(synth.make_frame(spec, grid, t))
    h = grid["h"]
    zeta = np.zeros_like(h)
    S_w = synth._stretch_S(h, grid["s_w"], grid["cs_w"], spec.hc)
    z_w = synth._zlevels(zeta, h, S_w)
    xi = (z_w + h[..., None]) / h[..., None]
    aks = np.clip(1e-2 * 4.0 * xi * (1.0 - xi), 0.0, None) * grid["mask_rho"][..., None]
    dt = f["aks"].dtype
    f["zeta"] = np.asfortranarray(zeta.astype(dt))
    f["aks"] = np.asfortranarray(aks.astype(dt))
    return f


def chi2_of(st):
    rel = (st["z"] + st["bath"]) / (st["bath"] + st["zeta"])
    counts, _ = np.histogram(rel, bins=20, range=(0.0, 1.0))
    exp = len(rel) / 20.0
    return float(((counts - exp) ** 2 / exp).sum()), counts / exp


def _bil(a, rel):
    I = np.floor(rel.ipos[0]).astype(int) - 1
    J = np.floor(rel.jpos[0]).astype(int) - 1
    fx, fy = rel.ipos[0] - np.floor(rel.ipos[0]), rel.jpos[0] - np.floor(rel.jpos[0])
    return ((1 - fx) * (1 - fy) * a[I, J] + fx * (1 - fy) * a[I + 1, J]
            + fx * fy * a[I + 1, J + 1] + (1 - fx) * fy * a[I, J + 1])


def run(grid: str, n: int, days: float, name: str, threads: int, release: str = "test"):
    """release "test": the tests' release, uniform in s over (-0.98, -0.02),
    i.e. the bottom and top 2 % of the column start empty; "full": uniform
    over the whole column."""
    over, steady = VARIANTS[name]
    params = {"scheme": 0, "hturb_on": 0}
    params.update(over)
    case = harness.make_case(grid, n, seed=9, spec_over={"land": "none"}, param_over=params)
    nsteps = int(round(days * 86400 / case.params["idt"]))
    if steady:
        for k in range(1, nsteps // 12 + 4):
            case.frames[(1, k)] = steady_frame(case.spec, case.grid, (k - 1) * float(case.params["dt"]))
    if steady or release == "full":
        # depths drawn from the frame-1 column, independent of the positions
        rel = case.release
        hb = _bil(case.grid["h"], rel)
        zt = _bil(case.frame(1)["zeta"].astype(np.float64), rel)
        lo, hi = (-0.98, -0.02) if release == "test" else (-1.0, 0.0)
        s = np.random.default_rng(1009).uniform(lo, hi, n)
        rel.z = zt + (zt + hb) * s
    t0 = time.time()
    o, _ = harness.run_oracle(case, nsteps, noise="philox", seed=21, nthreads=threads)
    c2, prof = chi2_of(o)
    return c2, prof, time.time() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", default="tiny")
    ap.add_argument("--n", type=int, default=20000)
    ap.add_argument("--days", type=float, default=2.0)
    ap.add_argument("--only", default=None)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--release", default="test", choices=["test", "full"])
    a = ap.parse_args()
    names = [a.only] if a.only else list(VARIANTS)
    print(f"grid {a.grid}, {a.n} particles, {a.days} days, release {a.release}, 20 bins "
          f"(chi2 p=0.001 at 43.8)")
    for name in names:
        c2, prof, sec = run(a.grid, a.n, a.days, name, a.threads, a.release)
        ends = f"bottom {prof[0]:.3f} {prof[1]:.3f} ... top {prof[-2]:.3f} {prof[-1]:.3f}"
        print(f"| {name} | {c2:.1f} | {ends} | {sec:.0f} s |", flush=True)


if __name__ == "__main__":
    main()
