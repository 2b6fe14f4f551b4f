"""GPU parity of the init lookup from particle lon/lat (rp_locate_lonlat:
LL2ij, interpolation_module.f90:110-268, then the ownership loop of
ini_ROMSPath): LL2ij's fractional indices and the located state against the
oracle bit for bit, on spherical and Cartesian grids and nested grids, then
steps from that state."""
import numpy as np
import pytest

import harness
from romspath_b200 import Tracker, schedule

pytestmark = pytest.mark.gpu


def _bilinear(a, ip, jp):
    I, J = np.floor(ip).astype(int), np.floor(jp).astype(int)
    X, Y = ip - I, jp - J
    return ((1 - X) * (1 - Y) * a[I - 1, J - 1] + X * (1 - Y) * a[I, J - 1] + X * Y * a[I, J]
            + (1 - X) * Y * a[I - 1, J])


def _release(case, n, seed):
    """lon/lat inside the outermost grid (the last one), plus a few outside"""
    rng = np.random.default_rng(seed)
    sp, g = case.specs[-1], case.grids[-1]
    ip = rng.uniform(1.0, sp.xi_rho - 1e-6, n)
    jp = rng.uniform(1.0, sp.eta_rho - 1e-6, n)
    lon, lat = _bilinear(g["lon_rho"], ip, jp), _bilinear(g["lat_rho"], ip, jp)
    lon[:5] = lon[:5] + 5.0                     # off every grid
    z = -rng.uniform(0.5, 15.0, n)
    dob = np.zeros(n)
    return lon, lat, z, dob


def _run(case, n, nsteps, spherical, seed=4):
    from oracle import oracle as O
    lon, lat, z, dob = _release(case, n, seed)
    params = dict(case.params, spherical=spherical)
    T = Tracker(case.specs, case.grids, params, numpar=n, seed=7, scl=case.scl, off=case.off)
    m = O.OracleModel(case.specs, case.grids, params, scl=case.scl, off=case.off)
    for (k, slot) in schedule.initial_loads():
        for ng in range(1, case.ngrid + 1):
            T.upload_frame(ng, slot, case.frame(k, ng))
            m.set_frame(ng, slot, case.stored(k, ng))
    gi, gj = T.locate_lonlat(lon, lat, z, dob)
    oi, oj = m.locate_lonlat(lon, lat, z, dob, spherical=spherical)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gj, oj)
    g0 = T.get_particles()
    o0 = m.state()
    o0["gid"] = o0["gid"].astype(np.float64)
    o0["isin"] = o0["isin"].astype(np.int32)
    diff = {k: v for k, v in harness.compare(g0, o0).items() if v}
    assert not diff, f"located state differs: {diff}"
    done = 0
    for ext, internal in harness._steps(case, nsteps):
        for (k, slot) in ext.loads:
            for ng in range(1, case.ngrid + 1):
                T.upload_frame(ng, slot, case.frame(k, ng))
                m.set_frame(ng, slot, case.stored(k, ng))
        for it in internal:
            if done >= nsteps:
                break
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise="philox", seed=7, step_index=it.step_index)
            done += 1
    g = T.get_particles()
    T.close()
    o = m.state()
    o["gid"] = o["gid"].astype(np.float64)
    o["isin"] = o["isin"].astype(np.int32)
    diff = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not diff, f"state after {nsteps} steps differs: {diff}"
    return gi, gj, g0


def test_spherical_single_grid():
    case = harness.make_case("cfg1", 10, seed=1)
    gi, gj, g0 = _run(case, 2000, 24, spherical=1)
    assert np.all(gi[0, :5] == -1.0)                       # off the grid: not found
    assert (g0["isin"] == 1).sum() > 1500


def test_cartesian_single_grid():
    case = harness.make_case("tiny", 10, seed=1)
    sp = case.spec
    X, Y = np.meshgrid(np.arange(sp.xi_rho) * 1000.0, np.arange(sp.eta_rho) * 1000.0, indexing="ij")
    case.grids[0]["lon_rho"], case.grids[0]["lat_rho"] = np.asfortranarray(X), np.asfortranarray(Y)
    _, _, g0 = _run(case, 1000, 24, spherical=0)
    assert (g0["isin"] == 1).sum() > 600


def test_spherical_nested_grids():
    case = harness.make_case("nest_tiny", 10, seed=1)
    _, _, g0 = _run(case, 2000, 24, spherical=1)
    assert len(np.unique(g0["gid"][g0["isin"] == 1])) == case.ngrid
