"""The oracle's init lookup: own sin/cos/asin, LL2ij (interpolation_module.f90:
110-268) on Cartesian and spherical grids, and InitGrid's nest maps
(grid_module.f90:441-481)."""
import math

import numpy as np
import pytest

import harness
from oracle import oracle as O
from romspath_b200 import synth


def _ulps(a, b):
    if a == b:
        return 0
    return abs(int(np.array(a).view(np.int64)) - int(np.array(b).view(np.int64)))


def test_sincos_asin_accuracy():
    rng = np.random.default_rng(1)
    for x in np.concatenate([rng.uniform(-4, 4, 4000), [0.0, 1e-300, math.pi / 2, -math.pi]]):
        s, c = O.sincos(x)
        assert abs(s - math.sin(x)) <= 4e-16 * max(1.0, abs(math.sin(x))) + 1e-300
        assert abs(c - math.cos(x)) <= 4e-16
    for x in np.concatenate([rng.uniform(-1, 1, 4000), [0.0, 0.5, -0.5, 1.0, -1.0, 1e-300]]):
        a = O.lib().orc_asin(float(x))
        assert _ulps(a, math.asin(x)) <= 4, (x, a, math.asin(x))
    assert math.isnan(O.lib().orc_asin(1.5))


def _bilinear(a, ip, jp):
    I, J = np.floor(ip).astype(int), np.floor(jp).astype(int)
    X, Y = ip - I, jp - J
    return ((1 - X) * (1 - Y) * a[I - 1, J - 1] + X * (1 - Y) * a[I, J - 1] + X * Y * a[I, J]
            + (1 - X) * Y * a[I - 1, J])


def _model(case):
    return O.OracleModel(case.specs, case.grids, case.params)


def test_ll2ij_cartesian_inverts_a_regular_grid():
    case = harness.make_case("tiny", 10, seed=1)
    sp = case.spec
    g = dict(case.grid)
    X, Y = np.meshgrid(np.arange(sp.xi_rho) * 1000.0, np.arange(sp.eta_rho) * 1000.0, indexing="ij")
    g["lon_rho"], g["lat_rho"] = np.asfortranarray(X), np.asfortranarray(Y)
    m = O.OracleModel(case.specs, [g], case.params)
    rng = np.random.default_rng(2)
    ip = rng.uniform(1.0, sp.xi_rho, 500)
    jp = rng.uniform(1.0, sp.eta_rho, 500)
    gi, gj = m.ll2ij(1, (ip - 1) * 1000.0, (jp - 1) * 1000.0, spherical=0)
    np.testing.assert_allclose(gi, ip, atol=1e-9)
    np.testing.assert_allclose(gj, jp, atol=1e-9)


def test_ll2ij_spherical_on_rotated_grid():
    case = harness.make_case("cfg1", 10, seed=1)
    sp, g = case.spec, case.grid
    m = _model(case)
    rng = np.random.default_rng(3)
    ip = rng.uniform(2.0, sp.xi_rho - 1.0, 400)
    jp = rng.uniform(2.0, sp.eta_rho - 1.0, 400)
    lon, lat = _bilinear(g["lon_rho"], ip, jp), _bilinear(g["lat_rho"], ip, jp)
    gi, gj = m.ll2ij(1, lon, lat, spherical=1)
    assert np.max(np.abs(gi - ip)) < 5e-3 and np.max(np.abs(gj - jp)) < 5e-3
    # a point off the grid is not found
    gi, gj = m.ll2ij(1, [-60.0], [30.0], spherical=1)
    assert gi[0] == -1.0 and gj[0] == -1.0


def _exact_nest():
    """A parent 20x16 at 1 km and a child 25x21 at 250 m whose rho point
    (1,1) sits on parent point (6,5): lon/lat values coincide exactly."""
    px, py = np.meshgrid(np.arange(20) * 1000.0, np.arange(16) * 1000.0, indexing="ij")
    cx, cy = np.meshgrid(5000.0 + np.arange(25) * 250.0, 4000.0 + np.arange(21) * 250.0, indexing="ij")
    return (px, py), (cx, cy)


def test_nest_maps_search():
    (px, py), (cx, cy) = _exact_nest()
    specs = [synth.GridSpec(25, 21, 4), synth.GridSpec(20, 16, 4)]      # finest first
    grids = [synth.make_grid(s) for s in specs]
    grids[0]["lon_rho"], grids[0]["lat_rho"] = np.asfortranarray(cx), np.asfortranarray(cy)
    grids[1]["lon_rho"], grids[1]["lat_rho"] = np.asfortranarray(px), np.asfortranarray(py)
    params = synth.config_params("tiny")
    m = O.OracleModel(specs, grids, params)
    scl, off = m.nest_maps([4.0])
    # grid 1 (child) -> grid 2 (parent): X2 = X1/4 + off; child (1,1) = parent (6,5)
    np.testing.assert_array_equal(scl[0][1], [0.25, 0.25])
    np.testing.assert_array_equal(off[0][1], [6.0 - 0.25, 5.0 - 0.25])
    np.testing.assert_array_equal(scl[1][0], [4.0, 4.0])
    np.testing.assert_array_equal(off[1][0], [1.0 - 4.0 * 6.0, 1.0 - 4.0 * 5.0])
    np.testing.assert_array_equal(scl[0][0], [1.0, 1.0])
    np.testing.assert_array_equal(off[1][1], [0.0, 0.0])


def _three_grids():
    """Three nested grids (finest first) with exactly coincident points, one
    pair with several coincident candidates, and NaN / -0.0 entries."""
    x0, y0 = np.meshgrid(np.arange(30) * 1000.0, np.arange(24) * 1000.0, indexing="ij")
    x1, y1 = np.meshgrid(6000.0 + np.arange(31) * 500.0, 5000.0 + np.arange(25) * 500.0, indexing="ij")
    x2, y2 = np.meshgrid(8000.0 + np.arange(33) * 125.0, 7000.0 + np.arange(29) * 125.0, indexing="ij")
    x0 = x0.copy()
    x0[0, 0] = np.nan
    y1 = y1.copy()
    x2 = x2 - 8000.0 + 8000.0
    return [(x2, y2), (x1, y1), (x0, y0)]


@pytest.mark.parametrize("case", ["nested", "disjoint"])
def test_host_nest_maps_match_oracle_search(case):
    from romspath_b200.tracker import nest_maps
    gl = _three_grids()
    if case == "disjoint":
        gl[0] = (gl[0][0] + 0.1, gl[0][1])          # no coincident point with the finest grid
    specs = [synth.GridSpec(a.shape[0], a.shape[1], 4) for a, _ in gl]
    grids = [synth.make_grid(s) for s in specs]
    for g, (lo, la) in zip(grids, gl):
        g["lon_rho"], g["lat_rho"] = np.asfortranarray(lo), np.asfortranarray(la)
    m = O.OracleModel(specs, grids, synth.config_params("tiny"))
    refine = [4.0, 2.0]
    so, oo = m.nest_maps(refine)
    sh, oh = nest_maps(grids, refine)
    np.testing.assert_array_equal(sh, so)
    np.testing.assert_array_equal(oh, oo)
    if case == "nested":
        # grid 2 (middle) -> grid 3 (coarsest), (1,1) on (7,6): the scale is
        # 1/grefine(2,3) = 1/refine(|2-3|) = 1/4, the reference indexing
        # refine by the grids' distance (grid_module.f90:443-449)
        np.testing.assert_array_equal(so[1][2], [0.25, 0.25])
        np.testing.assert_array_equal(oo[1][2], [7.0 - 0.25, 6.0 - 0.25])
        # grid 1 -> grid 3: refine(2)^2 = 4
        np.testing.assert_array_equal(so[0][2], [0.25, 0.25])


def test_synth_pair_maps_equal_reference_chain_maps():
    """On a chain of nested grids (refinement 4 per level, finest first)
    the affine maps the synthetic workloads use for every grid pair
    (synth.nest_maps, which config 4's siblings also use) equal the
    reference's own: grefine(a,b) = refine(|a-b|)^|a-b| and the offsets from
    the first coincident lon/lat point (grid_module.f90:441-481), found both
    by the oracle's search and by rp_nest_maps."""
    from romspath_b200.tracker import nest_maps
    specs = [synth.GridSpec(33, 29, 4, dx=64.0, dy=64.0, x0=6144.0, y0=4864.0),
             synth.GridSpec(31, 25, 4, dx=256.0, dy=256.0, x0=5120.0, y0=4096.0),
             synth.GridSpec(30, 24, 4, dx=1024.0, dy=1024.0)]
    grids = [synth.make_grid(s) for s in specs]
    for sp, g in zip(specs, grids):
        lo, la = np.meshgrid(sp.x0 + np.arange(sp.xi_rho) * sp.dx, sp.y0 + np.arange(sp.eta_rho) * sp.dy,
                             indexing="ij")
        g["lon_rho"], g["lat_rho"] = np.asfortranarray(lo), np.asfortranarray(la)
    refine = [4.0, 4.0]
    s_syn, o_syn = synth.nest_maps(specs)
    s_lib, o_lib = nest_maps(grids, refine)
    m = O.OracleModel(specs, grids, synth.config_params("tiny"))
    s_orc, o_orc = m.nest_maps(refine)
    np.testing.assert_array_equal(s_lib, s_orc)
    np.testing.assert_array_equal(o_lib, o_orc)
    np.testing.assert_array_equal(np.asarray(s_lib), s_syn)
    np.testing.assert_array_equal(np.asarray(o_lib), o_syn)
    # fine -> parent skips a level: 1/refine(2)^2
    np.testing.assert_array_equal(s_syn[0][2], [1.0 / 16.0, 1.0 / 16.0])
