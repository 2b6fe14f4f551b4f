"""The oracle's diagnostics (ROMSPath.f90:935-986 and their initial values,
247-264, 353-355, 408-427): bottom stress interpolation against a direct
restatement, and the running minimum / running sums against the per-step
values the oracle itself reports."""
import numpy as np
import pytest

import harness
from oracle import oracle as O

DIAG = {"salttemp_on": 1, "salttemp_mean": 1, "write_bottom": 1}


def _case(npart=120, **pov):
    p = dict(DIAG)
    p.update(pov)
    return harness.make_case("tiny", npart, seed=3, spec_over={"diag": True}, param_over=p)


def _model(case):
    m = O.OracleModel(case.specs, case.grids, case.params, scl=case.scl, off=case.off)
    for slot, k in ((1, 1), (2, 2), (3, 3)):
        m.set_frame(1, slot, case.stored(k))
    return m


def _str_direct(case, var, ip, jp, slot_frame):
    """getInterpStr restated for interior points: bilinear on the u (bustr)
    or v (bvstr) points, dry corners zeroed, all-dry cell zero."""
    g = case.grid
    f = slot_frame["bustr" if var == "u" else "bvstr"]
    m = g["mask_u" if var == "u" else "mask_v"]
    if var == "u":
        I = int(np.floor(ip - 0.5)); J = int(np.floor(jp))
        X = (ip - 0.5) - I; Y = jp - J
    else:
        I = int(np.floor(ip)); J = int(np.floor(jp - 0.5))
        X = ip - I; Y = (jp - 0.5) - J
    cff = [(1 - X) * (1 - Y), X * (1 - Y), X * Y, (1 - X) * Y]
    idx = [(I, J), (I + 1, J), (I + 1, J + 1), (I, J + 1)]
    v = [f[i - 1, j - 1] for i, j in idx]
    mk = [m[i - 1, j - 1] for i, j in idx]
    nw = sum(mk)
    if 0 < nw < 4:
        v = [vv if mm else 0.0 for vv, mm in zip(v, mk)]
    elif nw == 0:
        cff = [0.0] * 4
        v = [0.0] * 4
    return cff[0] * v[0] + cff[1] * v[1] + cff[2] * v[2] + cff[3] * v[3]


@pytest.mark.parametrize("var", ["u", "v"])
def test_bottom_stress_interpolation(var):
    case = _case()
    m = _model(case)
    rng = np.random.default_rng(1)
    sp = case.spec
    fr = case.stored(2)
    code = 0 if var == "u" else 1     # ORC_V_BUSTR, ORC_V_BVSTR
    import ctypes as C
    for _ in range(400):
        ip = rng.uniform(2.0, sp.xi_rho - 2.0)
        jp = rng.uniform(2.0, sp.eta_rho - 2.0)
        fl = C.c_uint32(0)
        got = O.lib().orc_getinterp_str(C.byref(m.g[0]), code, ip, jp, 2, C.byref(fl))
        want = _str_direct(case, var, ip, jp, fr)
        assert got == want or abs(got - want) <= 1e-15 * max(1e-12, abs(want)), (ip, jp, got, want)


def test_running_minimum_and_sums():
    """P_HOB is the running minimum of bath + z (the step's btemp), starting
    at 9999; mean_salt/mean_temp are the initial value plus each step's
    P_Salt/P_Temp, summed in order; bustr changes only on a new minimum."""
    case = _case(npart=150, vturb_on=1, hturb_on=1)
    m = O.OracleModel(case.specs, case.grids, case.params, scl=case.scl, off=case.off)
    from romspath_b200 import schedule
    for (k, slot) in schedule.initial_loads():
        m.set_frame(1, slot, case.stored(k))
    m.init_particles(case.release, tb=1)
    s0 = m.state()
    assert np.all(s0["p_hob"] == 9999.0)
    isin0 = s0["isin"].astype(bool)
    assert isin0.sum() > 100
    np.testing.assert_array_equal(s0["mean_salt"], s0["p_salt"])
    assert np.all(s0["p_salt"][isin0] > 30.0)
    hob = np.full(150, 9999.0)
    ms, mt = s0["mean_salt"].copy(), s0["mean_temp"].copy()
    prev_bu = s0["p_bustr"].copy()
    prev_age = s0["age"].copy()
    done = 0
    for ext, internal in harness._steps(case, 36):
        for (k, slot) in ext.loads:
            m.set_frame(1, slot, case.stored(k))
        for it in internal:
            if done >= 36:
                break
            m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise="philox", seed=7, step_index=it.step_index)
            st = m.state()
            act = st["age"] != prev_age      # particles the step updated
            prev_age = st["age"].copy()
            bt = st["bath"] + st["z"]
            new = act & (bt <= hob)
            hob = np.where(act, np.minimum(bt, hob), hob)
            ms = np.where(act, ms + st["p_salt"], ms)
            mt = np.where(act, mt + st["p_temp"], mt)
            np.testing.assert_array_equal(st["p_hob"], hob)
            np.testing.assert_array_equal(st["mean_salt"], ms)
            np.testing.assert_array_equal(st["mean_temp"], mt)
            assert np.all(st["p_bustr"][~new] == prev_bu[~new])
            prev_bu = st["p_bustr"].copy()
            done += 1
    assert np.count_nonzero(prev_bu) > 50


def test_off_leaves_diagnostics_alone():
    case = harness.make_case("tiny", 80, seed=3)
    o, _ = harness.run_oracle(case, 12)
    assert np.all(o["p_salt"] == 0.0) and np.all(o["p_hob"] == 9999.0) and np.all(o["mean_salt"] == 0.0)


def test_output_record_lonlat_and_means():
    """dataOutput's lon/lat are plain bilinear interpolants of lon_rho and
    lat_rho; the record's salt/temp are the sums over mI; the writer then
    resets the sums and P_HOB."""
    case = _case(npart=100)
    m = O.OracleModel(case.specs, case.grids, case.params, scl=case.scl, off=case.off)
    from romspath_b200 import schedule
    for (k, slot) in schedule.initial_loads():
        m.set_frame(1, slot, case.stored(k))
    m.init_particles(case.release, tb=1)
    for it in list(harness._steps(case, 5))[0][1][:5]:
        m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise="philox", seed=7, step_index=it.step_index)
    st = m.state()
    rec = m.output_record(6)
    g = case.grid
    for n in range(100):
        ip, jp = st["x"][n], st["y"][n]
        I, J = int(np.floor(ip)), int(np.floor(jp))
        X, Y = ip - I, jp - J
        c = [(1 - X) * (1 - Y), X * (1 - Y), X * Y, (1 - X) * Y]
        for name, key in (("lon_rho", "lon"), ("lat_rho", "lat")):
            a = g[name]
            v = [a[I - 1, J - 1], a[I, J - 1], a[I, J], a[I - 1, J]]
            want = c[0] * v[0] + c[1] * v[1] + c[2] * v[2] + c[3] * v[3]
            assert rec[key][n] == want
    np.testing.assert_array_equal(rec["salt"], st["mean_salt"] / 6.0)
    np.testing.assert_array_equal(rec["hob"], st["p_hob"])
    after = m.state()
    assert np.all(after["mean_salt"] == 0.0) and np.all(after["p_hob"] == 9999.0)
