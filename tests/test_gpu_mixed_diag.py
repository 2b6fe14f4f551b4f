"""The diagnostics in the mixed-precision form (FP32 fields for salt, temp
and the bottom stress, FP32 interpolation; ROMSPath.f90:935-986) against
the exact form on the same FP32-stored frames: identical initial values
(both run the same initial lookup), and after a deterministic run values
within the mixed form's position error; output records take the current
positions."""
import numpy as np
import pytest

import harness
from romspath_b200 import Tracker, schedule

pytestmark = pytest.mark.gpu

SOV = {"diag": True, "field_dtype": "f32"}
POV = dict(harness.DIAG_PARAMS, vturb_on=0, hturb_on=0)


def _pair(nsteps, npart=400, name="tiny", resort=0):
    case = harness.make_case(name, npart, seed=3, spec_over=SOV, param_over=POV)
    out = {}
    for form in ("f32", "mixed"):
        g, T = harness.run_gpu(case, nsteps, field_dtype=form, resort=resort)
        out[form] = (g, T)
    return case, out


def test_initial_values_identical():
    case, out = _pair(0)
    a, b = out["f32"][0], out["mixed"][0]
    for k in ("p_salt", "p_temp", "mean_salt", "mean_temp", "p_hob", "p_bustr", "p_bvstr"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for _, T in out.values():
        T.close()


@pytest.mark.parametrize("resort", [0, 6])
def test_values_track_the_exact_form(resort):
    case, out = _pair(48, resort=resort)
    a, b = out["f32"][0], out["mixed"][0]
    for _, T in out.values():
        T.close()
    ok = (a["status"] == 1.0) & (b["status"] == 1.0)
    assert ok.sum() > 200
    dpos = np.hypot(a["x"] - b["x"], a["y"] - b["y"])[ok]
    assert np.median(dpos) < 1e-3
    # salt ~0.07 psu/m, temp ~0.25 C/m in depth: errors follow the depth error
    for k, med, p90 in (("p_salt", 2e-3, 2e-2), ("p_temp", 1e-2, 1e-1), ("p_hob", 2e-2, 2e-1)):
        d = np.abs(a[k] - b[k])[ok]
        assert np.median(d) < med and np.percentile(d, 90) < p90, (k, np.median(d), np.percentile(d, 90))
    for k in ("mean_salt", "mean_temp"):
        r = (np.abs(a[k] - b[k]) / np.abs(a[k]))[ok]
        assert np.median(r) < 1e-4, (k, np.median(r))
    # the bottom stress: same order as the exact form's, mostly within 2 %
    scale = np.abs(a["p_bustr"][ok]).max()
    d = np.abs(a["p_bustr"] - b["p_bustr"])[ok] / scale
    assert np.median(d) < 2e-2


def test_output_record_uses_current_positions():
    case = harness.make_case("tiny", 300, seed=4, spec_over=SOV, param_over=POV)
    T = Tracker(case.specs, case.grids, case.params, numpar=300, field_dtype="mixed", seed=7, resort=6)
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, case.frame(k))
    T.locate(case.release, t_b=1)
    done = 0
    for ext, internal in harness._steps(case, 24):
        for (k, slot) in ext.loads:
            T.upload_frame(1, slot, case.frame(k))
        for it in internal:
            if done >= 24:
                break
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            done += 1
    rec = T.output_record(25)
    st = T.get_particles()
    T.close()
    np.testing.assert_array_equal(rec["zp"], st["z"])
    g = case.grid
    ip, jp = st["x"], st["y"]
    I, J = np.floor(ip).astype(int), np.floor(jp).astype(int)
    X, Y = ip - I, jp - J
    a = g["lon_rho"]
    lon = ((1 - X) * (1 - Y) * a[I - 1, J - 1] + X * (1 - Y) * a[I, J - 1] + X * Y * a[I, J]
           + (1 - X) * Y * a[I - 1, J])
    np.testing.assert_allclose(rec["lon"], lon, rtol=0, atol=1e-12)
    assert np.all(rec["salt"][st["status"] == 1.0] > 30.0)
