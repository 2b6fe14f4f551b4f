"""WETDRY (per-frame wet/dry masks) in the mixed-precision form against the
exact form on the same FP32-stored frames: u, v, w, the diagnostics and
behave's fields take each ring slot's own masks, so trajectories and
values follow the exact form within the mixed form's error, and differ
from the same mixed run without WETDRY."""
import numpy as np
import pytest

import harness
from romspath_b200 import synth

pytestmark = pytest.mark.gpu


def _run(form, pov, sov, nsteps=60, npart=400):
    case = harness.make_case("tiny", npart, seed=3, spec_over=dict(sov, field_dtype="f32"),
                             param_over=dict(pov, vturb_on=0, hturb_on=0))
    g, T = harness.run_gpu(case, nsteps, field_dtype=form)
    T.close()
    return g


def test_trajectories_track_the_exact_form():
    a = _run("f32", {"wetdry": 1}, {"wetdry": True})
    b = _run("mixed", {"wetdry": 1}, {"wetdry": True})
    c = _run("mixed", {}, {"wetdry": True})
    ok = (a["status"] == 1.0) & (b["status"] == 1.0)
    assert ok.sum() > 200
    d = np.hypot(a["x"] - b["x"], a["y"] - b["y"])[ok]
    assert np.median(d) < 1e-3 and np.percentile(d, 90) < 1e-2, (np.median(d), np.percentile(d, 90))
    assert np.mean(a["status"] == b["status"]) > 0.98
    # the masks matter: without WETDRY the mixed form moves many particles elsewhere
    e = np.hypot(c["x"] - b["x"], c["y"] - b["y"])
    assert np.mean(e > 1e-2) > 0.1


def test_diagnostics_and_behave_under_wetdry():
    pov = dict(harness.DIAG_PARAMS, wetdry=1, **dict(synth.FUCHS_SAMPLE, behavior=10, va_flag=0))
    sov = {"wetdry": True, "diag": True, "behave": True}
    a = _run("f32", pov, sov, nsteps=36)
    b = _run("mixed", pov, sov, nsteps=36)
    ok = (a["status"] == 1.0) & (b["status"] == 1.0)
    assert ok.sum() > 200
    for k, med in (("p_salt", 5e-3), ("p_temp", 3e-2)):
        dd = np.abs(a[k] - b[k])[ok]
        assert np.median(dd) < med, (k, np.median(dd))
    act = a["age"] > 0
    assert np.mean(a["p_ssf"][act] == b["p_ssf"][act]) > 0.95
    r = (np.abs(a["p_vort"] - b["p_vort"]) / np.maximum(np.abs(a["p_vort"]), 1e-12))[act]
    assert np.median(r) < 5e-3
