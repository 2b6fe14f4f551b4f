"""behave (behavior_module.f90:186-393) in the mixed-precision form against
the exact form on the same FP32-stored frames and the same draws: the
constant swim of Behavior 1 and the Fuchs response of Behavior 10 (its
fields interpolated in FP32, the response in FP64 shared with the exact
form) follow the exact form within the mixed form's own error."""
import numpy as np
import pytest

import harness
from romspath_b200 import synth

pytestmark = pytest.mark.gpu

F10 = dict(synth.FUCHS_SAMPLE, behavior=10, va_flag=0, b0wv=0.3, b1w=0.1)


def _pair(pov, nsteps=36, noise="philox", npart=400):
    case = harness.make_case("tiny", npart, seed=3, spec_over={"behave": True, "field_dtype": "f32"},
                             param_over=dict(pov, vturb_on=0, hturb_on=0))
    hook = harness.noise_array(case, nsteps) if noise == "hook" else None
    out = {}
    for form in ("f32", "mixed"):
        g, T = harness.run_gpu(case, nsteps, noise=noise, hook=hook, field_dtype=form)
        T.close()
        out[form] = g
    return out["f32"], out["mixed"]


def test_behavior1_swim():
    a, b = _pair({"behavior": 1, "swimfast": 0.0005})
    ok = (a["status"] == 1.0) & (b["status"] == 1.0)
    assert ok.sum() > 200
    dz = np.abs(a["z"] - b["z"])[ok]
    assert np.median(dz) < 1e-3, np.median(dz)


@pytest.mark.parametrize("noise", ["philox", "hook"])
def test_behavior10_response(noise):
    a, b = _pair(F10, noise=noise)
    act = a["age"] > 0
    assert act.sum() > 200
    same = a["p_ssf"][act] == b["p_ssf"][act]
    assert same.mean() > 0.97, same.mean()
    for k in ("p_acc", "p_vort"):
        r = (np.abs(a[k] - b[k]) / np.maximum(np.abs(a[k]), 1e-12))[act]
        assert np.median(r) < 2e-3, (k, np.median(r))
    r = (np.abs(a["p_behavew"] - b["p_behavew"]) / np.abs(a["p_behavew"]))[act][same]
    assert np.median(r) < 2e-3
    assert 0 < b["p_ssf"][act].mean() < 1
    ok = (a["status"] == 1.0) & (b["status"] == 1.0)
    assert np.median(np.abs(a["z"] - b["z"])[ok]) < 5e-3
