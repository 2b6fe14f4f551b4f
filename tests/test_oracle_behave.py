"""The oracle's behave (behavior_module.f90:186-393) and its own exp/log:
accuracy of the series, the Laplace deviates, the constant swim of
Behavior 1 and the Fuchs swim/sink outputs of Behavior 10."""
import math

import numpy as np
import pytest

import harness
from oracle import oracle as O
from romspath_b200 import synth


def _ulps(a, b):
    a, b = np.float64(a), np.float64(b)
    if a == b:
        return 0
    return abs(int(np.array(a).view(np.int64)) - int(np.array(b).view(np.int64)))


def test_exp_log_accuracy():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-700, 700, 3000), rng.uniform(-2, 2, 3000), [0.0, 1e-300, -1e-300]])
    worst = max(_ulps(O.lib().orc_exp(float(x)), math.exp(x)) for x in xs)
    assert worst <= 4, worst
    ys = np.concatenate([np.exp(rng.uniform(-700, 700, 3000)), rng.uniform(0.5, 2.0, 3000), [5e-324, 1e-310]])
    worst = max(_ulps(O.lib().orc_log(float(y)), math.log(y)) for y in ys if abs(math.log(y)) > 1e-3)
    assert worst <= 4, worst
    assert O.lib().orc_log(0.0) == -math.inf and math.isnan(O.lib().orc_log(-1.0))
    assert O.lib().orc_exp(800.0) == math.inf and O.lib().orc_exp(-800.0) == 0.0


def test_philox_uniforms_in_open_interval_and_distinct_from_normals():
    u = np.array([O.lib().orc_philox_uniform(7, p, 3, k) for p in range(2000) for k in range(5)])
    assert np.all((u > 0) & (u < 1))
    assert abs(u.mean() - 0.5) < 0.01 and abs(u.var() - 1 / 12) < 0.003


def _run(pov, sov=None, nsteps=24, noise="philox"):
    p = dict(pov)
    case = harness.make_case("tiny", 200, seed=3, spec_over=dict(sov or {}, behave=True), param_over=p)
    hook = harness.noise_array(case, nsteps) if noise == "hook" else None
    return harness.run_oracle(case, nsteps, noise=noise, hook=hook)[0], case


def test_behavior1_adds_constant_swim():
    off = {"vturb_on": 0, "hturb_on": 0}
    o0, _ = _run(off)
    o1, case = _run({**off, "behavior": 1, "swimfast": 0.0005})
    act = (o0["status"] == 1.0) & (o1["status"] == 1.0)
    # a uniform upward drift of swimfast*idt per step, up to the reflections
    dz = (o1["z"] - o0["z"])[act]
    assert np.median(dz) > 0.5 * 24 * 0.0005 * 300
    assert np.all(o1["p_acc"] == 0.0)


@pytest.mark.parametrize("va_flag", [0, 1, 2])
def test_behavior10_outputs(va_flag):
    pov = {**synth.FUCHS_SAMPLE, "behavior": 10, "va_flag": va_flag, "b0wv": 0.3, "b1w": 0.1}
    o, case = _run(pov)
    act = o["age"] > 0
    assert np.all(np.isin(o["p_ssf"][act], [0.0, 1.0]))
    assert 0 < o["p_ssf"][act].mean() < 1
    # sinking speed: Stokes-like fall of a 250 um larva (cm/s, negative)
    r = 250.0 / 2.0e4
    wsink = (3 * 0.01026 - math.sqrt(4 / 3 * 980 * r**3 * 1.026 * (1.06 - 1.026) + 9 * 0.01026**2)) / (r * 1.026)
    sink = o["p_ssf"] == 1.0
    np.testing.assert_allclose(o["p_behavew"][sink & act], wsink, rtol=1e-12)
    assert np.all(o["p_vort"][act] >= 0.0) and np.all(o["p_acc"][act] >= 0.0)


def test_hook_and_mt_streams_run():
    pov = {**synth.FUCHS_SAMPLE, "behavior": 10, "va_flag": 0}
    o, _ = _run(pov, noise="hook", nsteps=12)
    assert np.isfinite(o["z"]).all()
