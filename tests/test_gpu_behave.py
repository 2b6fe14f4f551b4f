"""GPU parity of behave (behavior_module.f90:186-393): Behavior 1 (constant
swim), 10 (Fuchs swim/sink response to turbulent and wave acceleration and
vorticity) and 11 (outputs only), with Process_VA / Process_WA, on Philox
and hook noise, against the oracle bit for bit: every particle column and
par(:,pAcc/pVort/pbehaveW/pSSF)."""
import numpy as np
import pytest

import harness
from romspath_b200 import Tracker, synth
from romspath_b200.tracker import RomsPathError

pytestmark = pytest.mark.gpu

BEH = tuple(harness.BEHAVE_GPU_TO_ORACLE.values())
F10 = dict(synth.FUCHS_SAMPLE, behavior=10, b0wv=0.3, b1w=0.1)


def _assert_same(g, o, what, fields):
    diff = harness.compare(g, o, fields)
    bad = {k: v for k, v in diff.items() if v}
    assert not bad, f"{what}: fields differing (particle counts): {bad}"


CASES = [
    # id, grid, npart, nsteps, noise, spec overrides, param overrides, resort
    ("b1-philox", "tiny", 200, 48, "philox", {}, {"behavior": 1, "swimfast": 0.0005}, 0),
    ("b10-va0", "tiny", 300, 48, "philox", {}, dict(F10, va_flag=0), 0),
    ("b10-va1", "tiny", 300, 48, "philox", {}, dict(F10, va_flag=1), 0),
    ("b10-va2", "tiny", 300, 48, "philox", {}, dict(F10, va_flag=2), 6),
    ("b10-hook", "tiny", 200, 24, "hook", {}, dict(F10, va_flag=0), 0),
    ("b10-va-only", "tiny", 200, 36, "philox", {}, dict(F10, va_flag=0, process_wa=0), 0),
    ("b10-wa-only", "tiny", 200, 36, "philox", {}, dict(F10, va_flag=2, process_va=0), 0),
    ("b11", "tiny", 200, 36, "philox", {}, dict(F10, behavior=11), 0),
    ("b10-f32", "tiny", 200, 36, "philox", {"field_dtype": "f32", "stokes": True}, dict(F10, va_flag=0), 0),
    ("b10-wetdry-diag", "tiny", 300, 48, "philox", {"wetdry": True, "diag": True},
     dict(F10, va_flag=0, wetdry=1, **harness.DIAG_PARAMS), 6),
    ("b10-nest", "nest_tiny", 400, 36, "philox", {}, dict(F10, va_flag=0), 6),
]


@pytest.mark.parametrize("variant", ["fused", "split"])
@pytest.mark.parametrize("cid,name,npart,nsteps,noise,sov,pov,resort", CASES, ids=[c[0] for c in CASES])
def test_behave_bit_exact(cid, name, npart, nsteps, noise, sov, pov, resort, variant):
    case = harness.make_case(name, npart, seed=3, spec_over=dict(sov, behave=True), param_over=pov)
    hook = harness.noise_array(case, nsteps) if noise == "hook" else None
    g, T = harness.run_gpu(case, nsteps, noise=noise, hook=hook, variant=variant, resort=resort)
    T.close()
    o, _ = harness.run_oracle(case, nsteps, noise=noise, hook=hook)
    fields = harness.FIELDS
    if pov.get("process_va") or pov.get("process_wa"):
        fields = fields + BEH
    if sov.get("diag"):
        fields = fields + tuple(harness.DIAG_GPU_TO_ORACLE.values())
    _assert_same(g, o, cid, fields)
    if pov.get("behavior") == 10:
        act = g["age"] > 0
        assert 0 < g["p_ssf"][act].mean() < 1


def test_behave_refusals():
    case = harness.make_case("tiny", 50, seed=3, spec_over={"behave": True}, param_over=F10)
    T = Tracker(case.specs, case.grids, case.params, numpar=50)
    f = {k: v for k, v in case.frame(1).items() if k not in ("turbaccel", "turbvort")}
    with pytest.raises(RomsPathError, match="Process_VA"):
        T.upload_frame(1, 1, f)
    T.close()
