"""GPU parity under WETDRY (the -DWETDRY build: per-frame wet/dry masks in
getInterp3D and getInterpStr, hydrodynamic_module.f90:510-570,
interpolation_module.f90:628-939, 1022-1136): every particle column and the
diagnostics against the oracle, bit for bit."""
import ctypes as C

import numpy as np
import pytest

import harness
from romspath_b200 import Tracker, _lib, schedule
from romspath_b200.tracker import RomsPathError

pytestmark = pytest.mark.gpu

WD = {"wetdry": 1}


def _assert_same(g, o, what, fields=harness.FIELDS):
    diff = harness.compare(g, o, fields)
    bad = {k: v for k, v in diff.items() if v}
    assert not bad, f"{what}: fields differing (particle counts): {bad}"


CASES = [
    # name, npart, nsteps, spec overrides, param overrides, resort
    ("tiny-det", "tiny", 300, 120, {}, {"vturb_on": 0, "hturb_on": 0}, 0),
    ("tiny-philox", "tiny", 300, 60, {}, {}, 0),
    ("tiny-f32", "tiny", 200, 36, {"field_dtype": "f32", "stokes": True}, {}, 0),
    ("tiny-resort", "tiny", 300, 60, {}, {}, 6),
    ("tiny-diag", "tiny", 300, 60, {"diag": True}, harness.DIAG_PARAMS, 0),
    ("nest-philox", "nest_tiny", 400, 48, {}, {}, 6),
]


@pytest.mark.parametrize("variant", ["fused", "split"])
@pytest.mark.parametrize("cid,name,npart,nsteps,sov,pov,resort", CASES, ids=[c[0] for c in CASES])
def test_wetdry_bit_exact(cid, name, npart, nsteps, sov, pov, resort, variant):
    case = harness.make_case(name, npart, seed=3, spec_over=dict(sov, wetdry=True), param_over=dict(pov, **WD))
    g, T = harness.run_gpu(case, nsteps, variant=variant, resort=resort)
    T.close()
    o, _ = harness.run_oracle(case, nsteps)
    fields = harness.FIELDS + (tuple(harness.DIAG_GPU_TO_ORACLE.values()) if sov.get("diag") else ())
    _assert_same(g, o, cid, fields)
    # the masks changed the run: it differs from the same run without WETDRY
    if name == "tiny" and not sov:
        case0 = harness.make_case(name, npart, seed=3, param_over=pov)
        o0, _ = harness.run_oracle(case0, nsteps)
        assert int((o0["x"] != o["x"]).sum()) > npart // 10


def test_wetdry_refusals():
    case = harness.make_case("tiny", 50, seed=3, spec_over={"wetdry": True}, param_over=WD)
    T = Tracker(case.specs, case.grids, case.params, numpar=50)
    f = case.frame(1)
    arrs = [np.asfortranarray(f[k]) for k in ("zeta", "u", "v", "w", "aks")]
    # the plain upload has no masks
    assert T.L.rp_upload_frame(T.h, 1, 1, *[a.ctypes.data_as(_lib.PD) for a in arrs], None, None) == -1
    # masks other than 0/1
    bad = dict(f)
    bad["wetdry_rho"] = f["wetdry_rho"] * 0.5
    with pytest.raises(RomsPathError, match="0 or 1"):
        T.upload_frame(1, 1, bad)
    T.close()
