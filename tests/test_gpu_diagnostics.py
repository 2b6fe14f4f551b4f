"""GPU parity of the diagnostics (SaltTempOn, SaltTempMean, WriteBottom;
ROMSPath.f90:935-986 with the initial values of ini_ROMSPath): salinity,
temperature, their running sums, height above bottom and bottom stress
against the oracle, bit for bit, together with every particle column."""
import numpy as np
import pytest

import harness
from romspath_b200 import Tracker, _lib
from romspath_b200.tracker import RomsPathError

pytestmark = pytest.mark.gpu

DIAG_FIELDS = tuple(harness.DIAG_GPU_TO_ORACLE.values())


def _assert_same(g, o, what, fields=harness.FIELDS + DIAG_FIELDS):
    diff = harness.compare(g, o, fields)
    bad = {k: v for k, v in diff.items() if v}
    assert not bad, f"{what}: fields differing (particle counts): {bad}"


CASES = [
    # name, npart, nsteps, noise, spec overrides, param overrides, resort
    ("tiny-det", "tiny", 200, 120, "off", {}, {"vturb_on": 0, "hturb_on": 0}, 0),
    ("tiny-philox", "tiny", 200, 60, "philox", {}, {}, 0),
    ("tiny-f32", "tiny", 200, 36, "philox", {"field_dtype": "f32", "stokes": True}, {}, 0),
    ("tiny-resort", "tiny", 200, 60, "philox", {}, {}, 6),
    ("tiny-nsb2", "tiny", 100, 24, "philox", {}, {"nsb": 2}, 0),
    ("tiny-oob", "tiny", 200, 60, "philox", {}, {"open_ocean_boundary": 1}, 0),
    ("cfg1", "cfg1", 300, 24, "philox", {}, {}, 0),
    ("nest-philox", "nest_tiny", 400, 48, "philox", {}, {}, 0),
    ("nest-resort", "nest_tiny", 400, 48, "philox", {}, {}, 6),
]


@pytest.mark.parametrize("variant", ["fused", "split"])
@pytest.mark.parametrize("cid,name,npart,nsteps,noise,sov,pov,resort", CASES, ids=[c[0] for c in CASES])
def test_diagnostics_bit_exact(cid, name, npart, nsteps, noise, sov, pov, resort, variant):
    p = dict(harness.DIAG_PARAMS)
    p.update(pov)
    case = harness.make_case(name, npart, seed=3, spec_over=dict(sov, diag=True), param_over=p)
    g, T = harness.run_gpu(case, nsteps, noise=noise, variant=variant, resort=resort)
    T.close()
    o, _ = harness.run_oracle(case, nsteps, noise=noise)
    _assert_same(g, o, cid)
    assert np.count_nonzero(g["p_bustr"]) > npart // 4
    assert np.mean(g["p_hob"][g["isin"] == 1] < 9999.0) > 0.9


@pytest.mark.parametrize("which", [("salttemp_on",), ("salttemp_on", "salttemp_mean"), ("write_bottom",)])
def test_each_switch_alone(which):
    p = {k: 1 for k in which}
    case = harness.make_case("tiny", 150, seed=4, spec_over={"diag": True}, param_over=p)
    g, T = harness.run_gpu(case, 36)
    d = T.get_diagnostics()
    T.close()
    o, _ = harness.run_oracle(case, 36)
    fields = [harness.DIAG_GPU_TO_ORACLE[k] for k in d]
    _assert_same(g, o, str(which), harness.FIELDS + tuple(fields))


def test_output_reset_between_records():
    """The writer's resets after a record (sums to 0, HOB to 9999) on the
    device, then more steps, against the oracle with the same resets."""
    from romspath_b200 import schedule
    from oracle import oracle as O
    case = harness.make_case("tiny", 200, seed=5, spec_over={"diag": True}, param_over=harness.DIAG_PARAMS)
    T = Tracker(case.specs, case.grids, case.params, numpar=200, seed=7, resort=6)
    m = O.OracleModel(case.specs, case.grids, case.params)
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, case.frame(k))
        m.set_frame(1, slot, case.stored(k))
    T.locate(case.release, t_b=1)
    m.init_particles(case.release, tb=1)
    done = 0
    for ext, internal in harness._steps(case, 72):
        for (k, slot) in ext.loads:
            T.upload_frame(1, slot, case.frame(k))
            m.set_frame(1, slot, case.stored(k))
        for it in internal:
            if done >= 72:
                break
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise="philox", seed=7, step_index=it.step_index)
            done += 1
            if done % 24 == 0:
                T.reset_diagnostics()
                m.st["mean_salt"][:] = 0.0
                m.st["mean_temp"][:] = 0.0
                m.st["p_hob"][:] = 9999.0
    g = T.get_particles()
    g.update({harness.DIAG_GPU_TO_ORACLE[k]: v for k, v in T.get_diagnostics().items()})
    T.close()
    o = m.state()
    o["gid"] = o["gid"].astype(np.float64)
    o["isin"] = o["isin"].astype(np.int32)
    _assert_same(g, o, "reset")
    # the last record was reset at step 72: sums and minimum start again
    assert np.all(g["mean_salt"] == 0.0) and np.all(g["p_hob"] == 9999.0)


def test_refusals():
    case = harness.make_case("tiny", 50, seed=3, spec_over={"diag": True}, param_over=harness.DIAG_PARAMS)
    T = Tracker(case.specs, case.grids, case.params, numpar=50)
    # an upload without the diagnostics' fields is refused
    f = {k: v for k, v in case.frame(1).items() if k not in ("salt", "temp", "bustr", "bvstr")}
    import ctypes as C
    arrs = [np.asfortranarray(f[k]) for k in ("zeta", "u", "v", "w", "aks")]
    rc = T.L.rp_upload_frame(T.h, 1, 1, *[a.ctypes.data_as(_lib.PD) for a in arrs], None, None)
    assert rc == -1
    # the no-allocation step refuses while diagnostics are on
    from romspath_b200 import schedule
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, case.frame(k))
    T.locate(case.release, t_b=1)
    st = T.device_state()
    ex = (C.c_double * 3)(0.0, 3600.0, 7200.0)
    ix = (C.c_double * 3)(0.0, 300.0, 600.0)
    assert T.L.rp_step_noalloc(T.h, C.byref(st), ex, ix, 2, 1, 2, 3) == -5
    T.close()
    # a diagnostic that is off cannot be read
    case2 = harness.make_case("tiny", 50, seed=3, spec_over={"diag": True}, param_over={"write_bottom": 1})
    T2 = Tracker(case2.specs, case2.grids, case2.params, numpar=50)
    for (k, slot) in schedule.initial_loads():
        T2.upload_frame(1, slot, case2.frame(k))
    T2.locate(case2.release, t_b=1)
    out = np.empty(50)
    assert T2.L.rp_get_diagnostics(T2.h, 50, out.ctypes.data_as(_lib.PD), None, None, None, None, None, None) == -3
    T2.close()
