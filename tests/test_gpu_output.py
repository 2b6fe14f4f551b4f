"""GPU parity of the output step (dataOutput / writeNetCDF,
ROMSPath.f90:1012-1024, 1924-2070): every record -- lon, lat, zp, age,
status, GID and the diagnostics, with the writer's means and resets --
against the oracle, bit for bit, in the caller's particle order also when
the device state is re-sorted."""
import numpy as np
import pytest

import harness
from romspath_b200 import Tracker, schedule
from romspath_b200.tracker import RomsPathError

pytestmark = pytest.mark.gpu


def _run(case, nsteps, every, resort=0, variant="fused", n_out=None):
    from oracle import oracle as O
    npart = case.release.z.shape[0]
    T = Tracker(case.specs, case.grids, case.params, numpar=npart, seed=7, scl=case.scl, off=case.off,
                resort=resort, variant=variant)
    m = O.OracleModel(case.specs, case.grids, case.params, scl=case.scl, off=case.off)
    for (k, slot) in schedule.initial_loads():
        for ng in range(1, case.ngrid + 1):
            T.upload_frame(ng, slot, case.frame(k, ng))
            m.set_frame(ng, slot, case.stored(k, ng))
    T.locate(case.release, t_b=1)
    m.init_particles(case.release, tb=1)
    mI = 1                                  # ROMSPath.f90:422
    recs = []
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
            mI += 1                         # 533
            if done % every == 0:           # 536-544
                g = T.output_record(mI, n=n_out)
                o = m.output_record(mI)
                recs.append((g, o))
                mI = 0                      # 2035
    T.close()
    return recs


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b, dtype=a.dtype)
    return int((~((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b)))).sum())


def _check(recs, n=None):
    assert recs
    for r, (g, o) in enumerate(recs):
        bad = {k: _same(v, o[k][: len(v)]) for k, v in g.items()}
        bad = {k: v for k, v in bad.items() if v}
        assert not bad, f"record {r}: columns differing (particle counts): {bad}"


@pytest.mark.parametrize("resort", [0, 6])
def test_records_with_diagnostics(resort):
    case = harness.make_case("tiny", 200, seed=3, spec_over={"diag": True}, param_over=harness.DIAG_PARAMS)
    recs = _run(case, 72, 12, resort=resort)
    _check(recs)
    g = recs[-1][0]
    assert set(g) == {"lon", "lat", "zp", "age", "status", "gid", "salt", "temp", "hob", "bustr", "bvstr"}
    assert np.all((g["lon"] > -72) & (g["lon"] < -69)) and np.all((g["lat"] > 40) & (g["lat"] < 43))
    assert np.all(g["salt"][g["status"] == 1.0] > 30.0)


def test_records_instantaneous_salt_temp():
    case = harness.make_case("tiny", 150, seed=4, spec_over={"diag": True}, param_over={"salttemp_on": 1})
    _check(_run(case, 36, 12, variant="split"))


def test_records_nested_grids():
    case = harness.make_case("nest_tiny", 300, seed=3)
    recs = _run(case, 48, 12, resort=6)
    _check(recs)
    assert len(np.unique(recs[-1][0]["gid"])) > 1


def test_record_subset():
    case = harness.make_case("tiny", 200, seed=5, spec_over={"diag": True}, param_over=harness.DIAG_PARAMS)
    recs = _run(case, 24, 12, resort=6, n_out=120)
    _check(recs)
    assert len(recs[0][0]["lon"]) == 120


def test_record_refusals():
    case = harness.make_case("tiny", 50, seed=3, spec_over={"diag": True}, param_over=harness.DIAG_PARAMS)
    T = Tracker(case.specs, case.grids, case.params, numpar=50)
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, case.frame(k))
    T.locate(case.release, t_b=1)
    with pytest.raises(RomsPathError, match="mI"):
        T.output_record(0)
    T.close()
    grids = [{k: v for k, v in g.items() if k not in ("lon_rho", "lat_rho")} for g in case.grids]
    T = Tracker(case.specs, grids, {**case.params, "salttemp_on": 0, "salttemp_mean": 0, "write_bottom": 0},
                numpar=50)
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, case.frame(k))
    T.locate(case.release, t_b=1)
    with pytest.raises(RomsPathError, match="rp_set_grid_lonlat"):
        T.output_record(1)
    out = {"zp": np.empty(50), "age": np.empty(50)}
    T.output_record(1, out=out)
    with pytest.raises(RomsPathError, match="off"):
        T.output_record(1, out={"salt": np.empty(50)})
    T.close()
