"""Failure handling on a live context, all of it injected on the host.

* The smoothing spline's secant search (pppack.f90:5275-5292) has no
  iteration cap in the reference; here it stops at rp_params.
  spline_max_iter and sets RP_FLAG_SPLINE.  With the cap at 4 and jagged
  AKs columns (the oracle flags 111 of 300 particles in 36 steps), the flag
  must be set on exactly the particles where the oracle (same cap) sets
  it, with every other column bit-identical.
* A frame with NaN diffusivities in one region and NaN velocities in
  another: the step returns RP_OK, every loop ends (bisections narrow, the
  secant search is capped, the column search is guarded), every status is
  one of the reference's values, and the result equals the oracle's bit
  for bit (NaN for NaN).
* Out-of-range grid ids and slots, steps on slots never loaded, oversized
  reads: RP_ERR_ARG / RP_ERR_STATE with a message, and the context keeps
  working (the following steps still match the oracle).
Nothing here faults or hangs the GPU: every failure is an argument or a
value the host hands over.
"""
import ctypes as C

import numpy as np
import pytest

import harness
from romspath_b200 import Tracker, _lib, schedule

pytestmark = pytest.mark.gpu

STATUSES = [0.0, 1.0, np.float32(1.1), np.float32(1.2), -8.0, -9.0]


def _jagged(case):
    """AKs columns made jagged: every other level scaled by 3 (a hard fit)."""
    for k in range(1, 12):
        f = dict(case.frame(k))
        a = np.array(f["aks"], copy=True)
        a[:, :, 1::2] *= 3.0
        f["aks"] = np.asfortranarray(a)
        case.frames[(1, k)] = f


def _tracker(case, **kw):
    return Tracker(case.specs, case.grids, case.params, numpar=case.release.z.shape[0],
                   field_dtype=kw.pop("field_dtype", case.spec.field_dtype), stokes=case.spec.stokes,
                   seed=7, scl=case.scl, off=case.off, **kw)


def _err(T):
    buf = C.create_string_buffer(512)
    T.L.rp_last_error(T.h, buf, 512)
    return buf.value.decode()


@pytest.mark.parametrize("variant", ["fused", "split"])
def test_spline_cap_flags_match_oracle(variant):
    case = harness.make_case("tiny", 300, seed=13)
    _jagged(case)
    T = _tracker(case, spline_max_iter=4, variant=variant)
    g, _ = harness.run_gpu(case, 36, tracker=T)
    T.close()
    o, _ = harness.run_oracle(case, 36, spline_max_iter=4)
    bad = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not bad, bad
    hit = (g["flags"] & _lib.FLAG_SPLINE) != 0
    print("particles with the spline cap hit:", int(hit.sum()), "of", hit.size)
    assert 0 < hit.sum() < hit.size
    # the same run without the cap sets no flag
    T = _tracker(case, variant=variant)
    g2, _ = harness.run_gpu(case, 36, tracker=T)
    T.close()
    assert not ((g2["flags"] & _lib.FLAG_SPLINE) != 0).any()


@pytest.mark.parametrize("kind", ["mixed", "mixed-i16"])
def test_spline_cap_mixed_form(kind):
    case = harness.make_case("tiny", 300, seed=13)
    _jagged(case)
    T = _tracker(case, spline_max_iter=1, field_dtype=kind)
    g, _ = harness.run_gpu(case, 36, tracker=T)
    T.close()
    hit = (g["flags"] & _lib.FLAG_SPLINE) != 0
    assert hit.any()
    assert np.isin(g["status"], STATUSES).all()


def _nan_frames(case):
    """Frames 2.. with NaN AKs over one block of cells and NaN u over another."""
    for k in range(2, 12):
        f = dict(case.frame(k))
        a = np.array(f["aks"], copy=True)
        a[4:10, 4:10, :] = np.nan
        u = np.array(f["u"], copy=True)
        u[14:18, 10:15, :] = np.nan
        f["aks"], f["u"] = np.asfortranarray(a), np.asfortranarray(u)
        case.frames[(1, k)] = f


@pytest.mark.parametrize("variant", ["fused", "split"])
def test_nan_frame_exact_form(variant):
    case = harness.make_case("tiny", 400, seed=14)
    _nan_frames(case)
    T = _tracker(case, variant=variant, resort=6)
    g, _ = harness.run_gpu(case, 36, tracker=T)
    T.close()
    o, _ = harness.run_oracle(case, 36)
    bad = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not bad, bad
    assert np.isin(g["status"], STATUSES).all()
    touched = ~np.isfinite(g["z"]) | ~np.isfinite(g["x"])
    print("particles carrying NaN:", int(touched.sum()))
    assert 0 < touched.sum() < touched.size


@pytest.mark.parametrize("kind", ["mixed", "mixed-i16"])
def test_nan_frame_mixed_form(kind):
    case = harness.make_case("tiny", 400, seed=14)
    _nan_frames(case)
    T = _tracker(case, field_dtype=kind, resort=6)
    g, _ = harness.run_gpu(case, 36, tracker=T)
    T.close()
    assert np.isin(g["status"], STATUSES).all()
    assert np.isfinite(g["age"]).all()


def test_bad_ids_and_slots_on_live_context():
    case = harness.make_case("nest_tiny", 200, seed=15)
    T = _tracker(case)
    L, h = T.L, T.h
    f = case.frame(1)
    arrs = [np.asfortranarray(f[k], dtype=np.float64) for k in ("zeta", "u", "v", "w", "aks")]
    ptrs = [a.ctypes.data_as(_lib.PD) for a in arrs]
    ex = (C.c_double * 3)(0.0, 3600.0, 7200.0)
    ix = (C.c_double * 3)(3300.0, 3600.0, 3900.0)
    # a step before any frame is loaded
    assert L.rp_step(h, ex, ix, 2, 1, 2, 3) == _lib.ERR_STATE
    assert "never loaded" in _err(T)
    # grid ids and slots outside 1..Ngrid / 1..3
    for ng, slot in ((0, 1), (3, 1), (-1, 1), (1, 0), (1, 4), (2, -2)):
        assert L.rp_upload_frame(h, ng, slot, *ptrs, None, None) == _lib.ERR_ARG, (ng, slot)
        assert _err(T)
    # a live context: frames loaded, particles located
    for (k, slot) in schedule.initial_loads():
        for ng in range(1, case.ngrid + 1):
            T.upload_frame(ng, slot, case.frame(k, ng))
    T.locate(case.release, t_b=1)
    for tb, tc, tf in ((0, 2, 3), (1, 4, 3), (1, 2, 0), (-3, 2, 3)):
        assert L.rp_step(h, ex, ix, 2, tb, tc, tf) == _lib.ERR_ARG
        assert "slots" in _err(T)
    n = C.c_int64(case.release.z.shape[0] + 1)
    out = np.zeros(n.value)
    assert L.rp_get_particles(h, n, out.ctypes.data_as(_lib.PD), *([None] * 10)) == _lib.ERR_ARG
    assert "exceeds" in _err(T)
    # the context still steps like the oracle after the refused calls
    g, _ = harness.run_gpu(case, 24, tracker=T)
    T.close()
    o, _ = harness.run_oracle(case, 24)
    bad = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not bad, bad


def test_one_level_grid_refused():
    """A grid with one s-level is refused at creation (the reference's
    linint search does not end there for a point below the first level)."""
    from romspath_b200 import synth
    from romspath_b200.tracker import RomsPathError
    sp = synth.GridSpec(24, 20, 1)
    with pytest.raises(RomsPathError):
        Tracker([sp], [synth.make_grid(sp)], synth.config_params("tiny"), numpar=10)


@pytest.mark.parametrize("kind", ["mixed", "mixed-i16"])
def test_spare_slot_contents_do_not_reach_the_mixed_step(kind):
    """The ring's fourth physical slot (the one an upload fills next) is read
    with every (point, level) word but weighs zero: a NaN frame parked there
    must leave the step's results bit for bit as with a finite one."""
    case = harness.make_case("tiny", 300, seed=21)
    nanf = {k: np.full_like(np.asarray(v, dtype=np.float64), np.nan) if np.ndim(v) else v
            for k, v in case.frame(1).items()}
    outs = []
    for parked in (case.frame(1), nanf):
        T = _tracker(case, field_dtype=kind, resort=0)
        for (k, slot) in schedule.initial_loads():
            T.upload_frame(1, slot, case.frame(k))
        # an upload writes the spare slot and frees the one it replaces:
        # `parked` then frame 1 again into slot 1 leaves `parked` in the spare
        T.upload_frame(1, 1, parked)
        T.upload_frame(1, 1, case.frame(1))
        T.locate(case.release, t_b=1)
        n = 0
        for ext in schedule.external_steps(1.0, int(case.params["dt"]), int(case.params["idt"])):
            if ext.loads:
                break                                  # no upload may overwrite the spare slot
            for it in ext.internal:
                T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
                n += 1
        st = T.get_particles()
        T.close()
        outs.append(st)
    assert n >= 12
    for key in ("x", "y", "z", "status", "age"):
        a, b = np.asarray(outs[0][key]), np.asarray(outs[1][key])
        assert np.array_equal(a.view(np.uint64) if a.dtype == np.float64 else a,
                              b.view(np.uint64) if b.dtype == np.float64 else b), key
    assert np.isfinite(np.asarray(outs[1]["z"])).all()
