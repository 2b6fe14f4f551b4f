"""Batched launches: rp_step_n (one CUDA graph per call) and the cap on
resident blocks per SM (more particles per thread) leave every result
unchanged, bit for bit (tolerance 0 ulp): the exact form against the CPU
oracle, the mixed form against its own step-by-step run."""
import numpy as np
import pytest

import harness

pytestmark = pytest.mark.gpu


def _run(case, nsteps, field_dtype=None, graph=False, blocks_per_sm=0, resort=0, seed=7):
    from romspath_b200 import Tracker, schedule
    T = Tracker(case.specs, case.grids, case.params, numpar=case.release.z.shape[0],
                field_dtype=field_dtype or case.spec.field_dtype, stokes=case.spec.stokes, seed=seed,
                scl=case.scl, off=case.off, resort=resort, blocks_per_sm=blocks_per_sm)
    for (k, slot) in schedule.initial_loads():
        for ng in range(1, case.ngrid + 1):
            T.upload_frame(ng, slot, case.frame(k, ng))
    T.locate(case.release, t_b=1)
    done = 0
    for ext, internal in harness._steps(case, nsteps):
        for (k, slot) in ext.loads:
            for ng in range(1, case.ngrid + 1):
                T.upload_frame(ng, slot, case.frame(k, ng))
        its = internal[: nsteps - done]
        if graph:
            T.step_n(its)
        else:
            for it in its:
                T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
        done += len(its)
        if done >= nsteps:
            break
    st = T.get_particles()
    T.close()
    return st


@pytest.mark.parametrize("name,npart,nsteps", [("tiny", 300, 40), ("nest_tiny", 400, 30),
                                               ("nest3_tiny", 600, 36)])
def test_graph_steps_match_oracle(name, npart, nsteps):
    case = harness.make_case(name, npart, seed=5)
    g = _run(case, nsteps, graph=True, blocks_per_sm=2, resort=6)
    o, _ = harness.run_oracle(case, nsteps, noise="philox", seed=7)
    bad = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not bad, bad


@pytest.mark.parametrize("kind", ["mixed", "mixed-i16"])
def test_graph_and_cap_mixed_match_step_by_step(kind):
    case = harness.make_case("tiny", 400, seed=6)
    a = _run(case, 36, field_dtype=kind)
    b = _run(case, 36, field_dtype=kind, graph=True, blocks_per_sm=1, resort=12)
    bad = {k: v for k, v in harness.compare(a, b).items() if v}
    assert not bad, bad


def _run_forms(case, nsteps, field_dtype, forms, seed=7):
    """One run whose kernel form changes every 6 internal steps (cycling
    through `forms`), re-sorted every 6 steps."""
    from romspath_b200 import Tracker, schedule
    T = Tracker(case.specs, case.grids, case.params, numpar=case.release.z.shape[0], field_dtype=field_dtype,
                stokes=case.spec.stokes, seed=seed, scl=case.scl, off=case.off, resort=6)
    for (k, slot) in schedule.initial_loads():
        for ng in range(1, case.ngrid + 1):
            T.upload_frame(ng, slot, case.frame(k, ng))
    T.locate(case.release, t_b=1)
    done = 0
    for ext, internal in harness._steps(case, nsteps):
        for (k, slot) in ext.loads:
            for ng in range(1, case.ngrid + 1):
                T.upload_frame(ng, slot, case.frame(k, ng))
        for it in internal[: nsteps - done]:
            T.set_kernel_form(forms[(done // 6) % len(forms)])
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            done += 1
        if done >= nsteps:
            break
    st = T.get_particles()
    T.close()
    return st


@pytest.mark.parametrize("name", ["tiny", "nest3_tiny"])
def test_kernel_forms_switched_exact_form(name):
    """The exact form under every kernel form, switched between steps: bit
    for bit the oracle's result."""
    case = harness.make_case(name, 400, seed=5)
    g = _run_forms(case, 36, case.spec.field_dtype, ["fused", "split", "smem", "fused-noprefetch", "fused-b64",
                                                      "fused-b256"])
    o, _ = harness.run_oracle(case, 36, noise="philox", seed=7)
    bad = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not bad, bad


@pytest.mark.parametrize("kind", ["mixed", "mixed-i16"])
@pytest.mark.parametrize("name", ["tiny", "cfg1"])
def test_kernel_forms_mixed(name, kind):
    """The mixed form's kernel forms agree: the fused kernel with and
    without the back substitution's load-ahead bit for bit; the split forms
    (local and shared-memory workspace) within 1e-6 cells and 1e-4 m of the
    fused kernel, with the same statuses and grids (they differ only in the
    rounding of contracted products)."""
    case = harness.make_case(name, 800, seed=6)
    a = _run_forms(case, 36, kind, ["fused"])
    b = _run_forms(case, 36, kind, ["fused-noprefetch"])
    bad = {k: v for k, v in harness.compare(a, b).items() if v}
    assert not bad, bad
    c = _run_forms(case, 36, kind, ["fused-b64", "fused-b256", "fused"])
    bad = {k: v for k, v in harness.compare(a, c).items() if v}
    assert not bad, bad                            # the block size changes nothing
    for forms in (["smem"], ["split"], ["fused", "smem", "split"]):
        c = _run_forms(case, 36, kind, forms)
        d = np.hypot(a["x"] - c["x"], a["y"] - c["y"])
        assert np.nanmax(d) < 1e-6, (forms, np.nanmax(d))
        assert np.nanmax(np.abs(a["z"] - c["z"])) < 1e-4, forms
        assert np.array_equal(a["status"], c["status"]) and np.array_equal(a["gid"], c["gid"]), forms
