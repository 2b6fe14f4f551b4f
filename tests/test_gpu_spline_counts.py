"""Counting of VTurb's smoothing-spline fits and chol1d passes
(rp_count_spline_passes / rp_spline_pass_counts).  In the exact form the
fit (smooth, pppack.f90:5108-5317) takes the reference's secant sequence,
so its counts equal the oracle's: one fit per particle-step with VTurb,
and 1 + secant iterations chol1d passes per fit (the first pass, at p = 0
or p = 1, then one per secant evaluation).  Counting changes no result."""
import numpy as np
import pytest

import harness
from romspath_b200 import Tracker
from romspath_b200.tracker import RomsPathError

pytestmark = pytest.mark.gpu

NSTEPS = 24


def _counted(case, variant="fused", field_dtype=None, resort=0):
    T = Tracker(case.specs, case.grids, case.params, numpar=case.release.z.shape[0],
                field_dtype=field_dtype or case.spec.field_dtype, stokes=case.spec.stokes, seed=5,
                scl=case.scl, off=case.off, variant=variant, resort=resort)
    T.count_spline_passes(True)
    g, T = harness.run_gpu(case, NSTEPS, noise="philox", seed=5, tracker=T)
    fits, passes = T.spline_pass_counts()
    return g, T, fits, passes


@pytest.mark.parametrize("variant,resort", [("fused", 0), ("split", 0), ("fused", 6)])
def test_exact_counts_equal_oracle(variant, resort):
    case = harness.make_case("tiny", 300, seed=2)
    g, T, fits, passes = _counted(case, variant=variant, resort=resort)
    T.close()
    stats = []
    o, _ = harness.run_oracle(case, NSTEPS, noise="philox", seed=5, spline_stats=stats)
    diff = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not diff, diff
    ofits = sum(s[0] for s in stats)
    oiters = sum(s[1] for s in stats)
    assert ofits > 0
    assert fits == ofits
    assert passes == ofits + oiters


def test_counting_changes_nothing_and_stops():
    case = harness.make_case("tiny", 300, seed=3)
    g, T, fits, passes = _counted(case)
    last = [it for _, internal in harness._steps(case, NSTEPS) for it in internal][NSTEPS - 1]
    T.count_spline_passes(False)
    T.step(last.ex, last.ix, last.ets, last.tb, last.tc, last.tf)
    assert T.spline_pass_counts() == (fits, passes)
    T.count_spline_passes(True)
    assert T.spline_pass_counts() == (0, 0)
    T.step(last.ex, last.ix, last.ets, last.tb, last.tc, last.tf)
    f3, p3 = T.spline_pass_counts()
    assert 0 < f3 <= p3
    T.close()
    h, U = harness.run_gpu(case, NSTEPS, noise="philox", seed=5)
    U.close()
    diff = {k: v for k, v in harness.compare(g, h).items() if v}
    assert not diff, diff


def test_mixed_counts_warm_start():
    """The mixed form starts each particle's secant search from its previous
    smoothing parameter: after the first step most fits take fewer passes
    than the reference's cold start."""
    case = harness.make_case("tiny", 300, seed=2)
    _, T, fits, passes = _counted(case, field_dtype="mixed")
    T.close()
    stats = []
    harness.run_oracle(case, NSTEPS, noise="philox", seed=5, spline_stats=stats)
    ofits = sum(s[0] for s in stats)
    oiters = sum(s[1] for s in stats)
    assert abs(fits - ofits) <= 0.02 * ofits
    assert fits <= passes
    assert passes / fits < (ofits + oiters) / ofits


def test_counts_before_start_refused():
    case = harness.make_case("tiny", 50, seed=2)
    T = Tracker(case.specs, case.grids, case.params, numpar=50, seed=5)
    with pytest.raises(RomsPathError):
        T.spline_pass_counts()
    T.close()
