"""A driver that reads frames ahead: each interval's steps are enqueued
(one graph), then the next interval's frame is uploaded while they run,
then the particles are read back.  A step binds its ring slots when it is
enqueued, so the exact form still equals the oracle bit for bit, also with
re-sorting and nested grids."""
import numpy as np
import pytest

import harness
from romspath_b200 import Tracker, schedule

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,npart,resort", [("tiny", 300, 0), ("tiny", 300, 6), ("nest_tiny", 400, 6)])
def test_read_ahead_upload_equals_oracle(name, npart, resort):
    case = harness.make_case(name, npart, seed=3)
    nsteps = 48
    T = Tracker(case.specs, case.grids, case.params, numpar=npart, seed=7, scl=case.scl, off=case.off,
                resort=resort)
    for (k, slot) in schedule.initial_loads():
        for ng in range(1, case.ngrid + 1):
            T.upload_frame(ng, slot, case.frame(k, ng))
    T.locate(case.release, t_b=1)
    exts = [e for e, _ in harness._steps(case, nsteps)]
    done = 0
    for (k, slot) in exts[0].loads:
        for ng in range(1, case.ngrid + 1):
            T.upload_frame(ng, slot, case.frame(k, ng))
    for j, e in enumerate(exts):
        its = e.internal[: nsteps - done]
        T.step_n(its)
        done += len(its)
        if j + 1 < len(exts):
            for (k, slot) in exts[j + 1].loads:
                for ng in range(1, case.ngrid + 1):
                    T.upload_frame(ng, slot, case.frame(k, ng))
        g = T.get_particles()
    T.close()
    assert done == nsteps
    o, _ = harness.run_oracle(case, nsteps)
    bad = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not bad, bad
