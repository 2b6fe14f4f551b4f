"""Frames from page-locked host arrays are copied by DMA straight into the
device staging (no host-side copy); results are the same, bit for bit
(tolerance 0 ulp), as the oracle's, and the caller may overwrite its arrays
as soon as rp_upload_frame returns."""
import numpy as np
import pytest

import harness

pytestmark = pytest.mark.gpu


def _pinned(a, keep):
    import torch
    t = torch.empty(a.size, dtype={np.float32: torch.float32, np.float64: torch.float64}[a.dtype.type],
                    pin_memory=True)
    buf = t.numpy()
    buf[:] = np.asfortranarray(a).ravel(order="F")
    keep.append(t)
    return buf.reshape(a.shape, order="F")


@pytest.mark.parametrize("sov", [None, {"field_dtype": "f32", "stokes": True}])
def test_pinned_frames_match_oracle(sov):
    from romspath_b200 import Tracker, schedule
    case = harness.make_case("tiny", 200, seed=4, spec_over=sov)
    keep = []
    T = Tracker(case.specs, case.grids, case.params, numpar=200, field_dtype=case.spec.field_dtype,
                stokes=case.spec.stokes, seed=7)

    def upload(slot, k):
        f = {q: _pinned(v, keep) for q, v in case.frame(k).items()}
        T.upload_frame(1, slot, f)
        for v in f.values():                  # the caller reuses its arrays at once
            v[...] = np.nan

    for (k, slot) in schedule.initial_loads():
        upload(slot, k)
    T.locate(case.release, t_b=1)
    done = 0
    for ext, internal in harness._steps(case, 36):
        for (k, slot) in ext.loads:
            upload(slot, k)
        for it in internal:
            if done >= 36:
                break
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            done += 1
    g = T.get_particles()
    T.close()
    o, _ = harness.run_oracle(case, 36, noise="philox", seed=7)
    bad = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not bad, bad
