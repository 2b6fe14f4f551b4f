"""Edge cases of the particle set: no particles at all, counts that do not
fill a 128-thread block (1, 127, 129, 257), and the full config-2 size plus
one particle (1,048,577: one more than the bench's blocks cover) — each
bit-identical to the oracle in the exact form, and the mixed form running
on the same sets."""
import os

import numpy as np
import pytest

import harness
from romspath_b200 import Tracker, schedule, synth

pytestmark = pytest.mark.gpu


def _same(g, o, what):
    bad = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not bad, f"{what}: fields differing (particle counts): {bad}"


@pytest.mark.parametrize("form", ["f64", "mixed"])
def test_no_particles(form):
    case = harness.make_case("tiny", 10, seed=1)
    T = Tracker(case.specs, case.grids, case.params, numpar=0, field_dtype=form, seed=3, resort=2)
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, case.frame(k))
    empty = synth.Release(ipos=np.zeros((1, 0)), jpos=np.zeros((1, 0)), z=np.zeros(0), dob=np.zeros(0))
    T.locate(empty, t_b=1)
    for _, internal in harness._steps(case, 6):
        for it in internal[:6]:
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
        break
    st = T.get_particles()
    assert all(v.shape == (0,) for v in st.values())
    T.close()


@pytest.mark.parametrize("npart", [1, 127, 129, 257])
@pytest.mark.parametrize("resort", [0, 5])
def test_ragged_counts_bit_exact(npart, resort):
    case = harness.make_case("tiny", npart, seed=npart)
    g, T = harness.run_gpu(case, 24, noise="philox", seed=9, resort=resort)
    T.close()
    o, _ = harness.run_oracle(case, 24, noise="philox", seed=9)
    _same(g, o, f"{npart} particles")
    m, T = harness.run_gpu(case, 24, noise="philox", seed=9, field_dtype="mixed", resort=resort)
    T.close()
    assert m["x"].shape == (npart,) and np.all(np.isfinite(m["x"]))


def test_full_size_bit_exact():
    """The config-2 grid (512 x 384 x 30, FP32 fields, Stokes, Kh = 1) with
    1,048,577 particles: two internal steps, the state re-sorted by cell
    before each, every column equal to the oracle's."""
    npart = (1 << 20) + 1
    case = harness.make_case("cfg2", npart, seed=4)
    g, T = harness.run_gpu(case, 2, noise="philox", seed=5, resort=1)
    T.close()
    o, _ = harness.run_oracle(case, 2, noise="philox", seed=5, nthreads=os.cpu_count() or 8)
    assert np.isin(g["status"], [1.0, np.float32(1.1), np.float32(1.2)]).sum() > npart // 2
    _same(g, o, "1,048,577 particles")
