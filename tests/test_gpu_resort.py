"""Re-sorting the particle state by grid and cell leaves every result
unchanged, bit for bit (tolerance 0 ulp): each particle's arithmetic does
not depend on its slot, and its noise is keyed on its id.

The exact form with re-sorting every few steps is compared with the CPU
oracle (single and nested grids, Philox and hook-fed noise); the mixed form
with re-sorting is compared with itself without it.  Results come back in
the caller's order (particle k = id - id base)."""
import numpy as np
import pytest

import harness

pytestmark = pytest.mark.gpu

CASES = [
    ("tiny-philox", "tiny", 300, 36, "philox"),
    ("tiny-hook", "tiny", 200, 24, "hook"),
    ("nest-philox", "nest_tiny", 400, 48, "philox"),
]


@pytest.mark.parametrize("cid,name,npart,nsteps,noise", CASES, ids=[c[0] for c in CASES])
def test_resorted_exact_form_matches_oracle(cid, name, npart, nsteps, noise):
    case = harness.make_case(name, npart, seed=7)
    hook = harness.noise_array(case, nsteps) if noise == "hook" else None
    g, T = harness.run_gpu(case, nsteps, noise=noise, hook=hook, resort=5)
    T.close()
    o, _ = harness.run_oracle(case, nsteps, noise=noise, hook=hook)
    bad = {k: v for k, v in harness.compare(g, o).items() if v}
    assert not bad, f"{cid}: {bad}"


class _DevArray:
    """A device column seen through __cuda_array_interface__."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


def test_resort_changes_the_order_but_not_the_results():
    """The device columns are really permuted (ids no longer ascending),
    while a partial read returns the caller's first n particles."""
    import torch
    case = harness.make_case("tiny", 256, seed=2)
    g, T = harness.run_gpu(case, 12, noise="philox", resort=1)
    st = T.device_state()
    T.synchronize()
    ids = torch.as_tensor(_DevArray(st.pid, 256, "<u4"), device="cuda").cpu().numpy()
    assert sorted(ids.tolist()) == list(range(256))
    assert not np.array_equal(ids, np.arange(256))
    part = T.get_particles(100)
    full = T.get_particles()
    for k in ("x", "y", "z", "status", "flags"):
        assert np.array_equal(part[k], full[k][:100])
    T.close()
    ref, T0 = harness.run_gpu(case, 12, noise="philox")
    T0.close()
    bad = {k: v for k, v in harness.compare(g, ref).items() if v}
    assert not bad, bad


@pytest.mark.parametrize("kind", ["mixed", "mixed-i16"])
def test_resorted_mixed_form_matches_unsorted(kind):
    case = harness.make_case("tiny", 400, seed=4)
    a, T0 = harness.run_gpu(case, 36, noise="philox", field_dtype=kind)
    b, T1 = harness.run_gpu(case, 36, noise="philox", field_dtype=kind, resort=4)
    T0.close()
    T1.close()
    bad = {k: v for k, v in harness.compare(a, b).items() if v}
    assert not bad, bad
