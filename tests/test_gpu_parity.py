"""GPU parity: the sm_100a particle step against the CPU oracle, bit for bit.

The FP64 form is compiled without FMA contraction and keeps the reference's
evaluation order, so every particle column must match the oracle exactly
(tolerance 0 ulp) on identical inputs: deterministic runs, runs on
hook-fed noise, and runs on Philox noise (same key and counters; both sides
use the same log/cos series for Box-Muller).
"""
import numpy as np
import pytest

import harness

pytestmark = pytest.mark.gpu


def _assert_same(g, o, what):
    diff = harness.compare(g, o)
    bad = {k: v for k, v in diff.items() if v}
    assert not bad, f"{what}: fields differing (particle counts): {bad}"


CASES = [
    # name, npart, nsteps, noise, spec overrides, param overrides
    ("tiny-det", "tiny", 200, 240, "off", None, {"vturb_on": 0, "hturb_on": 0}),
    ("tiny-hook", "tiny", 200, 60, "hook", None, None),
    ("tiny-philox", "tiny", 200, 60, "philox", None, None),
    ("tiny-oob", "tiny", 200, 60, "philox", None, {"open_ocean_boundary": 1}),
    ("tiny-nsb1", "tiny", 100, 24, "philox", None, {"nsb": 1}),
    ("tiny-nsb2", "tiny", 100, 24, "philox", None, {"nsb": 2}),
    ("tiny-noadv", "tiny", 100, 24, "philox", None, {"scheme": 0}),
    ("tiny-vt1", "tiny", 100, 24, "philox", {"vtransform": 1}, None),
    ("tiny-vt3", "tiny", 100, 24, "philox", {"vtransform": 3}, None),
    ("tiny-f32", "tiny", 200, 36, "philox", {"field_dtype": "f32", "stokes": True}, None),
    ("cfg1-vturb", "cfg1", 300, 30, "philox", None, None),
    ("cfg1-hook", "cfg1", 300, 24, "hook", None, None),
    ("cfg2-philox", "cfg2", 200, 14, "philox", None, None),
    ("nest-det", "nest_tiny", 400, 120, "off", None, {"vturb_on": 0, "hturb_on": 0}),
    ("nest-philox", "nest_tiny", 400, 72, "philox", None, None),
    ("nest-hook", "nest_tiny", 300, 36, "hook", None, None),
    ("nest-oob", "nest_tiny", 300, 60, "philox", None, {"open_ocean_boundary": 1}),
    # two sibling children (5x and 3x) of one parent, config 4's grid order
    ("nest3-det", "nest3_tiny", 600, 96, "off", None, {"vturb_on": 0, "hturb_on": 0}),
    ("nest3-philox", "nest3_tiny", 600, 72, "philox", None, None),
    ("nest3-hook", "nest3_tiny", 400, 36, "hook", None, None),
]


@pytest.mark.parametrize("variant", ["split", "fused"])
@pytest.mark.parametrize("cid,name,npart,nsteps,noise,sov,pov", CASES, ids=[c[0] for c in CASES])
def test_step_bit_exact(cid, name, npart, nsteps, noise, sov, pov, variant):
    case = harness.make_case(name, npart, seed=3, spec_over=sov, param_over=pov)
    hook = harness.noise_array(case, nsteps) if noise == "hook" else None
    g, T = harness.run_gpu(case, nsteps, noise=noise, hook=hook, variant=variant)
    T.close()
    o, _ = harness.run_oracle(case, nsteps, noise=noise, hook=hook)
    _assert_same(g, o, cid)
    # the run must actually have moved particles
    assert np.isin(g["status"], [1.0, np.float32(1.1), np.float32(1.2)]).sum() > 0


def test_staggered_release_and_statuses():
    """Particles released over time (pDOB), skipped before release."""
    case = harness.make_case("tiny", 150, seed=5)
    case.release.dob[:] = np.repeat([0.0, 3000.0, 7500.0], 50)
    g, T = harness.run_gpu(case, 40, noise="philox")
    T.close()
    o, _ = harness.run_oracle(case, 40, noise="philox")
    _assert_same(g, o, "staggered")
    # later releases aged less
    assert g["age"][:50].max() > g["age"][100:].max()


def test_deterministic_1000_steps_within_1e9_cells():
    """Turbulence off: trajectories agree to <= 1e-9 grid cells after 1000
    internal steps (here: exactly)."""
    case = harness.make_case("cfg1", 400, seed=11, param_over={"vturb_on": 0, "hturb_on": 0})
    g, T = harness.run_gpu(case, 1000, noise="off")
    T.close()
    o, _ = harness.run_oracle(case, 1000, noise="off")
    dx = np.abs(g["x"] - o["x"]).max()
    dy = np.abs(g["y"] - o["y"]).max()
    assert dx <= 1e-9 and dy <= 1e-9
    _assert_same(g, o, "1000 steps")


def test_nested_handoff_happens():
    """The nested case actually moves particles between grids."""
    case = harness.make_case("nest_tiny", 400, seed=3)
    g0, T0 = harness.run_gpu(case, 0)
    T0.close()
    g, T = harness.run_gpu(case, 72)
    T.close()
    assert (g0["gid"] != g["gid"]).sum() > 20
    assert set(np.unique(g["gid"])) == {1.0, 2.0}


def test_sibling_nest_handoff_all_directions():
    """The three-grid sibling case moves particles from each child to the
    parent and from the parent into each child."""
    import collections
    case = harness.make_case("nest3_tiny", 600, seed=3)
    g0, T0 = harness.run_gpu(case, 0)
    T0.close()
    g, T = harness.run_gpu(case, 72)
    T.close()
    moves = collections.Counter(zip(g0["gid"].astype(int), g["gid"].astype(int)))
    for a, b in ((1, 3), (2, 3), (3, 1), (3, 2)):
        assert moves[(a, b)] > 0, moves


def test_split_contexts_match_one_context():
    """Two contexts holding disjoint id ranges (one per GPU in a multi-GPU
    run) reproduce one context holding all particles."""
    from romspath_b200 import Tracker, replicas, schedule
    case = harness.make_case("tiny", 300, seed=12)
    full, Tf = harness.run_gpu(case, 30, seed=9)
    Tf.close()
    parts = []
    for rank in range(2):
        rel, start = replicas.shard_release(case.release, rank, 2)
        T = Tracker(case.specs, case.grids, case.params, numpar=rel.z.shape[0], field_dtype="f64", seed=9)
        T.set_id_base(start)
        c2 = harness.Case(case.name, case.specs, case.grids, case.params, rel, case.frames)
        g, _ = harness.run_gpu(c2, 30, seed=9, tracker=T)
        T.close()
        parts.append(g)
    joined = {k: np.concatenate([p[k] for p in parts]) for k in harness.FIELDS}
    diff = {k: v for k, v in harness.compare(joined, full).items() if v}
    assert not diff, diff
