"""The adjoint pair split over particle shards, as ranks of a multi-GPU run
hold them: two contexts with disjoint blocks of the release and global id
bases (rp_set_id_base) give each particle the same final position and the
same gradient as one context with all particles, bit for bit, and their
dL/dkappa values sum to the one context's (the all-reduce a multi-GPU run
does at loss time; equal to rounding of the sum's order)."""
import numpy as np
import pytest

import harness
from romspath_b200 import replicas

pytestmark = pytest.mark.gpu

TARGET = (12.0, 10.0)


def _run(case, rel, base):
    from romspath_b200 import Tracker, schedule
    from romspath_b200.adjoint import Adjoint, attribution_loss, step_table
    n = rel.z.shape[0]
    T = Tracker(case.specs, case.grids, case.params, numpar=n, field_dtype="f64", seed=7)
    T.set_id_base(base)
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, case.frame(k))
    T.locate(rel, t_b=1)
    steps, _ = step_table(2.0, int(case.params["dt"]), int(case.params["idt"]))
    steps = steps[:30]
    kmax = max(max(s.frame_b, s.frame_c, s.frame_f) for s in steps)
    adj = Adjoint(T)
    adj.load_frames(kmax, lambda ng, k: case.frame(k, ng))
    adj.forward(steps, kappa=1.0, checkpoint_every=8)
    fin = T.get_particles()
    L, gx, gy = attribution_loss(fin["x"], fin["y"], TARGET)
    ax, ay, az, ak = adj.backward(gx, gy, np.zeros_like(gx))
    T.close()
    return fin, L, (ax, ay, az), ak


def test_shards_reproduce_one_context():
    case = harness.make_case("tiny", 240, seed=11)
    full, L, g, ak = _run(case, case.release, 0)
    assert abs(ak) > 0 and L > 1.0
    parts = []
    for r in range(2):
        rel, start = replicas.shard_release(case.release, r, 2)
        parts.append((start,) + _run(case, rel, start))
    for k in ("x", "y", "z", "status"):
        cat = np.concatenate([p[1][k] for p in parts])
        assert np.array_equal(cat.view(np.uint64), full[k].view(np.uint64)), k
    for q in range(3):
        cat = np.concatenate([p[3][q] for p in parts])
        assert np.array_equal(cat.view(np.uint64), g[q].view(np.uint64)), q
    assert abs(sum(p[2] for p in parts) - L) <= 1e-12 * L
    ks = sum(p[4] for p in parts)
    assert abs(ks - ak) <= 1e-12 * abs(ak)
