"""Multi-rank path on CPU: two gloo ranks each step their shard of the
particles (the oracle stands in for the GPU step) with global particle ids,
gather to all ranks, and must reproduce a one-rank run bit for bit; the
output-time reductions (the vertical concentration profile, a quantity
summed over particles as dL/dkappa is) equal the one-rank values."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import harness
from romspath_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        case = harness.make_case("nest_tiny", 150, seed=6)
        rel, start = replicas.shard_release(case.release, rank, world)
        case.release = rel
        m = O.OracleModel(case.specs, case.grids, case.params, scl=case.scl, off=case.off)
        from romspath_b200 import schedule
        for (k, slot) in schedule.initial_loads():
            for ng in (1, 2):
                m.set_frame(ng, slot, case.stored(k, ng))
        m.init_particles(rel, tb=1, pid=np.arange(start, start + rel.z.shape[0], dtype=np.uint32))
        for ext in list(schedule.external_steps(1.0, 3600, 300))[:2]:
            for (k, slot) in ext.loads:
                for ng in (1, 2):
                    m.set_frame(ng, slot, case.stored(k, ng))
            for it in ext.internal:
                m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise="philox", seed=3,
                       step_index=it.step_index, nthreads=1)
        st = m.state()
        g = replicas.gather({k: st[k] for k in ("x", "y", "z", "status", "gid", "pid")}, world)
        prof = replicas.global_profile(st)
        # a per-particle additive quantity stands in for dL/dkappa's shares
        gk = replicas.kappa_gradient(float(np.sum(st["x"])))
        if rank == 0:
            np.savez(out, prof=prof, gk=np.array(gk), **g)
    finally:
        dist.destroy_process_group()


def test_shard_blocks_cover_range():
    for n in (0, 1, 7, 150, 1 << 20):
        for w in (1, 2, 3, 8):
            blocks = [replicas.shard(n, r, w) for r in range(w)]
            assert sum(c for _, c in blocks) == n
            assert all(blocks[r][0] + blocks[r][1] == blocks[r + 1][0] for r in range(w - 1))


def test_two_gloo_ranks_match_one_rank(tmp_path):
    out = str(tmp_path / "g.npz")
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    g = np.load(out)
    case = harness.make_case("nest_tiny", 150, seed=6)
    o, _ = harness.run_oracle(case, 24, noise="philox", seed=3, nthreads=1)
    assert np.array_equal(g["pid"], np.arange(150))
    for k in ("x", "y", "z", "status"):
        assert np.array_equal(g[k].view(np.uint64), o[k].view(np.uint64)), k
    assert np.array_equal(g["gid"], o["gid"].astype(np.int32))
    prof = replicas.column_profile(o)
    assert prof.sum() > 100
    assert np.array_equal(g["prof"], prof)
    assert abs(float(g["gk"]) - float(np.sum(o["x"]))) <= 1e-12 * abs(float(np.sum(o["x"])))
