"""Asynchronous output records (rp_output_record_async / rp_output_wait):
a record packed after an interval's steps and copied into page-locked
arrays while the next interval runs equals the synchronous record of the
same run, bit for bit, record after record (diagnostics' resets included)."""
import numpy as np
import pytest
import torch

import harness
from romspath_b200 import Tracker, schedule
from romspath_b200.tracker import RomsPathError

pytestmark = pytest.mark.gpu


def _pinned(n):
    t = torch.empty(n, dtype=torch.float64, pin_memory=True)
    return t.numpy(), t


def _tracker(case, npart):
    T = Tracker(case.specs, case.grids, case.params, numpar=npart, seed=7, resort=6)
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, case.frame(k))
    T.locate(case.release, t_b=1)
    return T


@pytest.mark.parametrize("form", ["f64", "mixed"])
def test_async_records_equal_sync_records(form):
    npart = 300
    case = harness.make_case("tiny", npart, seed=5, spec_over={"diag": True}, param_over=harness.DIAG_PARAMS)
    A = Tracker(case.specs, case.grids, case.params, numpar=npart, seed=7, resort=6, field_dtype=form)
    B = Tracker(case.specs, case.grids, case.params, numpar=npart, seed=7, resort=6, field_dtype=form)
    for T in (A, B):
        for (k, slot) in schedule.initial_loads():
            T.upload_frame(1, slot, case.frame(k))
        T.locate(case.release, t_b=1)
    keep = []
    bufs = []
    for _ in range(2):
        d = {}
        for k in Tracker.RECORD:
            d[k], t = _pinned(npart)
            keep.append(t)
        bufs.append(d)
    exts = [e for e, _ in harness._steps(case, 48)]
    sync, got = [], []
    mI = 1
    for j, e in enumerate(exts[:4]):
        for (k, slot) in e.loads:
            A.upload_frame(1, slot, case.frame(k))
            B.upload_frame(1, slot, case.frame(k))
        A.step_n(e.internal)
        B.step_n(e.internal)
        mI += len(e.internal)
        sync.append({k: v.copy() for k, v in A.output_record(mI).items()})
        B.output_record_async(mI, bufs[j % 2])
        B.output_wait()
        got.append({k: v.copy() for k, v in bufs[j % 2].items()})
        mI = 0
    A.close()
    B.close()
    assert len(got) == 4
    for r, (a, b) in enumerate(zip(sync, got)):
        for k in a:
            assert np.array_equal(a[k].view(np.uint64), b[k].view(np.uint64)), (r, k)


def test_async_overlaps_next_interval_and_refuses_pageable_arrays():
    npart = 300
    case = harness.make_case("tiny", npart, seed=6)
    A = _tracker(case, npart)
    B = _tracker(case, npart)
    keep = []
    out = {}
    for k in ("lon", "lat", "zp", "age", "status", "gid"):
        out[k], t = _pinned(npart)
        keep.append(t)
    exts = [e for e, _ in harness._steps(case, 36)]
    # record after interval 0, then interval 1 is enqueued before waiting
    for T in (A, B):
        T.step_n(exts[0].internal)
    ref = A.output_record(1)
    B.output_record_async(1, out)
    for (k, slot) in exts[1].loads:
        B.upload_frame(1, slot, case.frame(k))
    B.step_n(exts[1].internal)
    B.output_wait()
    for k in out:
        assert np.array_equal(ref[k], out[k]), k
    with pytest.raises(RomsPathError, match="page-locked"):
        B.output_record_async(1, {"zp": np.empty(npart)})
    A.close()
    B.close()
