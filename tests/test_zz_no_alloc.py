"""rp_step_noalloc: the allocation-free step gives rp_step's results.

Some callers cannot allocate device memory when they step particles (a
driver whose particle arrays already live on the device in its own data
regions, a framework whose allocator owns the device memory, a time loop
that must not call cudaMalloc because it synchronises the device).  For
them rp_step_noalloc runs the split step on caller-owned device columns and
keeps its one scratch array in a fixed device buffer.  These tests give it
particle columns allocated by the caller (through torch, not by the
library) and check two consecutive calls against rp_step, bit for bit (the
tolerance of every parity test here: 0 ulp), on a single grid with FP64
fields, FP32 fields with Stokes drift, WETDRY masks and two nested grids.
They also check that the calls after the first change neither the device's
free memory nor torch's allocations, and that the step is ordered against
the caller's own stream: the columns are written on a torch side stream
just before the call and read back on it just after, with no host
synchronisation in between.  The file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

import harness

pytestmark = pytest.mark.gpu

COLS64 = ("x", "y", "z", "age", "status", "wd", "zeta", "bath")


def _caller_state(torch, st, dob, n, stream):
    """Device columns owned by the caller, written on `stream` from a host state."""
    dev = torch.device("cuda", 0)
    cols = {}
    with torch.cuda.stream(stream):
        for k in COLS64:
            cols[k] = torch.empty(n, dtype=torch.float64, device=dev)
        cols["dob"] = torch.empty(n, dtype=torch.float64, device=dev)
        cols["gid"] = torch.empty(n, dtype=torch.int32, device=dev)
        cols["isin"] = torch.empty(n, dtype=torch.int8, device=dev)
        cols["pid"] = torch.arange(n, dtype=torch.int32, device=dev)
        cols["flags"] = torch.empty(n, dtype=torch.int32, device=dev)
        # host -> device on the side stream, not waited for by the host
        host = {k: torch.from_numpy(np.ascontiguousarray(st[k])).pin_memory() for k in COLS64}
        host["dob"] = torch.from_numpy(np.ascontiguousarray(dob, dtype=np.float64)).pin_memory()
        host["gid"] = torch.from_numpy(st["gid"].astype(np.int32)).pin_memory()
        host["isin"] = torch.from_numpy(st["isin"].astype(np.int8)).pin_memory()
        host["flags"] = torch.from_numpy(st["flags"].astype(np.int32)).pin_memory()
        for k, h in host.items():
            cols[k].copy_(h, non_blocking=True)
    from romspath_b200 import _lib
    S = _lib.RpDeviceState()
    S.n = n
    for k, t in cols.items():
        setattr(S, k, t.data_ptr())
    S.stream = stream.cuda_stream
    return S, cols, host


def _host(torch, cols, stream):
    """Read the columns back on the caller's stream (copies queued behind the step)."""
    with torch.cuda.stream(stream):
        out = {k: cols[k].to("cpu", non_blocking=True) for k in cols}
    stream.synchronize()
    g = {k: out[k].numpy() for k in COLS64}
    g["gid"] = out["gid"].numpy().astype(np.float64)
    g["isin"] = out["isin"].numpy().astype(np.int32)
    g["flags"] = out["flags"].numpy().view(np.uint32)
    return g


CASES = [
    # id, config, particles, spec overrides, param overrides
    ("f64", "tiny", 256, {}, {}),
    ("f32-stokes", "tiny", 256, {"field_dtype": "f32", "stokes": True}, {}),
    ("wetdry", "tiny", 256, {"wetdry": True}, {"wetdry": 1}),
    ("nested", "nest_tiny", 300, {}, {}),
]


@pytest.mark.parametrize("cid,name,n,sov,pov", CASES, ids=[c[0] for c in CASES])
def test_noalloc_step_matches_rp_step_two_calls(cid, name, n, sov, pov):
    import torch
    from romspath_b200 import Tracker, schedule
    case = harness.make_case(name, n, seed=8, spec_over=sov, param_over=pov)   # RK4 + HTurb + VTurb on
    mk = lambda: Tracker(case.specs, case.grids, case.params, numpar=n, field_dtype=case.spec.field_dtype,
                         stokes=case.spec.stokes, seed=3, scl=case.scl, off=case.off, variant="split")
    ref, na = mk(), mk()
    for T in (ref, na):
        for (k, slot) in schedule.initial_loads():
            for ng in range(1, case.ngrid + 1):
                T.upload_frame(ng, slot, case.frame(k, ng))
        T.locate(case.release, t_b=1)
    side = torch.cuda.Stream()
    S, cols, _pinned = _caller_state(torch, na.get_particles(), case.release.dob, n, side)
    ext = list(schedule.external_steps(1.0, 3600, 300))[1]
    free_after, alloc_after = [], []
    for call, it in enumerate(ext.internal[:3]):
        ref.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
        exa = (C.c_double * 3)(*it.ex)
        ixa = (C.c_double * 3)(*it.ix)
        rc = na.L.rp_step_noalloc(na.h, C.byref(S), exa, ixa, it.ets, it.tb, it.tc, it.tf)
        assert rc == 0, rc
        g = _host(torch, cols, side)
        r = ref.get_particles()
        diff = {k: v for k, v in harness.compare(g, r).items() if v}
        assert not diff, f"{cid} call {call + 1}: {diff}"
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
        alloc_after.append(torch.cuda.memory_stats().get("allocation.all.allocated", 0))
    moved = np.isin(g["status"], [1.0, np.float32(1.1), np.float32(1.2)]).sum()
    assert moved > 0
    # calls after the first allocate nothing: device free memory and torch's
    # allocation count stay put (the read-backs allocate host tensors only)
    assert free_after[1] == free_after[0] and free_after[2] == free_after[1], free_after
    assert alloc_after[2] == alloc_after[1], alloc_after
    ref.close()
    na.close()


def test_noalloc_refuses_oversize():
    import torch
    from romspath_b200 import Tracker, _lib, schedule
    n = 64
    case = harness.make_case("tiny", n, seed=8)
    na = Tracker([case.spec], [case.grid], case.params, numpar=n, field_dtype=case.spec.field_dtype, seed=3,
                 variant="split")
    for (k, slot) in schedule.initial_loads():
        na.upload_frame(1, slot, case.frame(k))
    na.locate(case.release, t_b=1)
    side = torch.cuda.Stream()
    S, cols, _pinned = _caller_state(torch, na.get_particles(), case.release.dob, n, side)
    side.synchronize()
    # sizes beyond the fixed scratch are refused with a clear error
    S.n = _lib.NOALLOC_MAX_PARTICLES + 1
    ext = list(schedule.external_steps(1.0, 3600, 300))[1]
    exa = (C.c_double * 3)(*ext.ex)
    rc = na.L.rp_step_noalloc(na.h, C.byref(S), exa, exa, 2, 1, 2, 3)
    assert rc == -1
    buf = C.create_string_buffer(256)
    na.L.rp_last_error(na.h, buf, 256)
    assert b"RP_NOALLOC_MAX_PARTICLES" in buf.value
    na.close()
