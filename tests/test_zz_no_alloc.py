"""rp_step_noalloc: the allocation-free step gives rp_step's results.

Some callers cannot allocate device memory when they step particles (a
driver whose particle arrays already live on the device in its own data
regions, a framework whose allocator owns the device memory, a time loop
that must not call cudaMalloc because it synchronises the device).  For
them rp_step_noalloc runs the split step on caller-owned device columns and
keeps its one scratch array in a fixed device buffer.  This test gives it
particle columns allocated by the caller (through torch, not by the
library) and checks two consecutive calls against rp_step, bit for bit (the
tolerance of every parity test here: 0 ulp).  It sits in its own file,
collected last.
"""
import ctypes as C

import numpy as np
import pytest

import harness

pytestmark = pytest.mark.gpu


def _caller_state(torch, st, dob, n):
    """Device columns owned by the caller, initialised from a host state."""
    dev = torch.device("cuda", 0)
    cols = {}
    for k in ("x", "y", "z", "age", "status", "wd", "zeta", "bath"):
        cols[k] = torch.tensor(st[k], dtype=torch.float64, device=dev)
    cols["dob"] = torch.tensor(dob, dtype=torch.float64, device=dev)
    cols["gid"] = torch.tensor(st["gid"].astype(np.int32), device=dev)
    cols["isin"] = torch.tensor(st["isin"].astype(np.int8), device=dev)
    cols["pid"] = torch.arange(n, dtype=torch.int32, device=dev)
    cols["flags"] = torch.tensor(st["flags"].astype(np.int32), device=dev)
    from romspath_b200 import _lib
    S = _lib.RpDeviceState()
    S.n = n
    for k, t in cols.items():
        setattr(S, k, t.data_ptr())
    return S, cols


def _host(cols):
    out = {k: cols[k].cpu().numpy() for k in ("x", "y", "z", "age", "status", "wd", "zeta", "bath")}
    out["gid"] = cols["gid"].cpu().numpy().astype(np.float64)
    out["isin"] = cols["isin"].cpu().numpy().astype(np.int32)
    out["flags"] = cols["flags"].cpu().numpy().view(np.uint32)
    return out


def test_noalloc_step_matches_rp_step_two_calls():
    import torch
    from romspath_b200 import Tracker, schedule
    n = 256
    case = harness.make_case("tiny", n, seed=8)       # RK4 + HTurb + VTurb on
    mk = lambda: Tracker([case.spec], [case.grid], case.params, numpar=n, field_dtype=case.spec.field_dtype,
                         stokes=case.spec.stokes, seed=3, variant="split")
    ref, na = mk(), mk()
    for T in (ref, na):
        for (k, slot) in schedule.initial_loads():
            T.upload_frame(1, slot, case.frame(k))
        T.locate(case.release, t_b=1)
    S, cols = _caller_state(torch, na.get_particles(), case.release.dob, n)
    torch.cuda.synchronize()
    ext = list(schedule.external_steps(1.0, 3600, 300))[1]
    for call, it in enumerate(ext.internal[:2]):
        ref.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
        exa = (C.c_double * 3)(*it.ex)
        ixa = (C.c_double * 3)(*it.ix)
        rc = na.L.rp_step_noalloc(na.h, C.byref(S), exa, ixa, it.ets, it.tb, it.tc, it.tf)
        assert rc == 0, rc
        na.synchronize()
        g = _host(cols)
        r = ref.get_particles()
        diff = {k: v for k, v in harness.compare(g, r).items() if v}
        assert not diff, f"call {call + 1}: {diff}"
    moved = np.isin(g["status"], [1.0, np.float32(1.1), np.float32(1.2)]).sum()
    assert moved > 0
    # sizes beyond the fixed scratch are refused with a clear error
    from romspath_b200 import _lib
    S.n = _lib.NOALLOC_MAX_PARTICLES + 1
    exa = (C.c_double * 3)(*ext.ex)
    rc = na.L.rp_step_noalloc(na.h, C.byref(S), exa, exa, 2, 1, 2, 3)
    assert rc == -1
    buf = C.create_string_buffer(256)
    na.L.rp_last_error(na.h, buf, 256)
    assert b"RP_NOALLOC_MAX_PARTICLES" in buf.value
    ref.close()
    na.close()
