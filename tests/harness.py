"""Run the CUDA path and the CPU oracle side by side on the same inputs.

Used by the GPU parity tests and by ``__graft_entry__.smoke``.  Both sides
get identical grids, identical stored frame values (FP64 sums of Stokes
drift rounded to the device storage precision), identical initial releases
and identical noise (noise hook arrays, or Philox with the same key and
step counter), and follow the same frame-slot schedule of the Fortran
driver (``romspath_b200.schedule``).
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Optional

import numpy as np

from romspath_b200 import schedule, synth

FIELDS = ("x", "y", "z", "age", "status", "gid", "isin", "wd", "zeta", "bath", "flags")


@dataclasses.dataclass
class Case:
    name: str
    spec: synth.GridSpec
    grid: Dict[str, np.ndarray]
    params: dict
    release: synth.Release
    frames: Dict[int, Dict[str, np.ndarray]]

    def frame(self, k: int) -> Dict[str, np.ndarray]:
        if k not in self.frames:
            self.frames[k] = synth.make_frame(self.spec, self.grid, (k - 1) * float(self.params["dt"]))
        return self.frames[k]

    def stored(self, k: int) -> Dict[str, np.ndarray]:
        return synth.stored_frame(self.frame(k), self.spec.field_dtype, self.spec.stokes)


def make_case(name: str, npart: int, seed: int = 0, spec_over: Optional[dict] = None,
              param_over: Optional[dict] = None) -> Case:
    spec = synth.config_spec(name)[0]
    if spec_over:
        spec = dataclasses.replace(spec, **spec_over)
    grid = synth.make_grid(spec)
    params = dict(synth.config_params(name))
    if param_over:
        params.update(param_over)
    frames: Dict[int, Dict[str, np.ndarray]] = {}
    c = Case(name, spec, grid, params, None, frames)  # type: ignore[arg-type]
    c.release = synth.uniform_release(spec, grid, c.frame(1), npart, seed=seed)
    return c


def noise_array(case: Case, nsteps: int, seed: int = 123) -> np.ndarray:
    ndraw = 2 + int(case.params["idt"]) // int(case.params["deltat"])
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nsteps, case.release.z.shape[0], ndraw))


def _steps(case: Case, nsteps: int):
    days = (nsteps * case.params["idt"]) / 86400.0 + 1.0
    k = 0
    for ext in schedule.external_steps(days, int(case.params["dt"]), int(case.params["idt"])):
        yield ext, ext.internal
        k += len(ext.internal)
        if k >= nsteps:
            return


def run_gpu(case: Case, nsteps: int, noise: str = "philox", seed: int = 7,
            hook: Optional[np.ndarray] = None, tracker=None, variant: str = "split"):
    from romspath_b200 import Tracker
    T = tracker or Tracker([case.spec], [case.grid], case.params, numpar=case.release.z.shape[0],
                           field_dtype=case.spec.field_dtype, stokes=case.spec.stokes, seed=seed,
                           variant=variant)
    for (k, slot) in schedule.initial_loads():
        T.upload_frame(1, slot, case.frame(k))
    T.locate(case.release, t_b=1)
    if noise == "hook":
        T.set_noise_hook(hook)
    done = 0
    for ext, internal in _steps(case, nsteps):
        for (k, slot) in ext.loads:
            T.upload_frame(1, slot, case.frame(k))
        for it in internal:
            if done >= nsteps:
                break
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            done += 1
    st = T.get_particles()
    return st, T


def run_oracle(case: Case, nsteps: int, noise: str = "philox", seed: int = 7,
               hook: Optional[np.ndarray] = None, nthreads: int = 8):
    from oracle import oracle as O
    m = O.OracleModel([case.spec], [case.grid], case.params)
    for (k, slot) in schedule.initial_loads():
        m.set_frame(1, slot, case.stored(k))
    m.init_particles(case.release, tb=1)
    done = 0
    for ext, internal in _steps(case, nsteps):
        for (k, slot) in ext.loads:
            m.set_frame(1, slot, case.stored(k))
        for it in internal:
            if done >= nsteps:
                break
            if noise == "hook":
                m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise="hook", hook=hook[done],
                       nthreads=nthreads)
            else:
                m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise="philox", seed=seed,
                       step_index=it.step_index, nthreads=nthreads)
            done += 1
    st = m.state()
    st["gid"] = st["gid"].astype(np.float64)
    st["isin"] = st["isin"].astype(np.int32)
    return st, m


def compare(g: Dict[str, np.ndarray], o: Dict[str, np.ndarray]) -> Dict[str, int]:
    """Number of particles whose field differs bit-for-bit, per field."""
    out = {}
    for f in FIELDS:
        a = np.asarray(g[f])
        b = np.asarray(o[f]).astype(a.dtype)
        if a.dtype.kind == "f":
            same = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
        else:
            same = a == b
        out[f] = int((~same).sum())
    return out
