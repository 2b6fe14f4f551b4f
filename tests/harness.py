"""Run the CUDA path and the CPU oracle side by side on the same inputs.

Used by the GPU parity tests and by ``__graft_entry__.smoke``.  Both sides
get identical grids (and, for nested grids, identical index maps),
identical stored frame values (FP64 sums of Stokes drift rounded to the
device storage precision), identical initial releases and identical noise
(noise hook arrays, or Philox with the same key and step counter), and
follow the same frame-slot schedule of the Fortran driver
(``romspath_b200.schedule``).
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Optional

import numpy as np

from romspath_b200 import schedule, synth

FIELDS = ("x", "y", "z", "age", "status", "gid", "isin", "wd", "zeta", "bath", "flags")
# diagnostics: Tracker.get_diagnostics names -> oracle state names
DIAG_GPU_TO_ORACLE = {"salt": "p_salt", "temp": "p_temp", "mean_salt": "mean_salt", "mean_temp": "mean_temp",
                      "hob": "p_hob", "bustr": "p_bustr", "bvstr": "p_bvstr"}
DIAG_PARAMS = {"salttemp_on": 1, "salttemp_mean": 1, "write_bottom": 1}
# behave's outputs: Tracker.get_behavior names -> oracle state names
BEHAVE_GPU_TO_ORACLE = {"acc": "p_acc", "vort": "p_vort", "behavew": "p_behavew", "ssf": "p_ssf"}


@dataclasses.dataclass
class Case:
    name: str
    specs: List[synth.GridSpec]
    grids: List[Dict[str, np.ndarray]]
    params: dict
    release: synth.Release
    frames: Dict
    scl: Optional[np.ndarray] = None
    off: Optional[np.ndarray] = None

    @property
    def spec(self) -> synth.GridSpec:
        return self.specs[0]

    @property
    def grid(self) -> Dict[str, np.ndarray]:
        return self.grids[0]

    @property
    def ngrid(self) -> int:
        return len(self.specs)

    def frame(self, k: int, ng: int = 1) -> Dict[str, np.ndarray]:
        key = (ng, k)
        if key not in self.frames:
            self.frames[key] = synth.make_frame(self.specs[ng - 1], self.grids[ng - 1],
                                                (k - 1) * float(self.params["dt"]))
        return self.frames[key]

    def stored(self, k: int, ng: int = 1) -> Dict[str, np.ndarray]:
        sp = self.specs[ng - 1]
        return synth.stored_frame(self.frame(k, ng), sp.field_dtype, sp.stokes)


def make_case(name: str, npart: int, seed: int = 0, spec_over: Optional[dict] = None,
              param_over: Optional[dict] = None, s_range=(-0.98, -0.02)) -> Case:
    """The named workload with `npart` particles; a single grid's release is
    uniform in s over `s_range` ((-1, 0): the whole water column)."""
    specs = synth.config_spec(name)
    if spec_over:
        specs = [dataclasses.replace(sp, **spec_over) for sp in specs]
    grids = [synth.make_grid(sp) for sp in specs]
    params = dict(synth.config_params(name))
    if param_over:
        params.update(param_over)
    c = Case(name, specs, grids, params, None, {})  # type: ignore[arg-type]
    if len(specs) > 1:
        c.scl, c.off = synth.nest_maps(specs)
        c.release = synth.nested_release(specs, grids, c.frame(1, len(specs)), npart, seed=seed)
    else:
        c.release = synth.uniform_release(specs[0], grids[0], c.frame(1), npart, seed=seed, s_range=s_range)
    return c


def noise_array(case: Case, nsteps: int, seed: int = 123) -> np.ndarray:
    """Hook draws [step][particle][draw]: normals, and with Process_VA/_WA
    behave's 2 normals then 5 uniforms in (0, 1) last."""
    ndraw = 2 + int(case.params["idt"]) // int(case.params["deltat"])
    beh = bool(case.params.get("process_va") or case.params.get("process_wa"))
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((nsteps, case.release.z.shape[0], ndraw + (7 if beh else 0)))
    if beh:
        a[..., ndraw + 2:] = (rng.integers(0, 2**32, a[..., ndraw + 2:].shape) + 0.5) / 2.0**32
    return a


def _steps(case: Case, nsteps: int):
    days = (nsteps * case.params["idt"]) / 86400.0 + 1.0
    k = 0
    for ext in schedule.external_steps(days, int(case.params["dt"]), int(case.params["idt"])):
        yield ext, ext.internal
        k += len(ext.internal)
        if k >= nsteps:
            return


def run_gpu(case: Case, nsteps: int, noise: str = "philox", seed: int = 7,
            hook: Optional[np.ndarray] = None, tracker=None, variant: str = "fused",
            field_dtype: Optional[str] = None, resort: int = 0):
    """Run the CUDA path; ``field_dtype="mixed"`` selects the mixed-precision
    form (the frames it is given are the same)."""
    from romspath_b200 import Tracker
    T = tracker or Tracker(case.specs, case.grids, case.params, numpar=case.release.z.shape[0],
                           field_dtype=field_dtype or case.spec.field_dtype, stokes=case.spec.stokes, seed=seed,
                           scl=case.scl, off=case.off, variant=variant, resort=resort)
    for (k, slot) in schedule.initial_loads():
        for ng in range(1, case.ngrid + 1):
            T.upload_frame(ng, slot, case.frame(k, ng))
    T.locate(case.release, t_b=1)
    if noise == "hook":
        T.set_noise_hook(hook)
    done = 0
    for ext, internal in _steps(case, nsteps):
        for (k, slot) in ext.loads:
            for ng in range(1, case.ngrid + 1):
                T.upload_frame(ng, slot, case.frame(k, ng))
        for it in internal:
            if done >= nsteps:
                break
            T.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
            done += 1
    st = T.get_particles()
    if T.diag:
        st.update({DIAG_GPU_TO_ORACLE[k]: v for k, v in T.get_diagnostics().items()})
    if T.va or T.wa:
        st.update({BEHAVE_GPU_TO_ORACLE[k]: v for k, v in T.get_behavior().items()})
    return st, T


def run_oracle(case: Case, nsteps: int, noise: str = "philox", seed: int = 7,
               hook: Optional[np.ndarray] = None, nthreads: int = 8, spline_stats: Optional[list] = None,
               spline_max_iter: int = 100):
    """The oracle's run of the same steps; ``spline_stats`` (a list) gets
    each step's (smoothing-spline fits, secant iterations)."""
    from oracle import oracle as O
    m = O.OracleModel(case.specs, case.grids, case.params, scl=case.scl, off=case.off,
                      spline_max_iter=spline_max_iter)
    for (k, slot) in schedule.initial_loads():
        for ng in range(1, case.ngrid + 1):
            m.set_frame(ng, slot, case.stored(k, ng))
    m.init_particles(case.release, tb=1)
    done = 0
    for ext, internal in _steps(case, nsteps):
        for (k, slot) in ext.loads:
            for ng in range(1, case.ngrid + 1):
                m.set_frame(ng, slot, case.stored(k, ng))
        for it in internal:
            if done >= nsteps:
                break
            if noise == "hook":
                m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise="hook", hook=hook[done],
                       nthreads=nthreads)
            else:
                m.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf, noise="philox", seed=seed,
                       step_index=it.step_index, nthreads=nthreads)
            if spline_stats is not None:
                spline_stats.append(m.stats())
            done += 1
    st = m.state()
    st["gid"] = st["gid"].astype(np.float64)
    st["isin"] = st["isin"].astype(np.int32)
    return st, m


def compare(g: Dict[str, np.ndarray], o: Dict[str, np.ndarray], fields=FIELDS) -> Dict[str, int]:
    """Number of particles whose field differs bit-for-bit, per field."""
    out = {}
    for f in fields:
        a = np.asarray(g[f])
        b = np.asarray(o[f]).astype(a.dtype)
        if a.dtype.kind == "f":
            same = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
        else:
            same = a == b
        out[f] = int((~same).sum())
    return out
