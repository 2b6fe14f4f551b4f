"""Host mirror of the reference's particle-step interface.

``Tracker`` is the Python face of the C ABI: it owns one device context
(grids, frame ring, particle state) and exposes the calls the kept Fortran
driver makes -- ``updateHydro`` hand-off (``upload_frame``), the initial
ownership loop (``locate``), ``update_particles`` (``step``) and the state
read-back used by ``dataOutput`` (``get_particles``).  ``run`` replays the
driver's external/internal time loop (ROMSPath.f90:151-178, 465-546).
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from . import schedule as _sched


class RomsPathError(RuntimeError):
    pass


def _pd(a):
    return a.ctypes.data_as(_lib.PD) if a is not None else None


def _pf(a):
    return a.ctypes.data_as(_lib.PF) if a is not None else None


class Tracker:
    def __init__(self, specs, grids: Sequence[Dict[str, np.ndarray]], params: dict, numpar: int,
                 field_dtype: str = "f64", stokes: bool = False, seed: int = 0, device: int = 0,
                 scl: Optional[np.ndarray] = None, off: Optional[np.ndarray] = None,
                 spline_max_iter: int = 100, variant: str = "fused", resort: int = 0, blocks_per_sm: int = 0):
        L = _lib.load()
        self.L = L
        self.ng = len(grids)
        self.field_dtype = field_dtype
        self._keep: List[np.ndarray] = []
        self._lonlat = []
        P = _lib.RpParams()
        P.numpar = int(numpar)
        P.idt = int(params["idt"])
        P.dt = int(params["dt"])
        P.scheme = int(params["scheme"])
        P.nsb = int(params["nsb"])
        P.vturb_on = int(params["vturb_on"])
        P.hturb_on = int(params["hturb_on"])
        P.open_ocean_boundary = int(params["open_ocean_boundary"])
        # behave: Behavior (0, 1, 10, 11), Process_VA / Process_WA
        P.behavior = int(params.get("behavior", 0))
        self.va = bool(params.get("process_va", 0))
        self.wa = bool(params.get("process_wa", 0))
        P.stokes = int(bool(stokes))
        # "f64" / "f32": fields stored at that width, FP64 arithmetic (exact);
        # "mixed": FP16 fields with per-level scales, FP32 positions with
        # compensated accumulation, FP64 age and spline fit (not exact);
        # "mixed-i16": the same with int16 fixed-point fields
        P.field_dtype = {"f64": _lib.FIELD_F64, "f32": _lib.FIELD_F32, "mixed": _lib.FIELD_MIXED,
                         "mixed-i16": _lib.FIELD_MIXED_I16}[field_dtype]
        P.spline_max_iter = int(spline_max_iter)
        for k in ("vertdist", "serr", "smth", "sub", "deltat", "aksback"):
            setattr(P, k, float(params[k]))
        for i, v in enumerate(list(params["constant_hturb"])[:_lib.MAXNGRID]):
            P.constant_hturb[i] = float(v)
        P.seed = int(seed)
        P.device = int(device)
        # kernel form: "fused" (one kernel, spline workspace in local
        # memory), "split" (a VTurb kernel writing each particle's
        # displacement to a scratch array, then the advection kernel) or,
        # in the mixed form, "smem" (the split form with the VTurb kernel's
        # spline workspace in shared memory)
        P.reserved[0] = self.FORMS[variant]
        # re-sort the particle state by grid and cell every `resort` internal
        # steps (0: never); results are unchanged
        P.reserved[1] = int(resort)
        # cap on resident blocks per SM of the step kernels (0: occupancy
        # limit); fewer blocks mean more particles per thread
        P.reserved[2] = int(blocks_per_sm)
        # diagnostics (namelist "other"): SaltTempOn, SaltTempMean, WriteBottom
        self.diag = ((_lib.DIAG_SALTTEMP if params.get("salttemp_on") else 0) |
                     (_lib.DIAG_SALTTEMP_MEAN if params.get("salttemp_mean") else 0) |
                     (_lib.DIAG_BOTTOM if params.get("write_bottom") else 0))
        P.reserved[3] = self.diag
        # WETDRY: per-frame wet/dry masks (frames then carry wetdry_rho/_u/_v)
        self.wetdry = bool(params.get("wetdry", 0))
        P.reserved[4] = int(self.wetdry)
        G = (_lib.RpGrid * self.ng)()
        for k, (sp, gr) in enumerate(zip(specs, grids)):
            g = G[k]
            g.xi_rho, g.eta_rho, g.n_rho = sp.xi_rho, sp.eta_rho, sp.N
            g.vtransform, g.hc = sp.vtransform, sp.hc
            for name in ("h", "pm", "pn", "s_rho", "cs_r", "s_w", "cs_w"):
                a = np.asfortranarray(gr[name], dtype=np.float64)
                self._keep.append(a)
                setattr(g, name, _pd(a))
            for name in ("mask_rho", "mask_u", "mask_v"):
                a = np.asfortranarray(gr[name], dtype=np.int32)
                self._keep.append(a)
                setattr(g, name, a.ctypes.data_as(_lib.PI32))
            if "lon_rho" in gr:
                self._lonlat.append((k + 1, np.asfortranarray(gr["lon_rho"], dtype=np.float64),
                                     np.asfortranarray(gr["lat_rho"], dtype=np.float64),
                                     np.asfortranarray(gr["angle"], dtype=np.float64) if "angle" in gr else None))
            if scl is not None:
                s = np.asfortranarray(np.asarray(scl[k], dtype=np.float64).reshape(self.ng, 2))
                o = np.asfortranarray(np.asarray(off[k], dtype=np.float64).reshape(self.ng, 2))
                self._keep += [s, o]
                g.scl, g.off = _pd(s), _pd(o)
        self.params = P
        self.ndraw = 2 + P.idt // int(P.deltat)
        h = C.c_void_p()
        rc = L.rp_create(C.byref(P), self.ng, G, C.byref(h))
        if rc != 0:
            raise RomsPathError(f"rp_create failed: {_lib.ERRORS.get(rc, rc)}")
        self.h = h
        self.n = 0
        # GRIDS(ng)%spherical: 1 for lon/lat grids (the default), 0 Cartesian
        sph = int(params.get("spherical", 1))
        for ng, lon, lat, ang in self._lonlat:
            self._check(L.rp_set_grid_lonlat(h, ng, _pd(lon), _pd(lat)), "rp_set_grid_lonlat")
            self._check(L.rp_set_grid_angle(h, ng, _pd(ang), sph), "rp_set_grid_angle")
        self._lonlat = []
        if P.behavior or self.va or self.wa:
            b = _lib.RpBehavior()
            b.behavior = P.behavior
            b.process_va, b.process_wa = int(self.va), int(self.wa)
            b.va_flag = int(params.get("va_flag", 0))
            b.swimfast = float(params.get("swimfast", 0.0))
            b.initsize = float(params.get("initsize", 0.0))
            for k in _lib.FUCHS:
                setattr(b, k, float(params.get(k, 0.0)))
            self._check(L.rp_set_behavior(h, C.byref(b)), "rp_set_behavior")
            self.ndraw += 7 if (self.va or self.wa) else 0

    # ------------------------------------------------------------ basics
    def _check(self, rc: int, what: str):
        if rc != 0:
            buf = C.create_string_buffer(512)
            self.L.rp_last_error(self.h, buf, 512)
            raise RomsPathError(f"{what}: {_lib.ERRORS.get(rc, rc)}: {buf.value.decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.L.rp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ frames
    def upload_frame(self, ng: int, slot: int, frame: Dict[str, np.ndarray]):
        """updateHydro(FIRST, tstep, tind=slot) output of grid ng."""
        f32 = frame["u"].dtype == np.float32
        conv = (lambda a: np.asfortranarray(a, dtype=np.float32)) if f32 else \
            (lambda a: np.asfortranarray(a, dtype=np.float64))
        arrs = [conv(frame[k]) for k in ("zeta", "u", "v", "w", "aks")]
        su = conv(frame["su"]) if "su" in frame else None
        sv = conv(frame["sv"]) if "sv" in frame else None
        if not self.params.stokes:
            su = sv = None
        p = _pf if f32 else _pd
        if self.wetdry or self.va or self.wa:
            # every field through the frame descriptor
            d = _lib.RpFrame()
            d.f32 = int(f32)
            keep = []
            for k, a in zip(("zeta", "u", "v", "w", "aks"), arrs):
                setattr(d, k, a.ctypes.data)
            for k, a in (("su", su), ("sv", sv)):
                if a is not None:
                    setattr(d, k, a.ctypes.data)
            st = self.diag & _lib.DIAG_SALTTEMP
            bt = self.diag & _lib.DIAG_BOTTOM
            for k, on in (("salt", st), ("temp", st), ("bustr", bt), ("bvstr", bt)):
                if on and k in frame:
                    a = conv(frame[k])
                    keep.append(a)
                    setattr(d, k, a.ctypes.data)
            for k in ("wetdry_rho", "wetdry_u", "wetdry_v") if self.wetdry else ():
                a = np.asfortranarray(frame[k], dtype=np.float64)
                keep.append(a)
                setattr(d, k, _pd(a))
            for k, on in (("turbaccel", self.va), ("turbvort", self.va), ("waveaccelu", self.wa),
                          ("waveaccelv", self.wa)):
                if on and k in frame:
                    a = conv(frame[k])
                    keep.append(a)
                    setattr(d, k, a.ctypes.data)
            rc = self.L.rp_upload_frame_desc(self.h, ng, slot, C.byref(d))
        elif self.diag:
            # salt/temp and bustr/bvstr of the diagnostics that are on
            st = self.diag & _lib.DIAG_SALTTEMP
            bt = self.diag & _lib.DIAG_BOTTOM
            extra = [conv(frame[k]) if on else None
                     for k, on in (("salt", st), ("temp", st), ("bustr", bt), ("bvstr", bt))]
            fn = self.L.rp_upload_frame_ext_f32 if f32 else self.L.rp_upload_frame_ext
            rc = fn(self.h, ng, slot, *[p(a) for a in arrs], p(su), p(sv), *[p(a) for a in extra])
        else:
            fn = self.L.rp_upload_frame_f32 if f32 else self.L.rp_upload_frame
            rc = fn(self.h, ng, slot, *[p(a) for a in arrs], p(su), p(sv))
        self._check(rc, "rp_upload_frame")

    # --------------------------------------------------------- particles
    def set_particles(self, x, y, z, dob, age, status, gid, isin):
        cols = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, dob, age, status, gid)]
        isin = np.ascontiguousarray(isin, dtype=np.int32)
        rc = self.L.rp_set_particles(self.h, len(cols[0]), *[_pd(a) for a in cols], isin.ctypes.data_as(_lib.PI32))
        self._check(rc, "rp_set_particles")
        self.n = len(cols[0])

    def locate(self, release, t_b: int = 1):
        """ini_ROMSPath ownership loop (ROMSPath.f90:367-432) on the device."""
        n = release.z.shape[0]
        ip = np.ascontiguousarray(release.ipos, dtype=np.float64)
        jp = np.ascontiguousarray(release.jpos, dtype=np.float64)
        z = np.ascontiguousarray(release.z, dtype=np.float64)
        dob = np.ascontiguousarray(release.dob, dtype=np.float64)
        rc = self.L.rp_locate_particles(self.h, n, _pd(ip), _pd(jp), _pd(z), _pd(dob), t_b)
        self._check(rc, "rp_locate_particles")
        self.n = n

    def locate_lonlat(self, lon, lat, z, dob, t_b: int = 1):
        """ini_ROMSPath from particle lon/lat: LL2ij of every grid on the
        device, then the ownership loop; returns LL2ij's (ipos, jpos),
        (Ngrid, n)."""
        n = len(lon)
        cols = [np.ascontiguousarray(a, dtype=np.float64) for a in (lon, lat, z, dob)]
        ip = np.empty((self.ng, n))
        jp = np.empty((self.ng, n))
        rc = self.L.rp_locate_lonlat(self.h, n, *[_pd(a) for a in cols], t_b, _pd(ip), _pd(jp))
        self._check(rc, "rp_locate_lonlat")
        self.n = n
        return ip, jp

    def get_particles(self, n: Optional[int] = None, out: Optional[Dict[str, np.ndarray]] = None
                      ) -> Dict[str, np.ndarray]:
        """par columns, isIn, pWD/pZeta/pBath and flags; ``out`` may hold
        preallocated (e.g. page-locked) arrays to fill."""
        n = self.n if n is None else n
        if out is None:
            out = {k: np.empty(n) for k in ("x", "y", "z", "age", "status", "gid", "wd", "zeta", "bath")}
            out["isin"] = np.empty(n, dtype=np.int32)
            out["flags"] = np.empty(n, dtype=np.uint32)
        isin = out["isin"]
        flags = out["flags"]
        rc = self.L.rp_get_particles(self.h, n, _pd(out["x"]), _pd(out["y"]), _pd(out["z"]), _pd(out["age"]),
                                     _pd(out["status"]), _pd(out["gid"]), isin.ctypes.data_as(_lib.PI32),
                                     _pd(out["wd"]), _pd(out["zeta"]), _pd(out["bath"]),
                                     flags.ctypes.data_as(_lib.PU32))
        self._check(rc, "rp_get_particles")
        return out

    def get_diagnostics(self, n: Optional[int] = None) -> Dict[str, np.ndarray]:
        """P_Salt, P_Temp, mean_salt, mean_temp (running sums), P_HOB,
        P_bustr, P_bvstr of the diagnostics that are on."""
        n = self.n if n is None else n
        names = []
        if self.diag & _lib.DIAG_SALTTEMP:
            names += ["salt", "temp"]
        if self.diag & _lib.DIAG_SALTTEMP_MEAN:
            names += ["mean_salt", "mean_temp"]
        if self.diag & _lib.DIAG_BOTTOM:
            names += ["hob", "bustr", "bvstr"]
        out = {k: np.empty(n) for k in names}
        order = ("salt", "temp", "mean_salt", "mean_temp", "hob", "bustr", "bvstr")
        rc = self.L.rp_get_diagnostics(self.h, n, *[_pd(out.get(k)) for k in order])
        self._check(rc, "rp_get_diagnostics")
        return out

    def get_behavior(self, n: Optional[int] = None) -> Dict[str, np.ndarray]:
        """par(:,pAcc/pVort/pbehaveW/pSSF) of behave."""
        n = self.n if n is None else n
        out = {k: np.empty(n) for k in ("acc", "vort", "behavew", "ssf")}
        rc = self.L.rp_get_behavior(self.h, n, *[_pd(out[k]) for k in ("acc", "vort", "behavew", "ssf")])
        self._check(rc, "rp_get_behavior")
        return out

    RECORD = ("lon", "lat", "zp", "age", "status", "gid", "salt", "temp", "hob", "bustr", "bvstr")

    def output_record(self, mI: int, n: Optional[int] = None, out: Optional[Dict[str, np.ndarray]] = None
                      ) -> Dict[str, np.ndarray]:
        """One output record (dataOutput + writeNetCDF's columns and resets);
        ``out`` may hold preallocated (e.g. page-locked) arrays."""
        n = self.n if n is None else n
        if out is None:
            names = ["lon", "lat", "zp", "age", "status", "gid"]
            if self.diag & _lib.DIAG_SALTTEMP:
                names += ["salt", "temp"]
            if self.diag & _lib.DIAG_BOTTOM:
                names += ["hob", "bustr", "bvstr"]
            out = {k: np.empty(n) for k in names}
        rc = self.L.rp_output_record(self.h, n, int(mI), *[_pd(out.get(k)) for k in self.RECORD])
        self._check(rc, "rp_output_record")
        return out

    def output_record_async(self, mI: int, out: Dict[str, np.ndarray], n: Optional[int] = None):
        """rp_output_record_async into page-locked arrays ``out`` (names as
        output_record); read them after output_wait()."""
        n = self.n if n is None else n
        rc = self.L.rp_output_record_async(self.h, n, int(mI), *[_pd(out.get(k)) for k in self.RECORD])
        self._check(rc, "rp_output_record_async")

    def output_wait(self):
        self._check(self.L.rp_output_wait(self.h), "rp_output_wait")

    def reset_diagnostics(self):
        """The writer's resets after an output record (sums to 0, HOB to 9999)."""
        self._check(self.L.rp_reset_diagnostics(self.h), "rp_reset_diagnostics")

    # --------------------------------------------------------------- step
    def step(self, ex, ix, ets: int, tb: int, tc: int, tf: int):
        exa = (C.c_double * 3)(*ex)
        ixa = (C.c_double * 3)(*ix)
        rc = self.L.rp_step(self.h, exa, ixa, ets, tb, tc, tf)
        self._check(rc, "rp_step")

    def step_n(self, steps):
        """Several internal steps (objects with ex, ix, ets, tb, tc, tf) in
        one call, launched as one CUDA graph."""
        k = len(steps)
        ex = np.ascontiguousarray([s.ex for s in steps], dtype=np.float64)
        ix = np.ascontiguousarray([s.ix for s in steps], dtype=np.float64)
        i32 = lambda v: np.ascontiguousarray(v, dtype=np.int32)
        ets, tb, tc, tf = (i32([s.ets for s in steps]), i32([s.tb for s in steps]), i32([s.tc for s in steps]),
                           i32([s.tf for s in steps]))
        rc = self.L.rp_step_n(self.h, k, _pd(ex), _pd(ix), *[a.ctypes.data_as(_lib.PI32) for a in (ets, tb, tc, tf)])
        self._check(rc, "rp_step_n")

    FORMS = {"fused": 0, "split": 1, "smem": 2, "fused-noprefetch": 3, "fused-b64": 4, "fused-b256": 5}

    def set_kernel_form(self, form: str):
        """Kernel form between steps (rp_set_kernel_form): "fused", "split",
        and in the mixed forms "smem", "fused-noprefetch", "fused-b64" and
        "fused-b256" (64- and 256-thread blocks)."""
        self._check(self.L.rp_set_kernel_form(self.h, self.FORMS[form]), "rp_set_kernel_form")

    def set_launch(self, resort: int, blocks_per_sm: int):
        """Re-sort interval (0: never) and resident blocks per SM (0: the
        occupancy limit) from the next step on; results are unchanged."""
        self._check(self.L.rp_set_launch(self.h, int(resort), int(blocks_per_sm)), "rp_set_launch")

    def set_id_base(self, base: int):
        """Particle k of the next locate/set_particles gets id base + k."""
        self._check(self.L.rp_set_id_base(self.h, int(base)), "rp_set_id_base")

    def set_step_index(self, k: int):
        self._check(self.L.rp_set_step_index(self.h, int(k)), "rp_set_step_index")

    def set_noise_hook(self, noise: Optional[np.ndarray]):
        """noise[step, particle, draw] of N(0,1) values, or None."""
        if noise is None:
            self._check(self.L.rp_set_noise_hook(self.h, None, 0), "rp_set_noise_hook")
            return
        a = np.ascontiguousarray(noise, dtype=np.float64)
        self._check(self.L.rp_set_noise_hook(self.h, _pd(a), a.shape[0]), "rp_set_noise_hook")

    def synchronize(self):
        self._check(self.L.rp_synchronize(self.h), "rp_synchronize")

    def last_step_stats(self):
        ms = C.c_float()
        k = C.c_int32()
        self._check(self.L.rp_last_step_stats(self.h, C.byref(ms), C.byref(k)), "rp_last_step_stats")
        return ms.value, k.value

    def kernel_launches(self) -> int:
        c = C.c_int64()
        self._check(self.L.rp_kernel_launches(self.h, C.byref(c)), "rp_kernel_launches")
        return c.value

    def count_spline_passes(self, on: bool = True):
        """Start (counts zeroed) or stop counting VTurb's smoothing-spline
        fits and their chol1d passes in the steps launched afterwards."""
        self._check(self.L.rp_count_spline_passes(self.h, 1 if on else 0), "rp_count_spline_passes")

    def spline_pass_counts(self):
        """(fits, chol1d passes) since counting was last started."""
        f = C.c_int64()
        p = C.c_int64()
        self._check(self.L.rp_spline_pass_counts(self.h, C.byref(f), C.byref(p)), "rp_spline_pass_counts")
        return f.value, p.value

    def device_state(self) -> _lib.RpDeviceState:
        st = _lib.RpDeviceState()
        self._check(self.L.rp_device_state_get(self.h, C.byref(st)), "rp_device_state_get")
        return st

    # ------------------------------------------------------------ driver
    def run(self, days: float, frame_for: Callable[[int, int], Dict[str, np.ndarray]],
            on_step: Optional[Callable] = None, max_steps: Optional[int] = None, load_initial: bool = True):
        """Replay run_ROMSPath's time loop: frames from frame_for(ng, k)."""
        P = self.params
        if load_initial:
            for (k, slot) in _sched.initial_loads():
                for ng in range(1, self.ng + 1):
                    self.upload_frame(ng, slot, frame_for(ng, k))
        done = 0
        for ext in _sched.external_steps(days, P.dt, P.idt):
            for (k, slot) in ext.loads:
                for ng in range(1, self.ng + 1):
                    self.upload_frame(ng, slot, frame_for(ng, k))
            for it in ext.internal:
                self.step(it.ex, it.ix, it.ets, it.tb, it.tc, it.tf)
                if on_step:
                    on_step(it)
                done += 1
                if max_steps is not None and done >= max_steps:
                    return done
        return done


def nest_maps(grids: Sequence[Dict[str, np.ndarray]], refine: Sequence[float]):
    """InitGrid's nest maps (rp_nest_maps) from the grids' lon_rho/lat_rho:
    (scl, off), each (Ngrid, Ngrid, 2) as GRIDS(ng)%scl(i, c)."""
    L = _lib.load()
    ng = len(grids)
    xi = np.array([g["lon_rho"].shape[0] for g in grids], dtype=np.int32)
    eta = np.array([g["lon_rho"].shape[1] for g in grids], dtype=np.int32)
    lons = [np.asfortranarray(g["lon_rho"], dtype=np.float64) for g in grids]
    lats = [np.asfortranarray(g["lat_rho"], dtype=np.float64) for g in grids]
    lp = (_lib.PD * ng)(*[_pd(a) for a in lons])
    tp = (_lib.PD * ng)(*[_pd(a) for a in lats])
    ref = np.ascontiguousarray(list(refine) + [1.0] * _lib.MAXNGRID, dtype=np.float64)
    scl = np.empty(ng * 2 * ng)
    off = np.empty(ng * 2 * ng)
    rc = L.rp_nest_maps(ng, xi.ctypes.data_as(_lib.PI32), eta.ctypes.data_as(_lib.PI32), lp, tp, _pd(ref),
                        _pd(scl), _pd(off))
    if rc != 0:
        raise RomsPathError(f"rp_nest_maps: {_lib.ERRORS.get(rc, rc)}")
    return (scl.reshape(ng, 2, ng).transpose(0, 2, 1).copy(), off.reshape(ng, 2, ng).transpose(0, 2, 1).copy())
