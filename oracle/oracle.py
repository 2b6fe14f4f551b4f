"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The checker for the CUDA path: only tests/, the smoke check and the
CPU-baseline leg of bench.py import this module.  Parity status: unpinned
against the reference binary (see romspath_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
MAXNGRID = 5

FLAG_OOB, FLAG_NODE, FLAG_WBOT, FLAG_WTOP, FLAG_SPLINE = 1, 2, 4, 8, 16
NOISE_MT, NOISE_PHILOX, NOISE_HOOK = 0, 1, 2

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, FP64, no FMA)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "romspath_oracle.c")
        if (not os.path.exists(LIB_PATH)) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
            build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


PD = C.POINTER(C.c_double)
PI32 = C.POINTER(C.c_int32)


# the fuchsparam namelist (ROMSPath.h:165-189)
FUCHS = ("vort_cr", "vort_sat", "b0pv", "b1pv", "b0wv", "b1w", "acc_cr", "acc_sat", "b0pa", "b1pa", "b0wa")
BEHAVE_FIELDS = ("turbaccel", "turbvort", "waveaccelu", "waveaccelv")


class OrcGrid(C.Structure):
    _fields_ = [
        ("xi_rho", C.c_int), ("eta_rho", C.c_int), ("N", C.c_int),
        ("vtransform", C.c_int), ("hc", C.c_double),
        ("h", PD), ("pm", PD), ("pn", PD),
        ("mask_rho", PI32), ("mask_u", PI32), ("mask_v", PI32),
        ("s_rho", PD), ("cs_r", PD), ("s_w", PD), ("cs_w", PD),
        ("scl", (C.c_double * 2) * MAXNGRID), ("off", (C.c_double * 2) * MAXNGRID),
        ("zeta", PD * 3), ("u", PD * 3), ("v", PD * 3), ("w", PD * 3), ("aks", PD * 3),
        ("salt", PD * 3), ("temp", PD * 3), ("bustr", PD * 3), ("bvstr", PD * 3),
        ("lon_rho", PD), ("lat_rho", PD),
        ("wd_rho", PD * 3), ("wd_u", PD * 3), ("wd_v", PD * 3),
        ("turbaccel", PD * 3), ("turbvort", PD * 3), ("waveaccelu", PD * 3), ("waveaccelv", PD * 3),
        ("angle", PD),
    ]


class OrcParams(C.Structure):
    _fields_ = [
        ("ngrid", C.c_int), ("idt", C.c_int), ("scheme", C.c_int), ("nsb", C.c_int),
        ("vturb_on", C.c_int), ("hturb_on", C.c_int), ("open_ocean_boundary", C.c_int),
        ("vertdist", C.c_double), ("serr", C.c_double), ("smth", C.c_double),
        ("sub", C.c_double), ("deltat", C.c_double), ("aksback", C.c_double),
        ("constant_hturb", C.c_double * MAXNGRID),
        ("spline_max_iter", C.c_int),
        ("salttemp_on", C.c_int), ("salttemp_mean", C.c_int), ("write_bottom", C.c_int),
        ("behavior", C.c_int), ("process_va", C.c_int), ("process_wa", C.c_int), ("va_flag", C.c_int),
        ("swimfast", C.c_double), ("initsize", C.c_double),
    ] + [(k, C.c_double) for k in FUCHS] + [("vt_variant", C.c_int), ("vt_dy_end", C.c_double)]


class OrcParticles(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("x", PD), ("y", PD), ("z", PD), ("dob", PD), ("age", PD), ("status", PD),
        ("gid", PI32), ("isin", C.POINTER(C.c_int8)),
        ("wd", PD), ("zeta", PD), ("bath", PD),
        ("flags", C.POINTER(C.c_uint32)), ("pid", C.POINTER(C.c_uint32)),
        ("p_salt", PD), ("p_temp", PD), ("mean_salt", PD), ("mean_temp", PD),
        ("p_hob", PD), ("p_bustr", PD), ("p_bvstr", PD),
        ("p_acc", PD), ("p_vort", PD), ("p_behavew", PD), ("p_ssf", PD),
    ]


class OrcMT(C.Structure):
    _fields_ = [("mt", C.c_uint32 * 624), ("mti", C.c_int)]


class OrcNoise(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("mt", C.POINTER(OrcMT)), ("seed", C.c_uint64),
        ("step", C.c_uint64), ("hook", PD), ("ndraw", C.c_int),
    ]


def _declare(L):
    L.orc_mt_init.argtypes = [C.POINTER(OrcMT), C.c_uint32]
    L.orc_mt_int32.argtypes = [C.POINTER(OrcMT)]
    L.orc_mt_int32.restype = C.c_uint32
    L.orc_mt_real3.argtypes = [C.POINTER(OrcMT)]
    L.orc_mt_real3.restype = C.c_double
    L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.orc_philox_normal.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32]
    L.orc_philox_normal.restype = C.c_double
    L.orc_log_pos.argtypes = [C.c_double]
    L.orc_log_pos.restype = C.c_double
    L.orc_cos2pi.argtypes = [C.c_double]
    L.orc_cos2pi.restype = C.c_double
    L.orc_polintd.argtypes = [PD, PD, C.c_double]
    L.orc_polintd.restype = C.c_double
    L.orc_linint.argtypes = [PD, PD, C.c_int, C.c_double, PD, PD]
    L.orc_getslevel.argtypes = [C.POINTER(OrcGrid), C.c_double, C.c_double, C.c_int]
    L.orc_getslevel.restype = C.c_double
    L.orc_getwlevel.argtypes = [C.POINTER(OrcGrid), C.c_double, C.c_double, C.c_int]
    L.orc_getwlevel.restype = C.c_double
    L.orc_inside.argtypes = [C.c_int, PD, PD, C.c_double, C.c_double]
    L.orc_inside.restype = C.c_int
    L.orc_bounds.argtypes = [C.POINTER(OrcGrid), C.c_double, C.c_double,
                             C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.orc_getinterp2d.argtypes = [C.POINTER(OrcGrid), C.c_int, C.c_double, C.c_double, C.c_int,
                                  C.POINTER(C.c_uint32)]
    L.orc_getinterp2d.restype = C.c_double
    L.orc_getinterp3d.argtypes = [C.POINTER(OrcGrid), C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_uint32)]
    L.orc_getinterp3d.restype = C.c_double
    L.orc_smooth.argtypes = [PD, PD, PD, C.c_int, C.c_double, PD, PD, C.c_int, C.POINTER(C.c_int)]
    L.orc_smooth.restype = C.c_double
    L.orc_ppvalu.argtypes = [PD, PD, C.c_int, C.c_int, C.c_double, C.c_int]
    L.orc_ppvalu.restype = C.c_double
    L.orc_update_particles.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcGrid), C.POINTER(OrcParticles),
                                       PD, PD, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(OrcNoise), C.c_int]
    L.orc_update_particles.restype = C.c_int
    L.orc_init_particles.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcGrid), C.POINTER(OrcParticles),
                                     PD, PD, C.c_int, C.c_int]
    L.orc_init_particles.restype = C.c_int
    L.orc_getinterp_str.argtypes = [C.POINTER(OrcGrid), C.c_int, C.c_double, C.c_double, C.c_int,
                                    C.POINTER(C.c_uint32)]
    L.orc_getinterp_str.restype = C.c_double
    L.orc_last_stats.argtypes = [C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.orc_output_lonlat.argtypes = [C.POINTER(OrcGrid), C.POINTER(OrcParticles), PD, PD]
    L.orc_output_lonlat.restype = None
    L.orc_exp.argtypes = [C.c_double]
    L.orc_exp.restype = C.c_double
    L.orc_log.argtypes = [C.c_double]
    L.orc_log.restype = C.c_double
    L.orc_philox_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32]
    L.orc_philox_uniform.restype = C.c_double
    L.orc_sincos.argtypes = [C.c_double, PD, PD]
    L.orc_sincos.restype = None
    L.orc_asin.argtypes = [C.c_double]
    L.orc_asin.restype = C.c_double
    L.orc_ll2ij.argtypes = [C.POINTER(OrcGrid), C.c_int, PD, PD, C.c_int64, PD, PD]
    L.orc_ll2ij.restype = None
    L.orc_nest_maps.argtypes = [C.c_int, C.POINTER(OrcGrid), PD, PD, PD]
    L.orc_nest_maps.restype = None


def _pd(a: np.ndarray):
    assert a.dtype == np.float64
    return a.ctypes.data_as(PD)


def _f64(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _i32(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.int32))


# ---------------------------------------------------------------- primitives

def polintd(xa, ya, x) -> float:
    xa = np.ascontiguousarray(xa, dtype=np.float64)
    ya = np.ascontiguousarray(ya, dtype=np.float64)
    return lib().orc_polintd(_pd(xa), _pd(ya), float(x))


def linint(xa, ya, x):
    xa = np.ascontiguousarray(xa, dtype=np.float64)
    ya = np.ascontiguousarray(ya, dtype=np.float64)
    y, m = C.c_double(), C.c_double()
    lib().orc_linint(_pd(xa), _pd(ya), len(xa), float(x), C.byref(y), C.byref(m))
    return y.value, m.value


def smooth(x, y, dy, s, max_iter=100):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    dy = np.ascontiguousarray(dy, dtype=np.float64)
    n = len(x)
    v = np.zeros(n * 7)
    a = np.zeros(n * 4)
    it = C.c_int()
    sfq = lib().orc_smooth(_pd(x), _pd(y), _pd(dy), n, float(s), _pd(v), _pd(a), max_iter, C.byref(it))
    return sfq, a.reshape(4, n).T.copy(), it.value


def ppvalu(brk, coef_k_by_l, x, jderiv):
    brk = np.ascontiguousarray(brk, dtype=np.float64)
    coef = np.asfortranarray(coef_k_by_l, dtype=np.float64)
    k, l = coef.shape
    return lib().orc_ppvalu(_pd(brk), _pd(coef.ravel(order="F")), l, k, float(x), jderiv)


def sincos(x):
    s, c = C.c_double(), C.c_double()
    lib().orc_sincos(float(x), C.byref(s), C.byref(c))
    return s.value, c.value


def inside(xb, yb, xo, yo) -> bool:
    nb = len(xb)
    xbb = np.zeros(nb + 1)
    ybb = np.zeros(nb + 1)
    xbb[:nb] = xb
    ybb[:nb] = yb
    return bool(lib().orc_inside(nb, _pd(xbb), _pd(ybb), float(xo), float(yo)))


class MT19937:
    def __init__(self, seed: int):
        self.s = OrcMT()
        lib().orc_mt_init(C.byref(self.s), seed & 0xFFFFFFFF)

    def int32(self) -> int:
        return lib().orc_mt_int32(C.byref(self.s))

    def real3(self) -> float:
        return lib().orc_mt_real3(C.byref(self.s))


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def log_pos(x) -> float:
    return lib().orc_log_pos(float(x))


def cos2pi(u) -> float:
    return lib().orc_cos2pi(float(u))


def philox_normal(seed, pid, step, draw) -> float:
    return lib().orc_philox_normal(seed, pid, step, draw)


# ---------------------------------------------------------------- the model

class OracleModel:
    """Grids + 3-slot frame ring + particle state, stepped by the oracle.

    ``grids`` is a list of dicts from ``synth.make_grid`` (Fortran order);
    ``specs`` the matching ``synth.GridSpec`` list; ``params`` the namelist
    dict of ``synth.config_params``; ``scl``/``off`` per-grid arrays of shape
    (ngrid, 2) (defaults: identity maps, single grid).
    """

    def __init__(self, specs, grids, params: dict, scl=None, off=None, spline_max_iter=100):
        L = lib()
        self.ng = len(grids)
        self.specs = specs
        self._keep: List[np.ndarray] = []
        self.g = (OrcGrid * self.ng)()
        for k, (sp, gr) in enumerate(zip(specs, grids)):
            G = self.g[k]
            G.xi_rho, G.eta_rho, G.N = sp.xi_rho, sp.eta_rho, sp.N
            G.vtransform, G.hc = sp.vtransform, sp.hc
            for name in ("h", "pm", "pn", "s_rho", "cs_r", "s_w", "cs_w"):
                a = _f64(gr[name])
                self._keep.append(a)
                setattr(G, name, _pd(a))
            for name in ("mask_rho", "mask_u", "mask_v"):
                a = _i32(gr[name])
                self._keep.append(a)
                setattr(G, name, a.ctypes.data_as(PI32))
            for name in ("lon_rho", "lat_rho", "angle"):
                if name in gr:
                    a = _f64(gr[name])
                    self._keep.append(a)
                    setattr(G, name, _pd(a))
            for i in range(self.ng):
                s = scl[k][i] if scl is not None else (1.0, 1.0)
                o = off[k][i] if off is not None else (0.0, 0.0)
                G.scl[i][0], G.scl[i][1] = s
                G.off[i][0], G.off[i][1] = o
        self.frames: Dict = {}
        p = OrcParams()
        p.ngrid = self.ng
        p.idt = int(params["idt"])
        p.scheme = int(params["scheme"])
        p.nsb = int(params["nsb"])
        p.vturb_on = int(params["vturb_on"])
        p.hturb_on = int(params["hturb_on"])
        p.open_ocean_boundary = int(params["open_ocean_boundary"])
        for name in ("vertdist", "serr", "smth", "sub", "deltat", "aksback"):
            setattr(p, name, float(params[name]))
        for i, v in enumerate(params["constant_hturb"][:MAXNGRID]):
            p.constant_hturb[i] = float(v)
        p.spline_max_iter = spline_max_iter
        # diagnostics (ROMSPath.f90:935-986): SaltTempOn, SaltTempMean, WriteBottom
        p.salttemp_on = int(params.get("salttemp_on", 0))
        p.salttemp_mean = int(params.get("salttemp_mean", 0))
        p.write_bottom = int(params.get("write_bottom", 0))
        self.params = p
        # behave (behavior_module.f90:186-393)
        p.behavior = int(params.get("behavior", 0))
        p.process_va = int(params.get("process_va", 0))
        p.process_wa = int(params.get("process_wa", 0))
        p.va_flag = int(params.get("va_flag", 0))
        p.swimfast = float(params.get("swimfast", 0.0))
        p.initsize = float(params.get("initsize", 0.0))
        for k in FUCHS:
            setattr(p, k, float(params.get(k, 0.0)))
        # VTurb experiment variants (well-mixed-condition attribution);
        # defaults are the reference's algorithm
        p.vt_variant = int(params.get("vt_variant", 0))
        p.vt_dy_end = float(params.get("vt_dy_end", float("nan")))
        # -DWETDRY: the frames' wet/dry masks replace the static ones in
        # getInterp3D and getInterpStr
        self.wetdry = bool(params.get("wetdry", 0))
        # draws per particle-step in a noise hook: HTurb 2, VTurb idt/deltat,
        # then behave's 2 normals and 5 uniforms when Process_VA or _WA
        self.ndraw = 2 + int(params["idt"]) // int(params["deltat"]) + (7 if (p.process_va or p.process_wa) else 0)
        self.P: Optional[OrcParticles] = None

    def set_frame(self, ng: int, slot: int, frame: Dict[str, np.ndarray]):
        """Frame values exactly as stored (FP64 arrays, Stokes already added)."""
        G = self.g[ng - 1]
        for name in ("zeta", "u", "v", "w", "aks", "salt", "temp", "bustr", "bvstr") + BEHAVE_FIELDS:
            if name not in frame:
                continue
            a = _f64(frame[name])
            self.frames[(ng, slot, name)] = a
            getattr(G, name)[slot - 1] = _pd(a)
        if self.wetdry:
            for name, field in (("wetdry_rho", "wd_rho"), ("wetdry_u", "wd_u"), ("wetdry_v", "wd_v")):
                a = _f64(frame[name])
                self.frames[(ng, slot, name)] = a
                getattr(G, field)[slot - 1] = _pd(a)

    def set_particles(self, x, y, z, dob, age, status, gid, isin, pid=None):
        n = len(x)
        self.st = {
            "x": _f64(x).copy(), "y": _f64(y).copy(), "z": _f64(z).copy(),
            "dob": _f64(dob).copy(), "age": _f64(age).copy(), "status": _f64(status).copy(),
            "gid": np.asarray(gid, dtype=np.int32).copy(), "isin": np.asarray(isin, dtype=np.int8).copy(),
            "wd": np.full(n, 9999.0), "zeta": np.full(n, 9999.0), "bath": np.full(n, 9999.0),
            "flags": np.zeros(n, dtype=np.uint32),
            "pid": (np.arange(n, dtype=np.uint32) if pid is None else np.asarray(pid, dtype=np.uint32).copy()),
        }
        # diagnostics as the particle read loop leaves them (ROMSPath.f90:247-264, 353-355)
        for k in ("p_salt", "p_temp", "mean_salt", "mean_temp", "p_bustr", "p_bvstr",
                  "p_acc", "p_vort", "p_behavew", "p_ssf"):          # 343-346
            self.st[k] = np.zeros(n)
        self.st["p_hob"] = np.full(n, 9999.0)
        self._bind()

    def _bind(self):
        s = self.st
        P = OrcParticles()
        P.n = len(s["x"])
        for k in ("x", "y", "z", "dob", "age", "status", "wd", "zeta", "bath"):
            setattr(P, k, _pd(s[k]))
        P.gid = s["gid"].ctypes.data_as(PI32)
        P.isin = s["isin"].ctypes.data_as(C.POINTER(C.c_int8))
        P.flags = s["flags"].ctypes.data_as(C.POINTER(C.c_uint32))
        P.pid = s["pid"].ctypes.data_as(C.POINTER(C.c_uint32))
        for k in ("p_salt", "p_temp", "mean_salt", "mean_temp", "p_hob", "p_bustr", "p_bvstr",
                  "p_acc", "p_vort", "p_behavew", "p_ssf"):
            setattr(P, k, _pd(s[k]))
        self.P = P

    def init_particles(self, release, tb: int = 1, pid=None, tc: Optional[int] = None):
        """ini_ROMSPath ownership + zbounds (ROMSPath.f90:367-432); initial
        diagnostics at slot tc (default: the slot after tb)."""
        n = release.z.shape[0]
        self.set_particles(np.ones(n), np.ones(n), release.z, release.dob, np.zeros(n),
                           np.full(n, 9.0), np.full(n, self.ng, dtype=np.int32), np.zeros(n, dtype=np.int8),
                           pid=pid)
        ip = np.ascontiguousarray(release.ipos, dtype=np.float64)
        jp = np.ascontiguousarray(release.jpos, dtype=np.float64)
        tc = (tb % 3) + 1 if tc is None else tc
        lib().orc_init_particles(C.byref(self.params), self.g, C.byref(self.P), _pd(ip), _pd(jp), tb, tc)

    def step(self, ex, ix, ets, tb, tc, tf, noise="philox", seed=0, step_index=0,
             hook: Optional[np.ndarray] = None, mt: Optional[MT19937] = None, nthreads=1):
        exa = np.array(ex, dtype=np.float64)
        ixa = np.array(ix, dtype=np.float64)
        nz = OrcNoise()
        if noise == "mt":
            nz.kind = NOISE_MT
            nz.mt = C.pointer(mt.s)
        elif noise == "hook":
            nz.kind = NOISE_HOOK
            hk = np.ascontiguousarray(hook, dtype=np.float64)
            nz.hook = _pd(hk)
            nz.ndraw = hk.shape[-1]
        else:
            nz.kind = NOISE_PHILOX
            nz.seed = seed
            nz.step = step_index
        rc = lib().orc_update_particles(C.byref(self.params), self.g, C.byref(self.P), _pd(exa), _pd(ixa),
                                        ets, tb, tc, tf, C.byref(nz), nthreads)
        if rc != 0:
            raise RuntimeError("oracle step failed")

    def stats(self):
        a, b = C.c_int64(), C.c_int64()
        lib().orc_last_stats(C.byref(a), C.byref(b))
        return a.value, b.value

    def ll2ij(self, ng: int, lon, lat, spherical: int):
        """LL2ij of grid ng (interpolation_module.f90:110-231)."""
        lon = np.ascontiguousarray(lon, dtype=np.float64)
        lat = np.ascontiguousarray(lat, dtype=np.float64)
        ip, jp = np.empty(len(lon)), np.empty(len(lon))
        lib().orc_ll2ij(C.byref(self.g[ng - 1]), int(spherical), _pd(lon), _pd(lat), len(lon), _pd(ip), _pd(jp))
        return ip, jp

    def locate_lonlat(self, lon, lat, z, dob, spherical: int, tb: int = 1, pid=None):
        """ini_ROMSPath from particle lon/lat: LL2ij for every grid, then the
        ownership loop (ROMSPath.f90:359-432)."""
        n = len(lon)
        ip = np.empty((self.ng, n))
        jp = np.empty((self.ng, n))
        for ng in range(1, self.ng + 1):
            ip[ng - 1], jp[ng - 1] = self.ll2ij(ng, lon, lat, spherical)

        class _R:
            pass
        r = _R()
        r.ipos, r.jpos, r.z, r.dob = ip, jp, np.asarray(z, dtype=np.float64), np.asarray(dob, dtype=np.float64)
        self.init_particles(r, tb=tb, pid=pid)
        return ip, jp

    def nest_maps(self, refine):
        """scl, off of every grid (InitGrid's search, grid_module.f90:441-481):
        arrays [ng][Ngrid][2] as GRIDS(ng)%scl(i, c)."""
        ref = np.ascontiguousarray(list(refine) + [1.0] * MAXNGRID, dtype=np.float64)
        scl = np.empty(self.ng * 2 * self.ng)
        off = np.empty(self.ng * 2 * self.ng)
        lib().orc_nest_maps(self.ng, self.g, _pd(ref), _pd(scl), _pd(off))
        return (scl.reshape(self.ng, 2, self.ng).transpose(0, 2, 1).copy(),
                off.reshape(self.ng, 2, self.ng).transpose(0, 2, 1).copy())

    def output_record(self, mI: int) -> Dict[str, np.ndarray]:
        """One output record of dataOutput / writeNetCDF (ROMSPath.f90:1012-1024,
        1924-2070): lon, lat, zp, age, status, gid and the diagnostics that are
        on (salt/temp as sum / mI under SaltTempMean), then the writer's resets
        (sums to 0, P_HOB to 9999)."""
        s = self.st
        n = len(s["x"])
        lon, lat = np.empty(n), np.empty(n)
        lib().orc_output_lonlat(self.g, C.byref(self.P), _pd(lon), _pd(lat))
        rec = {"lon": lon, "lat": lat, "zp": s["z"].copy(), "age": s["age"].copy(),
               "status": s["status"].copy(), "gid": s["gid"].astype(np.float64)}
        p = self.params
        if p.salttemp_on:
            if p.salttemp_mean:
                rec["salt"] = s["mean_salt"] / float(mI)
                rec["temp"] = s["mean_temp"] / float(mI)
                s["mean_salt"][:] = 0.0
                s["mean_temp"][:] = 0.0
            else:
                rec["salt"] = s["p_salt"].copy()
                rec["temp"] = s["p_temp"].copy()
        if p.write_bottom:
            rec["hob"] = s["p_hob"].copy()
            rec["bustr"] = s["p_bustr"].copy()
            rec["bvstr"] = s["p_bvstr"].copy()
            s["p_hob"][:] = 9999.0
        return rec

    def state(self) -> Dict[str, np.ndarray]:
        return {k: v.copy() for k, v in self.st.items()}
