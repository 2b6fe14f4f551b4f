"""The adjoint pair (rp_forward / rp_backward) and its checks from Python.

Release attribution: gradients of a loss of the final particle positions
with respect to every particle's initial position and to a multiplier kappa
of the vertical diffusivity.  The model and its piecewise treatment are
described with the C entry points in include/romspath_gpu.h.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Dict, List, Tuple

import numpy as np

from . import _lib
from . import schedule as _sched


def step_table(days: float, dt: int, idt: int, step0: int = 0) -> Tuple[List[_lib.RpAdjStep], int]:
    """The internal steps of run_ROMSPath's time loop (ROMSPath.f90:465-546)
    with the frame number held in each ring slot, as rp_adj_step records;
    returns the table and the largest frame number it uses."""
    slot_frame = {}
    for (k, slot) in _sched.initial_loads():
        slot_frame[slot] = k
    out: List[_lib.RpAdjStep] = []
    kmax = max(slot_frame.values())
    for ext in _sched.external_steps(days, dt, idt):
        for (k, slot) in ext.loads:
            slot_frame[slot] = k
            kmax = max(kmax, k)
        for it in ext.internal:
            st = _lib.RpAdjStep()
            for q in range(3):
                st.ex[q] = it.ex[q]
                st.ix[q] = it.ix[q]
            st.ets = it.ets
            st.frame_b, st.frame_c, st.frame_f = slot_frame[it.tb], slot_frame[it.tc], slot_frame[it.tf]
            st.step_index = step0 + it.step_index
            out.append(st)
    return out, kmax


def attribution_loss(x: np.ndarray, y: np.ndarray, target: Tuple[float, float], sigma: float = 5.0):
    """L = sum_p exp(-|x_p - target|^2 / (2 sigma^2)) (grid cells) and its
    gradient with respect to the final x, y."""
    dx = x - target[0]
    dy = y - target[1]
    k = np.exp(-(dx * dx + dy * dy) / (2.0 * sigma * sigma))
    return float(k.sum()), -k * dx / (sigma * sigma), -k * dy / (sigma * sigma)


class Adjoint:
    """Adjoint pair on a Tracker's context (particles set by locate or
    set_particles, one grid or nested grids)."""

    def __init__(self, tracker):
        self.T = tracker
        self.L = tracker.L
        self.h = tracker.h
        self.steps: List[_lib.RpAdjStep] = []
        self.n = 0

    def _check(self, rc, what):
        self.T._check(rc, what)

    def load_frames(self, nframes: int, frame_for: Callable[[int, int], Dict[str, np.ndarray]]):
        """Frames 1..nframes of every grid into the store (frame_for(ng, k))."""
        self._check(self.L.rp_adj_frames(self.h, int(nframes)), "rp_adj_frames")
        for ng in range(1, self.T.ng + 1):
            for k in range(1, nframes + 1):
                f = frame_for(ng, k)
                arrs = [np.asfortranarray(f[q], dtype=np.float64) for q in ("zeta", "u", "v", "w", "aks")]
                st = self.T.params.stokes and "su" in f
                su = np.asfortranarray(f["su"], dtype=np.float64) if st else None
                sv = np.asfortranarray(f["sv"], dtype=np.float64) if st else None
                rc = self.L.rp_adj_set_frame(self.h, ng, k, *[a.ctypes.data_as(_lib.PD) for a in arrs],
                                             su.ctypes.data_as(_lib.PD) if su is not None else None,
                                             sv.ctypes.data_as(_lib.PD) if sv is not None else None)
                self._check(rc, "rp_adj_set_frame")

    def forward(self, steps: List[_lib.RpAdjStep], kappa: float = 1.0, checkpoint_every: int = 48):
        arr = (_lib.RpAdjStep * len(steps))(*steps)
        self._check(self.L.rp_forward(self.h, len(steps), arr, float(kappa), int(checkpoint_every)), "rp_forward")
        self.steps = steps
        self.n = self.T.n
        self.kappa = float(kappa)

    def backward(self, dLdx: np.ndarray, dLdy: np.ndarray, dLdz: np.ndarray):
        n = self.n
        ins = [np.ascontiguousarray(a, dtype=np.float64) for a in (dLdx, dLdy, dLdz)]
        outs = [np.empty(n) for _ in range(3)]
        gk = C.c_double()
        rc = self.L.rp_backward(self.h, *[a.ctypes.data_as(_lib.PD) for a in ins],
                                *[a.ctypes.data_as(_lib.PD) for a in outs], C.byref(gk))
        self._check(rc, "rp_backward")
        return outs[0], outs[1], outs[2], gk.value

    def tangent(self, kappa: float = None) -> np.ndarray:
        """d(final x, y, z)/d(x0, y0, z0, kappa) per particle: (n, 3, 4)."""
        jac = np.empty((self.n, 3, 4))
        rc = self.L.rp_tangent(self.h, float(self.kappa if kappa is None else kappa), jac.ctypes.data_as(_lib.PD))
        self._check(rc, "rp_tangent")
        return jac

    def replay(self, x0=None, y0=None, z0=None, kappa: float = None):
        n = self.n
        ins = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (x0, y0, z0)]
        outs = [np.empty(n) for _ in range(3)]
        rc = self.L.rp_adj_replay(self.h, *[None if a is None else a.ctypes.data_as(_lib.PD) for a in ins],
                                  float(self.kappa if kappa is None else kappa),
                                  *[a.ctypes.data_as(_lib.PD) for a in outs])
        self._check(rc, "rp_adj_replay")
        return outs[0], outs[1], outs[2]
