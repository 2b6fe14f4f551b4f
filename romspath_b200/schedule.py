"""Frame-slot and time schedule of the kept Fortran driver.

Restates ``run_ROMSPath`` / ``run_External_Timestep`` /
``run_Internal_Timestep`` (ROMSPath.f90:151-178, 465-546) and the three
initial ``updateHydro`` calls of ``ini_ROMSPath`` (ROMSPath.f90:307-309):
which frame goes into which ring slot, the external times ``ex`` and the
internal times ``ix`` handed to ``update_particles``.

Quirk kept on purpose: the global ``tstep`` is still 1 after the three
initial loads and is only incremented at the end of each external step, so
at ``ets = 3`` frame 3 is loaded a second time; the slots then hold frames
(1,2,3), (1,2,3), (2,3,3), (3,3,4), (3,4,5), ... for ets = 1, 2, 3, 4, 5.
"""
from __future__ import annotations

import dataclasses
from typing import Iterator, List, Tuple


@dataclasses.dataclass
class InternalStep:
    ets: int
    its: int
    ex: Tuple[float, float, float]
    ix: Tuple[float, float, float]
    tb: int
    tc: int
    tf: int
    step_index: int          # 0-based count of internal steps since start


@dataclasses.dataclass
class ExternalStep:
    ets: int
    loads: List[Tuple[int, int]]   # (frame number, slot) to load before stepping
    ex: Tuple[float, float, float]
    tb: int
    tc: int
    tf: int
    internal: List[InternalStep]


def initial_loads() -> List[Tuple[int, int]]:
    """ROMSPath.f90:307-309: frames 1, 2, 3 into slots t_b=1, t_c=2, t_f=3."""
    return [(1, 1), (2, 2), (3, 3)]


def external_steps(days: float, dt: int, idt: int) -> Iterator[ExternalStep]:
    """Yield the external steps of a run of ``days`` days."""
    seconds = int(_real32_mul(days, 86400.0))           # int(days*86400.0), REAL arithmetic
    step_t = seconds // dt
    tb, tc, tf = 1, 2, 3
    tstep = 1
    k = 0
    for ets in range(1, step_t + 1):
        step_it = int(dt / idt)
        loads: List[Tuple[int, int]] = []
        if ets > 2:
            tb = tb % 3 + 1
            tc = tc % 3 + 1
            tf = tf % 3 + 1
            loads.append((tstep, tf))
        ex = (float((ets - 2) * dt), float((ets - 1) * dt), float(ets * dt))
        internal = []
        for its in range(1, step_it + 1):
            ix = (ex[1] + float((its - 2) * idt), ex[1] + float((its - 1) * idt),
                  ex[1] + float(its * idt))
            internal.append(InternalStep(ets, its, ex, ix, tb, tc, tf, k))
            k += 1
        yield ExternalStep(ets, loads, ex, tb, tc, tf, internal)
        tstep += 1


def _real32_mul(a: float, b: float) -> float:
    import numpy as np
    return float(np.float32(a) * np.float32(b))
