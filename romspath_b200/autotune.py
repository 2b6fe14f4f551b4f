"""Autotuning of the launch settings on the run itself.

The step's results do not depend on the launch settings (re-sort interval,
resident blocks per SM -- hence particles per thread -- ; the kernel form
is fixed at context creation), so the tuner times real frame intervals of
the run under each candidate setting and keeps the fastest: no step is
wasted.  Block size is fixed at 128 threads by the kernels' launch bounds.
"""
from __future__ import annotations

from typing import Callable, Dict, Iterable, List, Tuple

DEFAULT_CANDIDATES: List[Tuple[int, int]] = [
    # (re-sort interval in internal steps, resident blocks per SM; 0 = occupancy limit)
    (12, 0), (24, 0), (6, 0), (0, 0), (12, 6), (12, 4),
]


def tune(tracker, run_interval: Callable[[], float], candidates: Iterable[Tuple[int, int]] = DEFAULT_CANDIDATES,
         reps: int = 2) -> Dict:
    """run_interval() advances the run by one frame interval and returns its
    device time in ms.  Each candidate runs `reps` intervals (the minimum
    counts); the best setting is left in place.  Returns the table."""
    table = []
    for resort, bps in candidates:
        tracker.set_launch(resort, bps)
        t = min(run_interval() for _ in range(reps))
        table.append({"resort": resort, "blocks_per_sm": bps, "ms_per_interval": t})
    best = min(table, key=lambda r: r["ms_per_interval"])
    tracker.set_launch(best["resort"], best["blocks_per_sm"])
    return {"best": best, "table": table}
