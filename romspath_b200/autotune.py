"""Autotuning of the launch settings on the run itself.

The step's results do not depend on the launch settings beyond rounding
(bit for bit in the exact forms): the kernel form (fused; split; in the
mixed forms the split form with the spline workspace in shared memory, and
the fused kernel without the back substitution's load-ahead), the re-sort
interval and the resident blocks per SM (hence particles per thread).  So
the tuner times real frame intervals of the run under each candidate and
keeps the fastest: no step is wasted.  It tunes in two stages: the kernel
form (which includes the block size of the fused step: 64, 128 or 256
threads) at the default re-sort interval and occupancy, then the re-sort
interval and blocks per SM for the chosen form.  The best form depends on
the grid and the particle count (on the 512x384x30 grid with 1,048,576
particles the fused kernel wins; on the 130x98x20 grid with 4,194,304 the
shared-memory split form does).
"""
from __future__ import annotations

from typing import Callable, Dict, Iterable, List, Optional, Tuple

MIXED_FORMS = ["fused", "fused-noprefetch", "smem", "fused-b64", "fused-b256"]
EXACT_FORMS = ["fused", "split"]

DEFAULT_CANDIDATES: List[Tuple[int, int]] = [
    # (re-sort interval in internal steps, resident blocks per SM; 0 = occupancy limit).
    # "Never re-sort" is not a candidate: timed over a few intervals right
    # after a re-sort it inherits that sort's order and looks fastest, while
    # over a long run the particles drift out of it.
    (12, 0), (24, 0), (6, 0), (48, 0), (12, 6), (12, 4),
]


def tune(tracker, run_interval: Callable[[], float], candidates: Iterable[Tuple[int, int]] = DEFAULT_CANDIDATES,
         reps: int = 2, forms: Optional[List[str]] = None) -> Dict:
    """run_interval() advances the run by one frame interval and returns its
    device time in ms.  Each candidate runs `reps` intervals (the minimum
    counts); the best setting is left in place.  `forms` (default: the
    mixed or the exact forms, by the tracker's field storage) are tried
    first at the first candidate's launch settings.  Returns the tables."""
    cands = list(candidates)
    if forms is None:
        forms = MIXED_FORMS if tracker.field_dtype.startswith("mixed") else EXACT_FORMS
    form_table = []
    r0, b0 = cands[0]
    tracker.set_launch(r0, b0)
    for form in forms:
        tracker.set_kernel_form(form)
        t = min(run_interval() for _ in range(reps))
        form_table.append({"form": form, "ms_per_interval": t})
    best_form = min(form_table, key=lambda r: r["ms_per_interval"])["form"]
    tracker.set_kernel_form(best_form)
    table = []
    for resort, bps in cands:
        tracker.set_launch(resort, bps)
        t = min(run_interval() for _ in range(reps))
        table.append({"form": best_form, "resort": resort, "blocks_per_sm": bps, "ms_per_interval": t})
    best = min(table, key=lambda r: r["ms_per_interval"])
    tracker.set_launch(best["resort"], best["blocks_per_sm"])
    return {"best": best, "forms": form_table, "table": table}
