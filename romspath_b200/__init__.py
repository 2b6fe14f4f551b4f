"""B200-native ROMSPath particle step.

The hot path of ROMSPath (``update_particles``, ROMSPath.f90:608-1008, and
everything it calls) as hand-written sm_100a CUDA behind the C ABI of
``include/romspath_gpu.h``.  ``Tracker`` is the host mirror of the calls the
Fortran driver makes; ``synth`` builds ROMS-shaped synthetic inputs;
``schedule`` replays the driver's frame-slot / time schedule.
"""
from . import schedule, synth  # noqa: F401
from ._lib import FLAG_NODE, FLAG_OOB, FLAG_SPLINE, FLAG_WBOT, FLAG_WTOP, load  # noqa: F401
from .tracker import RomsPathError, Tracker  # noqa: F401

__all__ = ["Tracker", "RomsPathError", "load", "synth", "schedule"]
