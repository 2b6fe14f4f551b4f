"""The kept Fortran driver's frame-slot schedule (ROMSPath.f90:307-309,
465-546), including the frame-3-loaded-twice quirk."""
from romspath_b200 import schedule


def frames_held(n_ext):
    slots = {}
    for f, s in schedule.initial_loads():
        slots[s] = f
    held = []
    for ext in schedule.external_steps(n_ext / 24.0, 3600, 300):
        for f, s in ext.loads:
            slots[s] = f
        held.append((slots[ext.tb], slots[ext.tc], slots[ext.tf]))
    return held


def test_frames_held_per_external_step():
    held = frames_held(7)
    assert held[:5] == [(1, 2, 3), (1, 2, 3), (2, 3, 3), (3, 3, 4), (3, 4, 5)]
    assert held[5] == (4, 5, 6)
    assert held[6] == (5, 6, 7)


def test_times():
    ext = list(schedule.external_steps(1.0, 3600, 300))
    assert len(ext) == 24
    assert all(len(e.internal) == 12 for e in ext)
    e1 = ext[0]
    assert e1.ex == (-3600.0, 0.0, 3600.0)
    assert e1.internal[0].ix == (-300.0, 0.0, 300.0)
    assert e1.internal[-1].ix == (3000.0, 3300.0, 3600.0)
    idx = [it.step_index for e in ext for it in e.internal]
    assert idx == list(range(288))


def test_days_uses_single_precision_product():
    # seconds = int(days*86400.0) in REAL arithmetic
    assert len(list(schedule.external_steps(10.0, 3600, 300))) == 240


def test_autotune_two_stages_with_a_fake_tracker():
    """The tuner picks the fastest kernel form first, then the fastest
    re-sort interval and occupancy for it, and leaves them in place."""
    from romspath_b200 import autotune

    class Fake:
        field_dtype = "mixed"

        def __init__(self):
            self.form, self.launch, self.calls = "fused", (12, 0), []

        def set_kernel_form(self, form):
            self.form = form

        def set_launch(self, resort, bps):
            self.launch = (resort, bps)

    T = Fake()
    cost = {"fused": 3.0, "fused-noprefetch": 3.2, "smem": 2.5, "fused-b64": 3.1, "fused-b256": 2.9}

    def interval():
        resort, bps = T.launch
        return cost[T.form] + (0.0 if resort == 24 else 0.1) + (0.05 if bps else 0.0)

    out = autotune.tune(T, interval, reps=1)
    assert T.form == "smem" and T.launch == (24, 0)
    assert out["best"] == {"form": "smem", "resort": 24, "blocks_per_sm": 0, "ms_per_interval": 2.5}
    assert [r["form"] for r in out["forms"]] == autotune.MIXED_FORMS
