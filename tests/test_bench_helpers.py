"""bench.py's host-side helpers on the CPU: the committed ncu figures it
reads (DRAM/L2 traffic, FP64 counts) are present and self-consistent for
the kernels its roofline and `spline` objects name, and the clock sampler
parses nvidia-smi's CSV and keeps the throttle reasons that reject a run."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_traffic_profiles_cover_the_headline_kernels():
    for wl, k in (("cfg2", "k_step_mixed"), ("cfg2", "k_step_fused"), ("cfg3", "k_step_mixed")):
        t = bench.profile_traffic(wl, k)
        assert t is not None and t > 1e9, (wl, k)
    assert bench.profile_traffic("cfg3", "k_step_mixed", "lts_bytes_per_launch") > \
        bench.profile_traffic("cfg3", "k_step_mixed")
    assert bench.profile_traffic("cfg2", "no_such_kernel") is None
    assert bench.profile_traffic("no_such_workload", "k_step_mixed") is None


def test_fp64_profiles_are_consistent():
    for k, form in (("k_step_mixed", "mixed"), ("k_step_fused", "f32")):
        p = bench.profile_fp64("cfg2", k)
        assert p["form"] == form
        assert p["fp64_flop_per_launch"] == p["dadd"] + p["dmul"] + 2 * p["dfma"]
        assert 0.0 < p["fp64_pipe_active_pct"] < 100.0
        assert p["particles"] == 1 << 20
    # the exact form does far more FP64 work per particle-step than the mixed one
    assert bench.profile_fp64("cfg2", "k_step_fused")["fp64_flop_per_launch"] > \
        10 * bench.profile_fp64("cfg2", "k_step_mixed")["fp64_flop_per_launch"]


def test_workload_descriptions():
    for wl in ("cfg1", "cfg2", "cfg3"):
        assert bench.WORKLOAD_DESCS[wl].startswith(wl + ":")


def test_clock_sampler_parses_samples(tmp_path):
    s = bench.ClockSampler(0)
    s.path = str(tmp_path / "clocks.csv")
    with open(s.path, "w") as f:
        f.write("0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active\n")
        f.write("0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active\n")
        f.write("0, 345, 1965, 120.0, 0x1, Not Active, Not Active, Not Active, Not Active\n")
        f.write("garbage line\n")

    class _Done:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    s.proc = _Done()
    out = s.stop()
    assert out["samples"] == 3
    assert out["sm_max_mhz"] == 1965.0
    assert out["sm_mhz"] == pytest.approx(1957.5)      # idle sample below half the max left out
    assert out["reasons"] == ["sw_power_cap"]
    assert not os.path.exists(str(tmp_path / "clocks.csv"))


def test_measured_peaks_fallback_or_file():
    peak, src = bench.measured_peaks()
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert src.startswith("measured")
        assert peak == float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    else:
        assert (peak, src) == (6650.0, "fallback (6.65 TB/s)")


def test_measured_peaks_file_forms(tmp_path):
    p = tmp_path / "peaks.json"
    p.write_text(json.dumps({"hbm_gbs": 6549.5, "bf16_tflops": 1590.0}))
    assert bench.measured_peaks(str(p)) == (6549.5, "measured (MEASURED_PEAKS.json hbm_gbs)")
    p.write_text(json.dumps({"gpu0": {"hbm_gbs": 6400.0}}))
    assert bench.measured_peaks(str(p))[0] == 6400.0
    p.write_text(json.dumps({"gpus": [{"index": 0}, {"hbm_gbs": 6300.0}]}))
    assert bench.measured_peaks(str(p))[0] == 6300.0          # objects inside lists
    p.write_text(json.dumps({"hbm_gbs": True, "detail": {"hbm_gbs": 6200.0}}))
    assert bench.measured_peaks(str(p))[0] == 6200.0          # a boolean is not a bandwidth
    p.write_text(json.dumps({"hbm_gbs": True}))
    assert bench.measured_peaks(str(p)) == (6650.0, "fallback (6.65 TB/s)")
    p.write_text("not json")
    assert bench.measured_peaks(str(p)) == (6650.0, "fallback (6.65 TB/s)")
    assert bench.measured_peaks(str(tmp_path / "absent.json"))[1].startswith("fallback")


def test_param_overrides():
    params = {"vturb_on": 1, "sub": 4.0, "deltat": 30.0}
    assert bench.parse_params([], params) == {}
    assert bench.parse_params(["vturb_on=0", "sub=2.5", "deltat=300"], params) == \
        {"vturb_on": 0, "sub": 2.5, "deltat": 300}
    with pytest.raises(SystemExit):
        bench.parse_params(["no_such=1"], params)
    with pytest.raises(SystemExit):
        bench.parse_params(["vturb_on"], params)
