"""Generate the golden fixtures in tests/golden/ from the CPU oracle.

The reference ships no tests, fixtures or known-answer files, and it cannot
be compiled here (Fortran + NetCDF, no Fortran compiler), so these vectors
are produced by the oracle -- the line-faithful FP64 restatement of the
reference step -- and serve as regression anchors for both the oracle and
the CUDA path.  Each fixture is self-contained: grid, the stored frame
values, the release, the noise (for hook runs) and the expected final
particle columns.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import harness  # noqa: E402

CASES = {
    # name: (config, particles, steps, noise, spec overrides, param overrides)
    "tiny_det": ("tiny", 120, 48, "off", None, {"vturb_on": 0, "hturb_on": 0}),
    "tiny_hook": ("tiny", 80, 24, "hook", None, None),
    "tiny_philox": ("tiny", 80, 24, "philox", None, None),
    "tiny_f32_stokes": ("tiny", 80, 24, "philox", {"field_dtype": "f32", "stokes": True}, None),
    "nest_philox": ("nest_tiny", 120, 36, "philox", None, None),
}


def case_from_fixture(d):
    """Rebuild a harness.Case from a fixture's stored arrays."""
    from romspath_b200 import synth
    specs = [synth.GridSpec(**{k: (v.item() if hasattr(v, "item") else v) for k, v in sp.items()})
             for sp in d["specs"]]
    ng = len(specs)
    grids = [{k[len(f"grid{g}_"):]: d[k] for k in d.files if k.startswith(f"grid{g}_")} for g in range(1, ng + 1)]
    params = d["params"].item()
    release = synth.Release(ipos=d["rel_ipos"], jpos=d["rel_jpos"], z=d["rel_z"], dob=d["rel_dob"])
    frames = {}
    for k in d.files:
        if k.startswith("frame_"):
            _, g, num, field = k.split("_", 3)
            frames.setdefault((int(g), int(num)), {})[field] = d[k]
    c = harness.Case("fixture", specs, grids, params, release, frames)
    if ng > 1:
        c.scl, c.off = d["scl"], d["off"]
    return c


def make(name):
    cfg, npart, nsteps, noise, sov, pov = CASES[name]
    case = harness.make_case(cfg, npart, seed=4, spec_over=sov, param_over=pov)
    hook = harness.noise_array(case, nsteps, seed=99) if noise == "hook" else None
    o, _ = harness.run_oracle(case, nsteps, noise=noise, hook=hook, seed=5, nthreads=1)
    nframes = 2 + (nsteps + 11) // 12 + 1
    out = {
        "specs": np.array([vars(sp) for sp in case.specs], dtype=object),
        "params": np.array(case.params, dtype=object),
        "rel_ipos": case.release.ipos, "rel_jpos": case.release.jpos,
        "rel_z": case.release.z, "rel_dob": case.release.dob,
        "nsteps": np.array(nsteps), "noise": np.array(noise), "seed": np.array(5),
    }
    for g in range(1, case.ngrid + 1):
        for k, v in case.grids[g - 1].items():
            out[f"grid{g}_" + k] = v
        for k in range(1, nframes + 1):
            for f, v in case.frame(k, g).items():
                out[f"frame_{g}_{k}_{f}"] = v
    if case.ngrid > 1:
        out["scl"], out["off"] = case.scl, case.off
    if hook is not None:
        out["hook"] = hook
    for f in harness.FIELDS:
        out["exp_" + f] = o[f]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: v.shape for k, v in out.items() if k.startswith("exp_")}["exp_x"])


if __name__ == "__main__":
    for n in CASES:
        make(n)
