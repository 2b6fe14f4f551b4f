"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py
from the oracle): the oracle must reproduce them exactly (CPU), and so must
the CUDA path (GPU)."""
import glob
import os

import numpy as np
import pytest

import harness

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def _load(path):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import case_from_fixture
    d = np.load(path, allow_pickle=True)
    return d, case_from_fixture(d)


def _expected(d):
    return {f: d["exp_" + f] for f in harness.FIELDS}


def test_fixtures_present():
    assert len(FIXTURES) >= 4


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_reproduces_golden(path):
    d, case = _load(path)
    noise = str(d["noise"])
    hook = d["hook"] if "hook" in d.files else None
    o, _ = harness.run_oracle(case, int(d["nsteps"]), noise=noise, hook=hook, seed=int(d["seed"]), nthreads=2)
    diff = {k: v for k, v in harness.compare(o, _expected(d)).items() if v}
    assert not diff, diff


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_gpu_reproduces_golden(path):
    d, case = _load(path)
    noise = str(d["noise"])
    hook = d["hook"] if "hook" in d.files else None
    g, T = harness.run_gpu(case, int(d["nsteps"]), noise=noise, hook=hook, seed=int(d["seed"]))
    T.close()
    diff = {k: v for k, v in harness.compare(g, _expected(d)).items() if v}
    assert not diff, diff
