"""The shared-reciprocal division (Markstein corrections) returns exactly the
IEEE quotient on the device, over random and adversarial operands."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "romspath_b200", "csrc")


def _lib():
    d = tempfile.mkdtemp()
    so = os.path.join(d, "divtest.so")
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-fmad=false", "-shared",
                    "-Xcompiler", "-fPIC", "-I", CSRC, os.path.join(HERE, "gpu_div_selftest.cu"), "-o", so],
                   check=True)
    return C.CDLL(so)


def _operands(n, rng):
    a = rng.uniform(1, 2, n) * 2.0 ** rng.integers(-120, 120, n) * rng.choice([-1, 1], n)
    b = rng.uniform(1, 2, n) * 2.0 ** rng.integers(-120, 120, n) * rng.choice([-1, 1], n)
    # mantissas near 1 and near 2, powers of two, equal operands, zeros, edges
    k = n // 8
    b[:k] = np.nextafter(2.0, 0) * 2.0 ** rng.integers(-40, 40, k)
    a[k:2 * k] = np.nextafter(2.0, 0) * 2.0 ** rng.integers(-40, 40, k)
    b[2 * k:3 * k] = 2.0 ** rng.integers(-60, 60, k)
    a[3 * k:3 * k + 10] = 0.0
    a[3 * k + 10:3 * k + 20] = -0.0
    a[3 * k + 20:4 * k] = b[3 * k + 20:4 * k]
    a[-50:] = 1e-200
    b[-25:] = 1e200
    return a, b


def test_division_is_correctly_rounded():
    L = _lib()
    L.div_selftest.argtypes = [C.c_int64] + [C.POINTER(C.c_double)] * 4
    rng = np.random.default_rng(11)
    n = 1 << 22
    a, b = _operands(n, rng)
    q = np.empty(n)
    r = np.empty(n)
    P = C.POINTER(C.c_double)
    assert L.div_selftest(n, a.ctypes.data_as(P), b.ctypes.data_as(P), q.ctypes.data_as(P),
                          r.ctypes.data_as(P)) == 0
    assert np.array_equal(q.view(np.uint64), r.view(np.uint64))
    assert np.array_equal(r.view(np.uint64), (a / b).view(np.uint64))
