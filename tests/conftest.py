"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and the built
libgalpy_cuda.so; everything else runs on the CPU (the oracle, the host-side
logic, and the engine's device code compiled as host C++ by
tests/harness/host_harness.cpp)."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libgalpy_cuda.so")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(TESTS, "golden", "golden.npz")))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    if not os.path.exists(O.PORT_SO):
        O.build()
    return O


@pytest.fixture(scope="session")
def mw14(golden):
    return golden["mw14_type"], golden["mw14_args"]


@pytest.fixture(scope="session")
def mw14_planar(golden):
    return golden["mw14_planar_type"], golden["mw14_planar_args"]


HARNESS_SRC = os.path.join(TESTS, "harness", "host_harness.cpp")
HARNESS_SO = os.path.join(TESTS, "_build", "libharness.so")


@pytest.fixture(scope="session")
def harness():
    """The engine's device code compiled as host C++ (test-only)."""
    os.makedirs(os.path.dirname(HARNESS_SO), exist_ok=True)
    deps = [HARNESS_SRC] + [os.path.join(ROOT, "galpy_b200", "csrc", f) for f in os.listdir(
        os.path.join(ROOT, "galpy_b200", "csrc"))]
    if not os.path.exists(HARNESS_SO) or any(
            os.path.getmtime(d) > os.path.getmtime(HARNESS_SO) for d in deps):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", HARNESS_SO,
                        HARNESS_SRC], check=True)
    return Harness(ctypes.CDLL(HARNESS_SO))


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_longlong)
METHOD_CODES = {"leapfrog": 0, "rk4": 1, "symplec4": 3, "dop853": 6}


class Harness:
    def __init__(self, lib):
        self.lib = lib

    def integrate(self, w, t, pot_type, pot_args, method, planar=False, var=False, f32=False,
                  dt=None, rtol=None, atol=None, max_attempts=0):
        w = np.ascontiguousarray(w, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64)
        n, nv = w.shape
        nt = t.shape[-1]
        out = np.zeros((n, nt, nv))
        err = np.zeros(n, np.int32)
        ns = np.zeros(n, np.int64)
        pt = np.ascontiguousarray(pot_type, np.int32)
        pa = np.ascontiguousarray(pot_args, np.float64)
        r = -12 * np.log(10) if rtol is None else np.log(rtol)
        a = -12 * np.log(10) if atol is None else np.log(atol)
        rc = self.lib.harness_integrate(
            int(planar), int(var), METHOD_CODES[method], int(f32), n, w.ctypes.data_as(_dp), nt,
            t.ctypes.data_as(_dp), int(t.ndim > 1), len(pt), pt.ctypes.data_as(_ip),
            pa.ctypes.data_as(_dp), ctypes.c_double(-9999.99 if dt is None else dt),
            ctypes.c_double(r), ctypes.c_double(a), ctypes.c_longlong(max_attempts),
            out.ctypes.data_as(_dp), err.ctypes.data_as(_ip), ns.ctypes.data_as(_lp))
        assert rc == 0, rc
        return out, err, ns

    def forces(self, x, y, z, pot_type, pot_args, planar=False):
        x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
        n = len(x)
        acc, tid, a32 = np.zeros((n, 3)), np.zeros((n, 6)), np.zeros((n, 3))
        pt = np.ascontiguousarray(pot_type, np.int32)
        pa = np.ascontiguousarray(pot_args, np.float64)
        rc = self.lib.harness_forces(int(planar), n, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                     z.ctypes.data_as(_dp), len(pt), pt.ctypes.data_as(_ip),
                                     pa.ctypes.data_as(_dp), acc.ctypes.data_as(_dp),
                                     tid.ctypes.data_as(_dp), a32.ctypes.data_as(_dp))
        assert rc == 0, rc
        return acc, tid, a32
