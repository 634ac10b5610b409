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
METHOD_CODES = {"leapfrog": 0, "rk4": 1, "rk6": 2, "symplec4": 3, "symplec6": 4, "dopr54": 5,
                "dop853": 6}


class Harness:
    """npot (integrate, dop853_queued, integrate_sos, forces): galpy's count
    of top-level potential entries when a wrapper carries wrapped ones
    (default len(pot_type))."""

    def __init__(self, lib):
        self.lib = lib

    def integrate(self, w, t, pot_type, pot_args, method, planar=False, var=False, f32=False,
                  dt=None, rtol=None, atol=None, max_attempts=0, npot=None):
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
            t.ctypes.data_as(_dp), int(t.ndim > 1), (len(pt) if npot is None else npot), pt.ctypes.data_as(_ip),
            pa.ctypes.data_as(_dp), ctypes.c_double(-9999.99 if dt is None else dt),
            ctypes.c_double(r), ctypes.c_double(a), ctypes.c_longlong(max_attempts),
            out.ctypes.data_as(_dp), err.ctypes.data_as(_ip), ns.ctypes.data_as(_lp))
        assert rc == 0, rc
        return out, err, ns

    def dop853_queued(self, w, t, pot_type, pot_args, planar=False, rtol=None, atol=None,
                      max_attempts=0, npot=None):
        """DOP853 with its dense output through the kernels' request record
        (served one request at a time); same return values as integrate."""
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
        rc = self.lib.harness_dop853_queued(
            int(planar), n, w.ctypes.data_as(_dp), nt, t.ctypes.data_as(_dp), int(t.ndim > 1),
            (len(pt) if npot is None else npot), pt.ctypes.data_as(_ip), pa.ctypes.data_as(_dp), ctypes.c_double(r),
            ctypes.c_double(a), ctypes.c_longlong(max_attempts), out.ctypes.data_as(_dp),
            err.ctypes.data_as(_ip), ns.ctypes.data_as(_lp))
        assert rc == 0, rc
        return out, err, ns

    def integrate_sos(self, w, psi, pot_type, pot_args, method, dpsi=None, rtol=None,
                      atol=None, max_attempts=0, surface=None, npot=None):
        """SOS machines on SOS states: 3D w [n][7], or planar w [n][5] with
        surface 0 (x = 0) or 1 (y = 0); returns raw rows [n][npsi][7 | 5]."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        n, nv = w.shape
        npsi = psi.shape[-1]
        system = 1 if surface is None else 2 + int(surface)
        out = np.zeros((n, npsi, nv))
        err = np.zeros(n, np.int32)
        ns = np.zeros(n, np.int64)
        pt = np.ascontiguousarray(pot_type, np.int32)
        pa = np.ascontiguousarray(pot_args, np.float64)
        r = -12 * np.log(10) if rtol is None else np.log(rtol)
        a = -12 * np.log(10) if atol is None else np.log(atol)
        rc = self.lib.harness_integrate_sos(
            system, METHOD_CODES[method], n, w.ctypes.data_as(_dp), npsi,
            psi.ctypes.data_as(_dp),
            int(psi.ndim > 1), (len(pt) if npot is None else npot), pt.ctypes.data_as(_ip), pa.ctypes.data_as(_dp),
            ctypes.c_double(-9999.99 if dpsi is None else dpsi), ctypes.c_double(r),
            ctypes.c_double(a), ctypes.c_longlong(max_attempts), out.ctypes.data_as(_dp),
            err.ctypes.data_as(_ip), ns.ctypes.data_as(_lp))
        assert rc == 0, rc
        return out, err, ns

    def forces(self, x, y, z, pot_type, pot_args, planar=False, t=0.0, npot=None):
        x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
        n = len(x)
        acc, tid, a32 = np.zeros((n, 3)), np.zeros((n, 6)), np.zeros((n, 3))
        pt = np.ascontiguousarray(pot_type, np.int32)
        pa = np.ascontiguousarray(pot_args, np.float64)
        rc = self.lib.harness_forces_at(
            int(planar), n, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp), z.ctypes.data_as(_dp),
            ctypes.c_double(t), (len(pt) if npot is None else npot), pt.ctypes.data_as(_ip), pa.ctypes.data_as(_dp),
            acc.ctypes.data_as(_dp), tid.ctypes.data_as(_dp), a32.ctypes.data_as(_dp))
        assert rc == 0, rc
        return acc, tid, a32

    # ----------------------------------------------------------- adjoint ---
    def _pot(self, pot_type, pot_args):
        pt = np.ascontiguousarray(pot_type, np.int32)
        pa = np.ascontiguousarray(pot_args, np.float64)
        return pt, pa, len(pt), pt.ctypes.data_as(_ip), pa.ctypes.data_as(_dp)

    def adj_nparam(self, pot_type, pot_args, planar=False):
        pt, pa, n, ptp, pap = self._pot(pot_type, pot_args)
        return self.lib.harness_adj_nparam(int(planar), n, ptp, pap)

    def adj_param_vjp(self, x, y, z, lam, pot_type, pot_args, planar=False):
        """g[i, p] = lam_i . d a(x_i) / d theta_p"""
        x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
        lam = np.ascontiguousarray(lam, np.float64)
        pt, pa, n, ptp, pap = self._pot(pot_type, pot_args)
        g = np.zeros((len(x), self.adj_nparam(pt, pa, planar)))
        self.lib.harness_adj_param_vjp(int(planar), len(x), x.ctypes.data_as(_dp),
                                       y.ctypes.data_as(_dp), z.ctypes.data_as(_dp),
                                       lam.ctypes.data_as(_dp), n, ptp, pap, g.ctypes.data_as(_dp))
        return g

    def adj_forward(self, w0, t0, tend, pot_type, pot_args, planar=False, rtol=1e-10, atol=1e-10,
                    hcap=100000):
        w0 = np.ascontiguousarray(w0, np.float64)
        nobj, nv = w0.shape
        pt, pa, n, ptp, pap = self._pot(pot_type, pot_args)
        yT, ns, err = np.zeros((nobj, nv)), np.zeros(nobj, np.int64), np.zeros(nobj, np.int32)
        h = np.zeros((nobj, hcap))
        rc = self.lib.harness_adj_forward(
            int(planar), nobj, w0.ctypes.data_as(_dp), ctypes.c_double(t0), ctypes.c_double(tend),
            ctypes.c_double(np.log(rtol)), ctypes.c_double(np.log(atol)), n, ptp, pap,
            yT.ctypes.data_as(_dp), ns.ctypes.data_as(_lp), err.ctypes.data_as(_ip),
            h.ctypes.data_as(_dp), ctypes.c_longlong(hcap))
        assert rc == 0, rc
        return yT, ns, err, h[:, :max(int(ns.max()), 1)].copy()

    def adj_replay(self, w0, t0, tend, pot_type, pot_args, h, ns, planar=False):
        w0 = np.ascontiguousarray(w0, np.float64)
        h = np.ascontiguousarray(h, np.float64)
        ns = np.ascontiguousarray(ns, np.int64)
        pt, pa, n, ptp, pap = self._pot(pot_type, pot_args)
        yT = np.zeros_like(w0)
        self.lib.harness_adj_replay(int(planar), len(w0), w0.ctypes.data_as(_dp),
                                    ctypes.c_double(t0), ctypes.c_double(tend), n, ptp, pap,
                                    h.ctypes.data_as(_dp), ctypes.c_longlong(h.shape[1]),
                                    ns.ctypes.data_as(_lp), yT.ctypes.data_as(_dp))
        return yT

    def adj_gradient(self, w0, t0, tend, pot_type, pot_args, gyT, planar=False, rtol=1e-10,
                     atol=1e-10):
        """(dL/dw0, per-orbit dL/dtheta, err) for dL/dy(tend) = gyT."""
        w0 = np.ascontiguousarray(w0, np.float64)
        gyT = np.ascontiguousarray(gyT, np.float64)
        pt, pa, n, ptp, pap = self._pot(pot_type, pot_args)
        gw = np.zeros_like(w0)
        gth = np.zeros((len(w0), self.adj_nparam(pt, pa, planar)))
        err = np.zeros(len(w0), np.int32)
        self.lib.harness_adj_gradient(
            int(planar), len(w0), w0.ctypes.data_as(_dp), ctypes.c_double(t0),
            ctypes.c_double(tend), ctypes.c_double(np.log(rtol)), ctypes.c_double(np.log(atol)),
            n, ptp, pap, gyT.ctypes.data_as(_dp), gw.ctypes.data_as(_dp), gth.ctypes.data_as(_dp),
            err.ctypes.data_as(_ip))
        return gw, gth, err

    def adj_backward_frozen(self, w0, t0, tend, pot_type, pot_args, h, ns, gyT, planar=False):
        """(dL/dw0, per-orbit dL/dtheta) of the map with frozen steps h [N, hcap]."""
        w0 = np.ascontiguousarray(w0, np.float64)
        gyT = np.ascontiguousarray(gyT, np.float64)
        h = np.ascontiguousarray(h, np.float64)
        ns = np.ascontiguousarray(ns, np.int64)
        pt, pa, n, ptp, pap = self._pot(pot_type, pot_args)
        gw = np.zeros_like(w0)
        gth = np.zeros((len(w0), self.adj_nparam(pt, pa, planar)))
        self.lib.harness_adj_backward_frozen(
            int(planar), len(w0), w0.ctypes.data_as(_dp), ctypes.c_double(t0),
            ctypes.c_double(tend), n, ptp, pap, h.ctypes.data_as(_dp),
            ctypes.c_longlong(h.shape[1]), ns.ctypes.data_as(_lp), gyT.ctypes.data_as(_dp),
            gw.ctypes.data_as(_dp), gth.ctypes.data_as(_dp))
        return gw, gth
