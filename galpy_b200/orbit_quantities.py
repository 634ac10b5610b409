"""Integrals of motion of stored orbits on the GPU.

galpy evaluates the energy and the Jacobi integral of an integrated orbit in
Python over its (N, nt) rows (Orbit.E, galpy/orbit/Orbits.py:2902, and
Orbit.Jacobi = E - Omega . L, :3298-3375).  Here the potential sums run in
the integration kernels' own force library:

* ``jacobi_device`` -- E - Omega . L (Omega = 0: the energy) of
  device-resident rectangular states, e.g. the SoA snapshots of a batch
  integration, without leaving the GPU;
* ``potential_values`` -- Phi at host points (R, z, phi), the potential sum
  behind Orbit.E / Orbit.Jacobi when galpy_hooks routes them;
* ``energies`` -- E or the Jacobi integral of galpy-layout cylindrical rows.
"""
import ctypes

import numpy as np

from . import _lib
from .integrate import compile_potential


def jacobi_device(comps, ncomp, w, J, omega=(0.0, 0.0, 0.0), planar=False, layout="soa",
                  group=None, stream=None):
    """J = v^2/2 + Phi(x) - Omega . (x cross v) of device-resident states.

    comps: uint8 CUDA tensor of compiled records (compile_potential); w:
    float64 CUDA tensor [nv, N] ('soa') or [N, nv] ('aos') or any strided
    view with those axes, rectangular (x, y[, z], vx, vy[, vz]); J: float64
    [N]; omega: the pattern-speed vector (galpy's OmegaP; a scalar is the z
    component, as galpy's Orbit.Jacobi takes it)."""
    import torch

    if not (J.is_cuda and J.dtype == torch.float64):
        raise ValueError("J must be a float64 CUDA tensor")
    if layout == "soa":
        sc, so = w.stride(0), w.stride(1)
    else:
        so, sc = w.stride(0), w.stride(1)
    om = np.zeros(3)
    if np.ndim(omega) == 0:
        om[2] = float(omega)
    else:
        om[:] = np.asarray(omega, dtype=np.float64)
    om_c = (ctypes.c_double * 3)(*om)
    s = stream if stream is not None else torch.cuda.current_stream(w.device)
    _lib.check(_lib.lib().galpy_cuda_jacobi_device(
        comps.data_ptr(), ncomp, group.data_ptr() if group is not None else None, int(planar),
        w.data_ptr(), J.shape[0], sc, so, om_c, J.data_ptr(), s.cuda_stream))


def _device():
    import torch

    if not torch.cuda.is_available():
        raise _lib.CudaError(_lib.ERR_NODEVICE, "no CUDA device visible")
    return torch.device("cuda", torch.cuda.current_device())


def potential_values(pot, R, z=0.0, phi=0.0, planar=False):
    """Phi(R, z, phi) of a supported potential at host points (arrays
    broadcast together), evaluated on the GPU; shaped like the broadcast."""
    import torch

    R, z, phi = np.broadcast_arrays(np.asarray(R, np.float64), np.asarray(z, np.float64),
                                    np.asarray(phi, np.float64))
    shape = R.shape
    dev = _device()
    buf, ncomp = compile_potential(pot, planar=planar)
    comps = torch.from_numpy(buf).to(dev)
    n = R.size
    nv = 4 if planar else 6
    w = np.zeros((nv, n))
    Rf, pf = R.ravel(), phi.ravel()
    w[0], w[1] = Rf * np.cos(pf), Rf * np.sin(pf)
    if not planar:
        w[2] = z.ravel()
    wd = torch.from_numpy(w).to(dev)
    Pd = torch.empty(n, dtype=torch.float64, device=dev)
    jacobi_device(comps, ncomp, wd, Pd, planar=planar)
    return Pd.cpu().numpy().reshape(shape)


def energies(pot, rows, planar=False, omega=0.0):
    """E (omega = 0) or the Jacobi integral E - Omega . L of galpy-layout
    cylindrical rows [..., (R, vR, vT, z, vz, phi)] (planar: (R, vR, vT,
    phi)), evaluated on the GPU."""
    import torch

    rows = np.asarray(rows, np.float64)
    shape = rows.shape[:-1]
    r = rows.reshape(-1, rows.shape[-1])
    R, vR, vT, phi = r[:, 0], r[:, 1], r[:, 2], r[:, -1]
    c, s = np.cos(phi), np.sin(phi)
    if planar:
        w = np.stack([R * c, R * s, vR * c - vT * s, vR * s + vT * c])
    else:
        w = np.stack([R * c, R * s, r[:, 3], vR * c - vT * s, vR * s + vT * c, r[:, 4]])
    dev = _device()
    buf, ncomp = compile_potential(pot, planar=planar)
    comps = torch.from_numpy(buf).to(dev)
    wd = torch.from_numpy(np.ascontiguousarray(w)).to(dev)
    Jd = torch.empty(len(r), dtype=torch.float64, device=dev)
    jacobi_device(comps, ncomp, wd, Jd, omega=omega, planar=planar)
    return Jd.cpu().numpy().reshape(shape)


def interpolate_device(rows, t, tq, out, stream=None):
    """Orbits between their stored rows, on the device: rows float64 CUDA
    tensor [N, nt, nv] in galpy's cylindrical layout (nv 6 or 4), t [nt] or
    [N, nt] increasing, tq [nq] or [N, nq], out [N, nq, nv] (all contiguous
    float64 CUDA tensors).  Per orbit and component (x = R cos phi and
    y = R sin phi in place of R and phi) the interpolating cubic spline with
    not-a-knot ends -- the spline galpy's Orbit.__call__ evaluates between
    integration times (Orbits.py:6739) -- then back to (R, phi).  Queries
    outside [t_0, t_end] extrapolate the end pieces."""
    import torch

    for name, x in (("rows", rows), ("t", t), ("tq", tq), ("out", out)):
        if not (x.is_cuda and x.dtype == torch.float64 and x.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous float64 CUDA tensor")
    n, nt, nv = rows.shape
    nq = tq.shape[-1]
    if t.shape[-1] != nt or out.shape != (n, nq, nv) or (t.dim() > 1 and t.shape[0] != n) or \
            (tq.dim() > 1 and tq.shape[0] != n):
        raise ValueError("inconsistent shapes")
    s = stream if stream is not None else torch.cuda.current_stream(rows.device)
    _lib.check(_lib.lib().galpy_cuda_orbit_interp_device(
        nv, n, nt, t.data_ptr(), int(t.dim() > 1), rows.data_ptr(), nq, tq.data_ptr(),
        int(tq.dim() > 1), out.data_ptr(), s.cuda_stream))


def interpolate(rows, t, tq):
    """interpolate_device for host arrays: rows [N, nt, nv] galpy-layout
    cylindrical rows, t [nt] or [N, nt] (increasing or decreasing), tq [nq]
    or [N, nq]; returns [N, nq, nv] (numpy)."""
    import torch

    rows = np.asarray(rows, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    tq = np.asarray(tq, dtype=np.float64)
    if t.ndim == 1 and t.size > 1 and t[1] < t[0]:  # a backward integration
        t, rows = t[::-1], rows[:, ::-1]
    elif t.ndim == 2 and t.shape[1] > 1:
        back = t[:, 1] < t[:, 0]
        if back.any():
            t, rows = t.copy(), rows.copy()
            t[back], rows[back] = t[back, ::-1], rows[back, ::-1]
    dev = _device()
    n, _, nv = rows.shape
    out = torch.empty((n, tq.shape[-1], nv), dtype=torch.float64, device=dev)
    interpolate_device(torch.from_numpy(np.ascontiguousarray(rows)).to(dev),
                       torch.from_numpy(np.ascontiguousarray(t)).to(dev),
                       torch.from_numpy(np.ascontiguousarray(tq)).to(dev), out)
    return out.cpu().numpy()
