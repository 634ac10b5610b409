"""oracle/spline.py -- TEST INFRASTRUCTURE ONLY.

The CPU checker of the device orbit interpolation
(galpy_cuda_orbit_interp_device): galpy's Orbit.__call__ between
integration times (galpy/orbit/Orbits.py:6460-6575) evaluates, per orbit and
phase component, the interpolants that _setupOrbitInterp builds
(Orbits.py:6739-6830): scipy's InterpolatedUnivariateSpline(t, y, k=3) per
orbit, or RectBivariateSpline(t, orbit index, ..., ky=1, s=0), whose value
at an integer orbit index is that orbit's interpolating cubic.  Both come
from FITPACK (a third-party library outside the reference tree; scipy's
bundled copy): with s = 0 the cubic's interior knots are the data points but
the second and the second to last -- the not-a-knot interpolating spline.
Fewer than 4 points: degree nt - 1 (galpy's k = max(1, nt - 1) for per-orbit
grids).

This module restates that interpolant from its definition (the not-a-knot
cubic through the points; line and parabola below 4 points), in numpy,
vectorised over orbits, as a dense solve per orbit -- a different route
from the device's moment-form Thomas sweep -- and the galpy unpacking
x = R cos phi, y = R sin phi -> (R, phi).  tests/test_oracle.py pins it
against scipy's FITPACK splines.

Only tests import this module.
"""
import numpy as np


def _cubic_coefficients(t, y):
    """Not-a-knot cubic spline through (t, y), len(t) >= 4: piecewise
    polynomials y_i + b_i s + c_i s^2 + d_i s^3 (s = t - t_i) on each
    interval, from the dense system of the continuity conditions (value at
    both ends of each piece, first and second derivative at interior knots,
    third derivative at t_1 and t_{m-2})."""
    m = len(t)
    npc = m - 1
    h = np.diff(t)
    A = np.zeros((3 * npc, 3 * npc))
    r = np.zeros(3 * npc)
    row = 0
    # value at the right end of each piece: b_i h + c_i h^2 + d_i h^3 = y_{i+1} - y_i
    for i in range(npc):
        A[row, 3 * i:3 * i + 3] = [h[i], h[i] ** 2, h[i] ** 3]
        r[row] = y[i + 1] - y[i]
        row += 1
    # first and second derivatives continuous at interior knots
    for i in range(npc - 1):
        A[row, 3 * i:3 * i + 3] = [1.0, 2 * h[i], 3 * h[i] ** 2]
        A[row, 3 * (i + 1)] = -1.0
        row += 1
        A[row, 3 * i + 1:3 * i + 3] = [2.0, 6 * h[i]]
        A[row, 3 * (i + 1) + 1] = -2.0
        row += 1
    # not-a-knot: third derivative continuous at t_1 and t_{m-2}
    A[row, 2] = 6.0
    A[row, 5] = -6.0
    row += 1
    A[row, 3 * (npc - 2) + 2] = 6.0
    A[row, 3 * (npc - 1) + 2] = -6.0
    row += 1
    sol = np.linalg.solve(A, r)
    return sol.reshape(npc, 3)


def interp1(t, y, tq):
    """The galpy interpolant of one component of one orbit at tq (increasing
    t; tq outside [t_0, t_end] extrapolates the end pieces)."""
    t = np.asarray(t, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    tq = np.asarray(tq, dtype=np.float64)
    m = len(t)
    if m == 1:
        return np.full(tq.shape, y[0])
    if m == 2:
        return y[0] + (tq - t[0]) / (t[1] - t[0]) * (y[1] - y[0])
    if m == 3:
        d01 = (y[1] - y[0]) / (t[1] - t[0])
        d12 = (y[2] - y[1]) / (t[2] - t[1])
        return y[0] + (tq - t[0]) * (d01 + (tq - t[1]) * (d12 - d01) / (t[2] - t[0]))
    coef = _cubic_coefficients(t, y)
    j = np.clip(np.searchsorted(t, tq, side="right") - 1, 0, m - 2)
    s = tq - t[j]
    b, c, d = coef[j, 0], coef[j, 1], coef[j, 2]
    return y[j] + s * (b + s * (c + s * d))


def interpolate(rows, t, tq):
    """rows [N, nt, nv] galpy cylindrical ((R, vR, vT, z, vz, phi) or
    (R, vR, vT, phi)), t [nt] or [N, nt] increasing, tq [nq] or [N, nq]:
    [N, nq, nv] as galpy's Orbit.__call__ interpolates them."""
    rows = np.asarray(rows, dtype=np.float64)
    n, nt, nv = rows.shape
    t = np.asarray(t, dtype=np.float64)
    tq = np.asarray(tq, dtype=np.float64)
    nq = tq.shape[-1]
    out = np.empty((n, nq, nv))
    for i in range(n):
        ti = t[i] if t.ndim > 1 else t
        qi = tq[i] if tq.ndim > 1 else tq
        R, phi = rows[i, :, 0], rows[i, :, -1]
        x = interp1(ti, R * np.cos(phi), qi)
        y = interp1(ti, R * np.sin(phi), qi)
        out[i, :, 0] = np.sqrt(x * x + y * y)
        out[i, :, -1] = np.arctan2(y, x)
        for k in range(1, nv - 1):
            out[i, :, k] = interp1(ti, rows[i, :, k], qi)
    return out
