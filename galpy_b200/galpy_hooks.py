"""Plug the engine into galpy's ``Orbit.integrate``.

After ``install()``, ``Orbit.integrate(ts, pot, method=m)`` accepts
``m`` any of galpy's C integrator names with ``_cuda`` for ``_c`` (leapfrog,
symplec4, symplec6, rk4, rk6, dopr54, dop853; not ias15) and runs the batch
on the GPU through this package; everything else in galpy is untouched.  The hooks patch the four places that decide galpy's integrator
dispatch (galpy/orbit/Orbits.py):

* ``Orbit.check_integrator`` (:1342-1370) -- the allow-list of method names
  (a ``*_cuda`` name is valid where galpy's ``*_c`` name is);
* ``Orbit._check_method_c_compatible`` (:1372-1392) -- ``"_c" in method`` is
  True for the ``*_cuda`` names; keep them when every potential component is
  one the engine implements, otherwise fall back to galpy's ``*_c`` method of
  the same integrator (and galpy's own fallback rules from there);
* ``Orbit._check_array_evenlyspaced`` (:1408-1416) -- ``dop853_cuda`` accepts
  unevenly spaced times like ``dop853_c``;
* the integration functions the dispatch at :1733-1826 calls
  (``integrateFullOrbit_c`` / ``integratePlanarOrbit_c`` and, when galpy's C
  extension is not loaded, ``integrateFullOrbit`` / ``integratePlanarOrbit``)
  -- a ``*_cuda`` method is routed to ``integrateFullOrbit_cuda`` /
  ``integratePlanarOrbit_cuda``, any other method to galpy's original;
* the same for ``Orbit.integrate_SOS`` (:2103-2278):
  ``integrateFullOrbit_sos_c`` / ``integrateFullOrbit_sos`` ->
  ``integrateFullOrbit_sos_cuda`` and ``integratePlanarOrbit_sos_c`` /
  ``integratePlanarOrbit_sos`` -> ``integratePlanarOrbit_sos_cuda``.

Beyond the dispatch they route ``Orbit.integrate_dxdv`` and ``Orbit.lyapunov``
(every orbit's deviations in one batched launch), the potential sums of
``Orbit.E`` / ``Orbit.Jacobi`` over many points, and ``Orbit._call_internal``
(``Orbit.__call__``, ``o.R(t)``, ... between integration times: the spline
interpolation on the GPU) -- each only where it applies, galpy's own code
otherwise.

The same routing can be written into galpy itself as a few-line patch of the
dispatch in ``Orbits._integrate_impl``; these hooks do it at run time.
"""
import numpy as np

from .integrate import (CUDA_METHODS, integrateFullOrbit_cuda, integrateFullOrbit_sos_cuda,
                        integratePlanarOrbit_cuda, integratePlanarOrbit_sos_cuda)
from .potentials import SUPPORTED_TYPES, T_SCF, T_SPIRALARMS, TIME_DEPENDENT_TYPES

_installed = {}


def _is_cuda(method):
    return isinstance(method, str) and method.lower() in CUDA_METHODS


def _supported(pot, planar, purpose="integrate"):
    """Whether the engine carries this potential for `purpose`: "integrate"
    (orbits, surfaces of section, variational runs) or "potential" (values
    at points, evaluated without a time: no time-dependent component and no
    planar disk perturbation, which the reference's C does not evaluate).
    An SCF expansion must have static coefficients."""
    try:
        if planar:
            from galpy.orbit.integratePlanarOrbit import _parse_pot
        else:
            from galpy.orbit.integrateFullOrbit import _parse_pot
        npot, pot_type, pot_args, tfuncs = _parse_pot(pot)
    except Exception:
        return False
    types = [int(t) for t in pot_type]
    if len(tfuncs) or not all(t in SUPPORTED_TYPES for t in types):
        return False
    if purpose == "potential" and any(t in TIME_DEPENDENT_TYPES for t in types):
        return False
    if T_SCF in types or T_SPIRALARMS in types or any(t < 0 for t in types):
        # time-dependent SCF coefficients, nested wrappers and spiral arms
        # with more than six terms are not carried
        from . import _lib

        pt = np.ascontiguousarray(types, np.int32)
        pa = np.ascontiguousarray(pot_args, np.float64)
        return _lib.lib().galpy_cuda_comp_records(
            int(planar), int(npot), pt.ctypes.data_as(_lib._ip), pa.ctypes.data_as(_lib._dp)) > 0
    return True


def _pad_phi(yo, full_dim):
    """galpy pads orbits without phi with phi = 0 before calling C."""
    if yo.shape[-1] in (3, 5):
        return np.pad(yo, ((0, 0), (0, 1)), "constant", constant_values=0), True
    return np.copy(yo), False


def _route_full(orig):
    def integrateFullOrbit_c(pot, yo, t, int_method, *args, **kwargs):
        if not _is_cuda(int_method):
            return orig(pot, yo, t, int_method, *args, **kwargs)
        kw = {k: kwargs[k] for k in ("rtol", "atol", "progressbar", "dt") if k in kwargs}
        return integrateFullOrbit_cuda(pot, np.copy(yo), t, int_method, **kw)

    return integrateFullOrbit_c


def _route_planar(orig):
    def integratePlanarOrbit_c(pot, yo, t, int_method, *args, **kwargs):
        if not _is_cuda(int_method):
            return orig(pot, yo, t, int_method, *args, **kwargs)
        kw = {k: kwargs[k] for k in ("rtol", "atol", "progressbar", "dt") if k in kwargs}
        return integratePlanarOrbit_cuda(pot, np.copy(yo), t, int_method, **kw)

    return integratePlanarOrbit_c


def _route_python(orig, planar):
    # galpy's pure-Python branch (taken when its C extension is not loaded)
    # receives vxvv without the phi padding the C branch adds.
    def integrate(pot, yo, t, int_method, *args, **kwargs):
        if not _is_cuda(int_method):
            return orig(pot, yo, t, int_method, *args, **kwargs)
        kw = {k: kwargs[k] for k in ("rtol", "atol", "progressbar", "dt") if k in kwargs}
        y, padded = _pad_phi(np.atleast_2d(yo), not planar)
        fn = integratePlanarOrbit_cuda if planar else integrateFullOrbit_cuda
        out, err = fn(pot, y, t, int_method, **kw)
        if out.ndim == 2:
            out = out[None]
        if padded:
            out = out[:, :, :-1]
        return out, err

    return integrate


def _route_sos(orig, python_branch):
    # Orbit.integrate_SOS (Orbits.py:2103-2278): the C branch pads orbits
    # without phi before the call (and drops the column after), the Python
    # branch (galpy's C extension not loaded) passes vxvv as it is
    def integrateFullOrbit_sos(pot, yo, psi, t0, int_method, *args, **kwargs):
        if not _is_cuda(int_method):
            return orig(pot, yo, psi, t0, int_method, *args, **kwargs)
        kw = {k: kwargs[k] for k in ("rtol", "atol", "progressbar", "dpsi") if k in kwargs}
        if python_branch:
            y, padded = _pad_phi(np.atleast_2d(yo), True)
        else:
            y, padded = np.copy(yo), False
        out, err = integrateFullOrbit_sos_cuda(pot, y, psi, t0, int_method, **kw)
        if python_branch and out.ndim == 2:
            out = out[None]
        if padded:
            out = np.delete(out, 5, axis=-1)
        return out, err

    return integrateFullOrbit_sos


def _route_sos_planar(orig, python_branch):
    # the planar counterpart (integratePlanarOrbit_sos_c / _sos); the C branch
    # pads orbits without phi, the Python branch does not
    def integratePlanarOrbit_sos(pot, yo, psi, t0, int_method, *args, **kwargs):
        if not _is_cuda(int_method):
            return orig(pot, yo, psi, t0, int_method, *args, **kwargs)
        kw = {k: kwargs[k] for k in ("surface", "rtol", "atol", "progressbar", "dpsi")
              if k in kwargs}
        if kw.get("surface") is None:
            kw.pop("surface", None)
        if python_branch:
            y = np.atleast_2d(yo)
            padded = y.shape[-1] == 3
            if padded:
                y = np.pad(y, ((0, 0), (0, 1)), "constant", constant_values=0)
        else:
            y, padded = np.copy(yo), False
        out, err = integratePlanarOrbit_sos_cuda(pot, y, psi, t0, int_method, **kw)
        if python_branch and out.ndim == 2:
            out = out[None]
        if padded:
            out = np.delete(out, 3, axis=-1)
        return out, err

    return integratePlanarOrbit_sos


def _cyl_to_rect_state(yo, planar):
    """galpy's rows (R, vR, vT[, z, vz], phi) -> (x, y[, z], vx, vy[, vz])."""
    R, vR, vT, phi = yo[:, 0], yo[:, 1], yo[:, 2], yo[:, -1]
    c, s = np.cos(phi), np.sin(phi)
    if planar:
        return np.stack([R * c, R * s, vR * c - vT * s, vR * s + vT * c], 1)
    return np.stack([R * c, R * s, yo[:, 3], vR * c - vT * s, vR * s + vT * c, yo[:, 4]], 1)


def _cyl_to_rect_dev(yo, dyo, planar):
    """Deviations (dR, dvR, dvT[, dz, dvz], dphi) at the rows yo -> the
    rectangular deviations, through the Jacobian of the cylindrical ->
    rectangular map (the conversion of galpy/orbit/integratePlanarOrbit.py:
    1463-1484 and integrateFullOrbit.py:935-944)."""
    R, vR, vT, phi = yo[:, 0], yo[:, 1], yo[:, 2], yo[:, -1]
    c, s = np.cos(phi), np.sin(phi)
    dR, dvR, dvT, dphi = dyo[:, 0], dyo[:, 1], dyo[:, 2], dyo[:, -1]
    dx = c * dR - R * s * dphi
    dy = s * dR + R * c * dphi
    dvx = c * dvR - s * dvT - (vR * s + vT * c) * dphi
    dvy = s * dvR + c * dvT + (vR * c - vT * s) * dphi
    if planar:
        return np.stack([dx, dy, dvx, dvy], 1)
    return np.stack([dx, dy, dyo[:, 3], dvx, dvy, dyo[:, 4]], 1)


def _rect_to_cyl_rows(out, planar):
    """Rectangular (x, v, dx, dv) rows in place -> galpy's cylindrical base
    state; returns (R, vR, vT, phi) for the deviation conversion.  The planar
    driver's angle is arccos(x/R) mapped to [0, 2 pi), the 3D one's atan2
    (the two galpy wrappers differ; both are kept)."""
    d = 2 if planar else 3
    x, y = out[..., 0], out[..., 1]
    vx, vy = out[..., d], out[..., d + 1]
    R = np.sqrt(x * x + y * y)
    if planar:
        phi = np.arccos(x / R)
        phi = np.where(y < 0.0, 2.0 * np.pi - phi, phi)
    else:
        phi = np.arctan2(y, x)
    c, s = np.cos(phi), np.sin(phi)
    vR = vx * c + vy * s
    vT = vy * c - vx * s
    if planar:
        out[..., 0], out[..., 1], out[..., 2], out[..., 3] = R, vR, vT, phi
    else:
        z, vz = np.copy(out[..., 2]), np.copy(out[..., 5])
        out[..., 0], out[..., 1], out[..., 2] = R, vR, vT
        out[..., 3], out[..., 4], out[..., 5] = z, vz, phi
    return R, vR, vT, phi, c, s


def _rect_to_cyl_dev(out, planar, R, vR, vT, c, s):
    """Rectangular deviations in out[..., 2*dim:] -> (dR, dvR, dvT[, dz,
    dvz], dphi), the inverse of the Jacobian above."""
    d = 2 if planar else 3
    k = 2 * d
    dx, dy = out[..., k], out[..., k + 1]
    dvx, dvy = out[..., k + d], out[..., k + d + 1]
    dR = c * dx + s * dy
    dphi = (c * dy - s * dx) / R
    dvR = c * dvx + s * dvy + vT * dphi
    dvT = c * dvy - s * dvx - vR * dphi
    if planar:
        out[..., k], out[..., k + 1], out[..., k + 2], out[..., k + 3] = dR, dvR, dvT, dphi
    else:
        dz, dvz = np.copy(out[..., k + 2]), np.copy(out[..., k + 5])
        out[..., k], out[..., k + 1], out[..., k + 2] = dR, dvR, dvT
        out[..., k + 3], out[..., k + 4], out[..., k + 5] = dz, dvz, dphi


def _route_dxdv(orig, planar):
    """galpy's integrate{Full,Planar}Orbit_dxdv (integrateFullOrbit.py:859,
    integratePlanarOrbit.py:1393) maps its single-orbit C integrator over the
    orbits in Python; for a *_cuda method all (orbit, deviation) pairs go to
    the GPU in one batched launch instead, with the same coordinate
    conversions around it."""
    def integrate_dxdv(pot, yo, dyo, t, int_method, rectIn, rectOut, *args, **kwargs):
        if not _is_cuda(int_method):
            return orig(pot, yo, dyo, t, int_method, rectIn, rectOut, *args, **kwargs)
        from .integrate import integrate_dxdv_batch

        yo = np.atleast_2d(np.asarray(yo, dtype=np.float64))
        dyo = np.atleast_2d(np.asarray(dyo, dtype=np.float64))
        w = _cyl_to_rect_state(yo, planar)
        dw = dyo if rectIn else _cyl_to_rect_dev(yo, dyo, planar)
        out, err = integrate_dxdv_batch(pot, np.hstack([w, dw]), np.asarray(t, np.float64),
                                        int_method, planar=planar, dt=kwargs.get("dt"),
                                        rtol=kwargs.get("rtol"), atol=kwargs.get("atol"))
        if np.any(err == -10):
            raise KeyboardInterrupt("Orbit integration interrupted by CTRL-C (SIGINT)")
        R, vR, vT, phi, c, s = _rect_to_cyl_rows(out, planar)
        if not rectOut:
            _rect_to_cyl_dev(out, planar, R, vR, vT, c, s)
        return out, err

    return integrate_dxdv


class _EngineAsC:
    """Inside integrate_dxdv / lyapunov with a *_cuda method, galpy decides
    between its C path and odeint from ``ext_loaded`` and ``_check_c``
    (Orbits.py:2418-2445, 2616-2634); this context lets that decision see
    the engine (it runs the potentials the check is about) and restores
    galpy's values afterwards."""

    def __init__(self, O):
        self.O = O

    def __enter__(self):
        self.saved = (self.O.ext_loaded, self.O._check_c)
        self.O.ext_loaded = True
        self.O._check_c = lambda *a, **k: True

    def __exit__(self, *exc):
        self.O.ext_loaded, self.O._check_c = self.saved
        return False


def _wrap_variational(orig, O):
    """Orbit.integrate_dxdv / Orbit.lyapunov: a *_cuda method with supported
    potentials runs galpy's own code with the engine taken as its C path
    (the dxdv mapper above does the integration); otherwise galpy's *_c
    method of the same integrator (and galpy's own fallbacks from there)."""
    import inspect

    sig = inspect.signature(orig)

    def wrapper(self, *args, **kwargs):
        ba = sig.bind(self, *args, **kwargs)
        ba.apply_defaults()
        method = ba.arguments.get("method")
        if not _is_cuda(method):
            return orig(self, *args, **kwargs)
        pot = ba.arguments.get("pot")
        if pot is None:
            pot = getattr(self, "_pot", None)
        planar = self.dim() == 2
        if pot is not None and _supported(O.toPlanarPotential(pot) if planar else pot, planar):
            with _EngineAsC(O):
                return orig(*ba.args, **ba.kwargs)
        ba.arguments["method"] = method[: -len("_cuda")] + "_c"
        return orig(*ba.args, **ba.kwargs)

    wrapper.__doc__ = orig.__doc__
    wrapper.__name__ = orig.__name__
    return wrapper


# Smallest number of points for which the potential sums of Orbit.E /
# Orbit.Jacobi go to the GPU (below it the launch latency dominates).
DEVICE_POTENTIAL_MIN_POINTS = 4096


def _route_potential_sum(orig, planar):
    """evaluatePotentials / evaluateplanarPotentials as Orbit.E (Orbits.py:
    2902) and Orbit.Jacobi (:3298, through E) call them: plain potential
    values of a supported static potential at many points run on the GPU
    (galpy_cuda_energy_device with zero velocities); anything else -- a
    derivative, a time-dependent or unsupported potential, physical output,
    a few points -- goes to galpy's own function."""
    def evaluate(pot, R, *args, **kwargs):
        plain = (not args[1:] if planar else len(args) <= 1) and not any(
            kwargs.get(k) for k in ("dR", "dphi", "use_physical")) and set(kwargs) <= {
            "phi", "t", "dR", "dphi", "use_physical", "z"}
        if not plain or np.size(R) < DEVICE_POTENTIAL_MIN_POINTS:
            return orig(pot, R, *args, **kwargs)
        try:
            if not _supported(pot, planar, "potential"):
                return orig(pot, R, *args, **kwargs)
        except Exception:
            return orig(pot, R, *args, **kwargs)
        from .orbit_quantities import potential_values

        z = 0.0 if planar else (args[0] if args else kwargs.get("z", 0.0))
        phi = kwargs.get("phi", args[0] if planar and args else 0.0)
        return potential_values(pot, R, z, phi, planar=planar)

    return evaluate


# Orbit.__call__ between integration times: at least this many (orbit,
# time) pairs are interpolated on the GPU
DEVICE_INTERP_MIN_POINTS = 4096


def _wrap_call_internal(orig):
    """Orbit._call_internal (Orbits.py:6460-6575), behind Orbit.__call__
    and the coordinate methods (o.R(t), o.x(t), ...): at times that are not
    the integration times of an Orbit integrated on one shared time grid,
    galpy fits scipy splines to every orbit (_setupOrbitInterp, :6739) and
    evaluates them in Python; here the same interpolants (not-a-knot cubics
    of x, y and the other components per orbit) are built and evaluated on
    the GPU (galpy_cuda_orbit_interp_device) for at least
    DEVICE_INTERP_MIN_POINTS (orbit, time) pairs of a 4- or 6-D orbit.
    Everything else -- the integration times themselves, per-orbit time
    grids, times outside the integrated range (galpy raises), quantities,
    small requests -- is galpy's own."""
    def _call_internal(self, *args, **kwargs):
        if len(args) != 1 or kwargs or not hasattr(self, "t") or np.ndim(self.t) != 1:
            return orig(self, *args, **kwargs)
        t = args[0]
        if hasattr(t, "unit") or np.ndim(t) != 1 or self.phasedim() not in (4, 6) or \
                self.__dict__.get("_integrate_t_asQuantity"):
            return orig(self, *args, **kwargs)
        tq = np.asarray(t, dtype=np.float64)
        self_t = np.asarray(self.t, dtype=np.float64)
        if (tq.size * self.size < DEVICE_INTERP_MIN_POINTS or np.isnan(self_t).any()
                or (tq.size == self_t.size and np.all(tq == self_t))
                or np.any(tq > self_t.max()) or np.any(tq < self_t.min())
                or self_t.size < 2):
            return orig(self, *args, **kwargs)
        from .orbit_quantities import interpolate

        out = interpolate(self.orbit, self_t, tq).transpose(2, 1, 0)  # [phasedim, nq, N]
        return out[:, 0] if tq.size == 1 else out

    return _call_internal


def install():
    """Patch galpy (must be importable) so that Orbit.integrate accepts the
    ``*_cuda`` methods.  Idempotent."""
    if _installed:
        return
    import galpy.orbit.Orbits as O

    Orbit = O.Orbit
    orig_check = Orbit.check_integrator
    orig_c_compat = Orbit._check_method_c_compatible
    orig_even = Orbit._check_array_evenlyspaced

    def check_integrator(method, no_symplec=False, allow_c_symplec=False):
        if not _is_cuda(method):
            return orig_check(method, no_symplec=no_symplec, allow_c_symplec=allow_c_symplec)
        # valid wherever galpy's *_c method of the same name is
        try:
            return orig_check(method[: -len("_cuda")] + "_c", no_symplec=no_symplec,
                              allow_c_symplec=allow_c_symplec)
        except ValueError:
            raise ValueError(f"{method:s} is not a valid `method`") from None

    def _check_method_c_compatible(method, pot):
        if _is_cuda(method):
            planar = getattr(pot, "dim", None) == 2 or (
                isinstance(pot, list) and len(pot) and getattr(pot[0], "dim", 3) == 2)
            if _supported(pot, planar):
                return method
            method = method[: -len("_cuda")] + "_c"
        return orig_c_compat(method, pot)

    def _check_array_evenlyspaced(t, method):
        if isinstance(method, str) and method.lower() == "dop853_cuda":
            return True
        return orig_even(t, method)

    _installed.update(
        check_integrator=orig_check, _check_method_c_compatible=orig_c_compat,
        _check_array_evenlyspaced=orig_even, integrateFullOrbit_c=O.integrateFullOrbit_c,
        integratePlanarOrbit_c=O.integratePlanarOrbit_c,
        integrateFullOrbit=O.integrateFullOrbit, integratePlanarOrbit=O.integratePlanarOrbit,
        integrateFullOrbit_sos_c=O.integrateFullOrbit_sos_c,
        integrateFullOrbit_sos=O.integrateFullOrbit_sos,
        integratePlanarOrbit_sos_c=O.integratePlanarOrbit_sos_c,
        integratePlanarOrbit_sos=O.integratePlanarOrbit_sos)
    Orbit.check_integrator = staticmethod(check_integrator)
    Orbit._check_method_c_compatible = staticmethod(_check_method_c_compatible)
    Orbit._check_array_evenlyspaced = staticmethod(_check_array_evenlyspaced)
    O.integrateFullOrbit_c = _route_full(_installed["integrateFullOrbit_c"])
    O.integratePlanarOrbit_c = _route_planar(_installed["integratePlanarOrbit_c"])
    O.integrateFullOrbit = _route_python(_installed["integrateFullOrbit"], False)
    O.integratePlanarOrbit = _route_python(_installed["integratePlanarOrbit"], True)
    O.integrateFullOrbit_sos_c = _route_sos(_installed["integrateFullOrbit_sos_c"], False)
    O.integrateFullOrbit_sos = _route_sos(_installed["integrateFullOrbit_sos"], True)
    O.integratePlanarOrbit_sos_c = _route_sos_planar(_installed["integratePlanarOrbit_sos_c"],
                                                     False)
    O.integratePlanarOrbit_sos = _route_sos_planar(_installed["integratePlanarOrbit_sos"], True)
    # variational integration (integrate_dxdv, lyapunov) and the potential
    # sums of Orbit.E / Orbit.Jacobi
    _installed.update(
        integrate_dxdv=Orbit.integrate_dxdv, lyapunov=Orbit.lyapunov,
        integrateFullOrbit_dxdv=O.integrateFullOrbit_dxdv,
        integratePlanarOrbit_dxdv=O.integratePlanarOrbit_dxdv,
        evaluatePotentials=O.evaluatePotentials,
        evaluateplanarPotentials=O.evaluateplanarPotentials)
    Orbit.integrate_dxdv = _wrap_variational(_installed["integrate_dxdv"], O)
    Orbit.lyapunov = _wrap_variational(_installed["lyapunov"], O)
    O.integrateFullOrbit_dxdv = _route_dxdv(_installed["integrateFullOrbit_dxdv"], False)
    O.integratePlanarOrbit_dxdv = _route_dxdv(_installed["integratePlanarOrbit_dxdv"], True)
    O.evaluatePotentials = _route_potential_sum(_installed["evaluatePotentials"], False)
    O.evaluateplanarPotentials = _route_potential_sum(_installed["evaluateplanarPotentials"],
                                                      True)
    # interpolation between integration times (Orbit.__call__ and friends)
    _installed.update(_call_internal=Orbit._call_internal)
    Orbit._call_internal = _wrap_call_internal(_installed["_call_internal"])


def uninstall():
    """Restore galpy's original functions."""
    if not _installed:
        return
    import galpy.orbit.Orbits as O

    Orbit = O.Orbit
    Orbit.check_integrator = staticmethod(_installed["check_integrator"])
    Orbit._check_method_c_compatible = staticmethod(_installed["_check_method_c_compatible"])
    Orbit._check_array_evenlyspaced = staticmethod(_installed["_check_array_evenlyspaced"])
    Orbit.integrate_dxdv = _installed["integrate_dxdv"]
    Orbit.lyapunov = _installed["lyapunov"]
    Orbit._call_internal = _installed["_call_internal"]
    for name in ("integrateFullOrbit_c", "integratePlanarOrbit_c", "integrateFullOrbit",
                 "integratePlanarOrbit", "integrateFullOrbit_sos_c", "integrateFullOrbit_sos",
                 "integratePlanarOrbit_sos_c", "integratePlanarOrbit_sos",
                 "integrateFullOrbit_dxdv", "integratePlanarOrbit_dxdv", "evaluatePotentials",
                 "evaluateplanarPotentials"):
        setattr(O, name, _installed[name])
    _installed.clear()
