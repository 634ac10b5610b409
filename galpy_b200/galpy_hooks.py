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

The same routing can be written into galpy itself as a few-line patch of the
dispatch in ``Orbits._integrate_impl``; these hooks do it at run time.
"""
import numpy as np

from .integrate import (CUDA_METHODS, integrateFullOrbit_cuda, integrateFullOrbit_sos_cuda,
                        integratePlanarOrbit_cuda, integratePlanarOrbit_sos_cuda)
from .potentials import SUPPORTED_TYPES

_installed = {}


def _is_cuda(method):
    return isinstance(method, str) and method.lower() in CUDA_METHODS


def _supported(pot, planar):
    try:
        if planar:
            from galpy.orbit.integratePlanarOrbit import _parse_pot
        else:
            from galpy.orbit.integrateFullOrbit import _parse_pot
        npot, pot_type, _, tfuncs = _parse_pot(pot)
    except Exception:
        return False
    return len(tfuncs) == 0 and all(int(t) in SUPPORTED_TYPES for t in pot_type)


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


def uninstall():
    """Restore galpy's original functions."""
    if not _installed:
        return
    import galpy.orbit.Orbits as O

    Orbit = O.Orbit
    Orbit.check_integrator = staticmethod(_installed["check_integrator"])
    Orbit._check_method_c_compatible = staticmethod(_installed["_check_method_c_compatible"])
    Orbit._check_array_evenlyspaced = staticmethod(_installed["_check_array_evenlyspaced"])
    for name in ("integrateFullOrbit_c", "integratePlanarOrbit_c", "integrateFullOrbit",
                 "integratePlanarOrbit", "integrateFullOrbit_sos_c", "integrateFullOrbit_sos",
                 "integratePlanarOrbit_sos_c", "integratePlanarOrbit_sos"):
        setattr(O, name, _installed[name])
    _installed.clear()
