"""oracle/oracle.py -- TEST INFRASTRUCTURE ONLY.

ctypes front end of the two CPU checkers:

* ``liboracle.so``          -- this project's C restatement of galpy's batched
  orbit integration (oracle/galpy_oracle.c), and
* ``_ref/libgalpy_ref.so``  -- the reference's own C sources
  (galpy/orbit/orbit_c_ext/integrate{Full,Planar}Orbit.c and the steppers
  and force files they call) built by ``make ref``; present only where the
  reference tree was available at build time.

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  Nothing in the galpy_b200 package may.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(_HERE, "liboracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libgalpy_ref.so")

DT_SENTINEL = -9999.99
METHODS = {"leapfrog": 0, "rk4": 1, "rk6": 2, "symplec4": 3, "symplec6": 4, "dopr54": 5,
           "dop853": 6}

_port = None
_ref = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_longlong)


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def reference_tree():
    """The reference checkout the oracle's recipe reads (its REF: the
    GALPY_REFERENCE_TREE environment variable, else the recipe's default);
    it need not exist."""
    import subprocess

    r = subprocess.run(["make", "-s", "-C", _HERE, "print-ref"], stdout=subprocess.PIPE,
                       text=True, check=True)
    return r.stdout.strip()


def build(ref=False):
    """Compile the oracle (and, if asked and the reference is present, _ref)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    tree = reference_tree()
    if ref and os.path.isdir(os.path.join(tree, "galpy")):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", "REF=" + tree], check=True)


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            build()
        lib = ctypes.CDLL(PORT_SO)
        lib.oracle_integrate.restype = ctypes.c_int
        lib.oracle_integrate.argtypes = [
            ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
            _ip, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _ip,
            ctypes.c_int, _lp, _lp, ctypes.c_longlong, ctypes.c_int,
        ]
        lib.oracle_integrate_dxdv.restype = ctypes.c_int
        lib.oracle_integrate_dxdv.argtypes = [
            ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
            _ip, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _ip,
            ctypes.c_int, _lp, ctypes.c_int,
        ]
        lib.oracle_integrate_sos.restype = ctypes.c_int
        lib.oracle_integrate_sos.argtypes = [
            ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, _ip, _dp,
            ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _ip, ctypes.c_int, _lp,
            ctypes.c_int,
        ]
        lib.oracle_integrate_sos_planar.restype = ctypes.c_int
        lib.oracle_integrate_sos_planar.argtypes = [
            ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip,
            _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _ip, ctypes.c_int, _lp,
            ctypes.c_int,
        ]
        lib.oracle_forces.restype = ctypes.c_int
        lib.oracle_forces.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int,
                                      _ip, _dp, _dp, ctypes.c_double]
        lib.oracle_potential.restype = ctypes.c_int
        lib.oracle_potential.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _ip, _dp, _dp]
        lib.oracle_expint.restype = ctypes.c_double
        lib.oracle_expint.argtypes = [ctypes.c_double]
        lib.oracle_set_phi_mode.restype = None
        lib.oracle_set_phi_mode.argtypes = [ctypes.c_int]
        lib.oracle_gammainc_P.restype = ctypes.c_double
        lib.oracle_gammainc_P.argtypes = [ctypes.c_double, ctypes.c_double]
        _port = lib
    return _port


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    """The reference's own C build, or None when it was not built here."""
    global _ref
    if _ref is None and ref_available():
        _ref = ctypes.CDLL(REF_SO)
    return _ref


def _tol(rtol, atol):
    # galpy passes natural logs of the tolerances, default 1e-12
    # (galpy/orbit/integratePlanarOrbit.py:712-723)
    r = -12.0 * np.log(10.0) if rtol is None else np.log(rtol)
    a = -12.0 * np.log(10.0) if atol is None else np.log(atol)
    return float(r), float(a)


# npot (every function below): galpy's count of top-level potential entries,
# which differs from len(pot_type) when a wrapper (negative type) carries
# wrapped components; default len(pot_type).
def _prep(yo, t, pot_type, pot_args):
    yo = np.array(yo, dtype=np.float64, order="C", copy=True)
    t = np.ascontiguousarray(t, dtype=np.float64)
    pt = np.ascontiguousarray(pot_type, dtype=np.int32)
    pa = np.ascontiguousarray(pot_args, dtype=np.float64)
    return yo, t, pt, pa


def integrate(yo, t, pot_type, pot_args, method, planar=False, dt=None, rtol=None, atol=None,
              nthreads=0, max_attempts=0, impl="port", npot=None):
    """Integrate nobj orbits with galpy's conventions.

    yo: (nobj, 6) cylindrical (R,vR,vT,z,vz,phi), or (nobj, 4) (R,vR,vT,phi)
    when planar.  t: (nt,) or (nobj, nt).  Returns (result, err, nsteps,
    nforce); result is (nobj, nt, 6|4) cylindrical.  nsteps/nforce are None
    for impl="ref" (the reference does not count them)."""
    yo, t, pt, pa = _prep(yo, t, pot_type, pot_args)
    nobj, nv = yo.shape
    nt = t.shape[-1]
    indiv_t = int(t.ndim > 1)
    r, a = _tol(rtol, atol)
    dtv = DT_SENTINEL if dt is None else float(dt)
    m = METHODS[method] if isinstance(method, str) else int(method)
    result = np.empty((nobj, nt, nv))
    err = np.zeros(nobj, dtype=np.int32)
    if impl == "port":
        nsteps = np.zeros(nobj, dtype=np.int64)
        nforce = np.zeros(nobj, dtype=np.int64)
        rc = port().oracle_integrate(
            int(planar), nobj, _ptr(yo, _dp), nt, _ptr(t, _dp), indiv_t, (len(pt) if npot is None else int(npot)), _ptr(pt, _ip),
            _ptr(pa, _dp), dtv, r, a, _ptr(result, _dp), _ptr(err, _ip), m, _ptr(nsteps, _lp),
            _ptr(nforce, _lp), int(max_attempts), int(nthreads))
        if rc != 0:
            raise ValueError(f"oracle_integrate returned {rc}")
        return result, err, nsteps, nforce
    lib = ref()
    if lib is None:
        raise RuntimeError("reference build oracle/_ref/libgalpy_ref.so is not present")
    fn = lib.integratePlanarOrbit if planar else lib.integrateFullOrbit
    fn.restype = None
    fn.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, _ip, _dp,
                   ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _ip,
                   ctypes.c_int, ctypes.c_void_p]
    if nthreads:
        os.environ["OMP_NUM_THREADS"] = str(nthreads)
    fn(nobj, _ptr(yo, _dp), nt, _ptr(t, _dp), indiv_t, (len(pt) if npot is None else int(npot)), _ptr(pt, _ip), _ptr(pa, _dp),
       None, dtv, r, a, _ptr(result, _dp), _ptr(err, _ip), m, None)
    return result, err, None, None


def integrate_dxdv(w, t, pot_type, pot_args, method, planar=False, dt=None, rtol=None,
                   atol=None, nthreads=0, impl="port", npot=None):
    """Variational integration, rectangular in and out.

    w: (nobj, 4*dim) = (x, v, dx, dv) per orbit; returns (result (nobj, nt,
    4*dim), err, nsteps).  impl="ref" calls the reference's single-orbit
    integrate{Full,Planar}Orbit_dxdv once per orbit."""
    w, t, pt, pa = _prep(w, t, pot_type, pot_args)
    nobj, nv = w.shape
    nt = t.shape[-1]
    indiv_t = int(t.ndim > 1)
    r, a = _tol(rtol, atol)
    dtv = DT_SENTINEL if dt is None else float(dt)
    m = METHODS[method] if isinstance(method, str) else int(method)
    result = np.empty((nobj, nt, nv))
    err = np.zeros(nobj, dtype=np.int32)
    if impl == "port":
        nsteps = np.zeros(nobj, dtype=np.int64)
        rc = port().oracle_integrate_dxdv(
            int(planar), nobj, _ptr(w, _dp), nt, _ptr(t, _dp), indiv_t, (len(pt) if npot is None else int(npot)), _ptr(pt, _ip),
            _ptr(pa, _dp), dtv, r, a, _ptr(result, _dp), _ptr(err, _ip), m, _ptr(nsteps, _lp),
            int(nthreads))
        if rc != 0:
            raise ValueError(f"oracle_integrate_dxdv returned {rc}")
        return result, err, nsteps
    lib = ref()
    if lib is None:
        raise RuntimeError("reference build oracle/_ref/libgalpy_ref.so is not present")
    if planar:
        fn = lib.integratePlanarOrbit_dxdv
        fn.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_int, _ip, _dp, ctypes.c_void_p,
                       ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _ip, ctypes.c_int,
                       ctypes.c_void_p]
    else:
        fn = lib.integrateFullOrbit_dxdv
        fn.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_int, _ip, _dp, ctypes.c_void_p,
                       ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _ip, ctypes.c_int]
    fn.restype = None
    for i in range(nobj):
        wi = np.ascontiguousarray(w[i])
        ti = np.ascontiguousarray(t[i] if indiv_t else t)
        res = np.empty((nt, nv))
        e = np.zeros(1, dtype=np.int32)
        args = [_ptr(wi, _dp), nt, _ptr(ti, _dp), (len(pt) if npot is None else int(npot)), _ptr(pt, _ip), _ptr(pa, _dp), None,
                dtv, r, a, _ptr(res, _dp), _ptr(e, _ip), m]
        if planar:
            args.append(None)
        fn(*args)
        result[i] = res
        err[i] = e[0]
    return result, err, None


def integrate_sos(yo, psi, pot_type, pot_args, method, dpsi=None, rtol=None, atol=None,
                  nthreads=0, impl="port", planar=False, surface=0, npot=None):
    """Surface-of-section integration (integrateFullOrbit_sos, or
    integratePlanarOrbit_sos when planar with surface 0 (x = 0) or 1 (y = 0)).

    yo: (nobj, 7) = (R, vR, vT, z, vz, phi, t0), planar (nobj, 5) = (R, vR,
    vT, phi, t0); psi: (npsi,) or (nobj, npsi) angle increments.  Returns
    (result (nobj, npsi, 7 | 5) in the input's coordinates with the time
    last, err, nsteps); nsteps is None for impl="ref"."""
    yo, psi, pt, pa = _prep(yo, psi, pot_type, pot_args)
    nobj, nv = yo.shape
    npsi = psi.shape[-1]
    indiv = int(psi.ndim > 1)
    r, a = _tol(rtol, atol)
    dv = DT_SENTINEL if dpsi is None else float(dpsi)
    m = METHODS[method] if isinstance(method, str) else int(method)
    result = np.empty((nobj, npsi, nv))
    err = np.zeros(nobj, dtype=np.int32)
    if impl == "port":
        nsteps = np.zeros(nobj, dtype=np.int64)
        if planar:
            rc = port().oracle_integrate_sos_planar(
                nobj, _ptr(yo, _dp), npsi, _ptr(psi, _dp), indiv, int(surface), (len(pt) if npot is None else int(npot)),
                _ptr(pt, _ip), _ptr(pa, _dp), dv, r, a, _ptr(result, _dp), _ptr(err, _ip), m,
                _ptr(nsteps, _lp), int(nthreads))
        else:
            rc = port().oracle_integrate_sos(nobj, _ptr(yo, _dp), npsi, _ptr(psi, _dp), indiv,
                                             (len(pt) if npot is None else int(npot)), _ptr(pt, _ip), _ptr(pa, _dp), dv, r, a,
                                             _ptr(result, _dp), _ptr(err, _ip), m,
                                             _ptr(nsteps, _lp), int(nthreads))
        if rc != 0:
            raise ValueError(f"oracle_integrate_sos returned {rc}")
        return result, err, nsteps
    lib = ref()
    if lib is None:
        raise RuntimeError("reference build oracle/_ref/libgalpy_ref.so is not present")
    if nthreads:
        os.environ["OMP_NUM_THREADS"] = str(nthreads)
    if planar:
        fn = lib.integratePlanarOrbit_sos
        fn.restype = None
        fn.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                       ctypes.c_int, _ip, _dp, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                       ctypes.c_double, _dp, _ip, ctypes.c_int, ctypes.c_void_p]
        fn(nobj, _ptr(yo, _dp), npsi, _ptr(psi, _dp), indiv, int(surface), (len(pt) if npot is None else int(npot)),
           _ptr(pt, _ip), _ptr(pa, _dp), None, dv, r, a, _ptr(result, _dp), _ptr(err, _ip), m,
           None)
        return result, err, None
    fn = lib.integrateFullOrbit_sos
    fn.restype = None
    fn.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, _ip, _dp,
                   ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _ip,
                   ctypes.c_int, ctypes.c_void_p]
    fn(nobj, _ptr(yo, _dp), npsi, _ptr(psi, _dp), indiv, (len(pt) if npot is None else int(npot)), _ptr(pt, _ip), _ptr(pa, _dp),
       None, dv, r, a, _ptr(result, _dp), _ptr(err, _ip), m, None)
    return result, err, None


def forces(R, z, phi, pot_type, pot_args, planar=False, t=0.0, npot=None):
    """Per-point (Rforce, zforce, phitorque, R2, z2, Rz, phi2, Rphi, zphi)
    (3D) or (Rforce, phitorque, R2, phi2, Rphi) (planar), at time t."""
    R = np.ascontiguousarray(R, dtype=np.float64)
    z = np.ascontiguousarray(np.broadcast_to(z, R.shape), dtype=np.float64)
    phi = np.ascontiguousarray(np.broadcast_to(phi, R.shape), dtype=np.float64)
    pt = np.ascontiguousarray(pot_type, dtype=np.int32)
    pa = np.ascontiguousarray(pot_args, dtype=np.float64)
    out = np.empty((R.size, 5 if planar else 9))
    rc = port().oracle_forces(int(planar), R.size, _ptr(R, _dp), _ptr(z, _dp), _ptr(phi, _dp),
                              (len(pt) if npot is None else int(npot)), _ptr(pt, _ip), _ptr(pa, _dp), _ptr(out, _dp), float(t))
    if rc:
        raise ValueError(f"oracle_forces returned {rc}")
    return out


def potential(R, z, phi, pot_type, pot_args, npot=None):
    R = np.ascontiguousarray(R, dtype=np.float64)
    z = np.ascontiguousarray(np.broadcast_to(z, R.shape), dtype=np.float64)
    phi = np.ascontiguousarray(np.broadcast_to(phi, R.shape), dtype=np.float64)
    pt = np.ascontiguousarray(pot_type, dtype=np.int32)
    pa = np.ascontiguousarray(pot_args, dtype=np.float64)
    out = np.empty(R.size)
    rc = port().oracle_potential(R.size, _ptr(R, _dp), _ptr(z, _dp), _ptr(phi, _dp), (len(pt) if npot is None else int(npot)),
                                 _ptr(pt, _ip), _ptr(pa, _dp), _ptr(out, _dp))
    if rc:
        raise ValueError(f"oracle_potential returned {rc}")
    return out


class phi_from_atan2:
    """Within the block the oracle's Cartesian force routes take the angle
    from atan2(y, x) instead of the reference's acos(x / R), which is
    ill-conditioned near the x axis (galpy_oracle.c, cyl_of).  Used by tests
    to separate that reference-side rounding from the engine's (whose forces
    are Cartesian)."""

    def __enter__(self):
        port().oracle_set_phi_mode(1)

    def __exit__(self, *exc):
        port().oracle_set_phi_mode(0)
        return False


def gammainc_P(a, x):
    return port().oracle_gammainc_P(float(a), float(x))


def expint_E1(x):
    return port().oracle_expint(float(x))


def energy_cyl(res, pot_type, pot_args):
    """E = v^2/2 + Phi for cylindrical rows (..., 6)."""
    R, vR, vT, z, vz, phi = (res[..., k] for k in range(6))
    pot = potential(R.ravel(), z.ravel(), phi.ravel(), pot_type, pot_args).reshape(R.shape)
    return 0.5 * (vR**2 + vT**2 + vz**2) + pot
