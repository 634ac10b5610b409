"""galpy-facing integration entry points.

Each function mirrors the galpy wrapper it stands in for -- same arguments,
same array shapes, same error behaviour -- and calls libgalpy_cuda.so through
ctypes exactly like galpy calls libgalpy:

  integrateFullOrbit_cuda         galpy/orbit/integrateFullOrbit.py:616-749
  integratePlanarOrbit_cuda       galpy/orbit/integratePlanarOrbit.py:989
  integrateFullOrbit_dxdv_cuda    galpy/orbit/integrateFullOrbit.py:752-856
  integratePlanarOrbit_dxdv_cuda  galpy/orbit/integratePlanarOrbit.py:1124-1225
  integrateFullOrbit_sos_cuda     galpy/orbit/integrateFullOrbit.py:1215-1355
  integratePlanarOrbit_sos_cuda   galpy/orbit/integratePlanarOrbit.py:1543-1693

plus ``integrate_dxdv_batch`` (all deviations of many orbits in one launch)
and ``integrate_device`` (device-resident torch tensors, asynchronous).
"""
import ctypes

import numpy as np

from . import _lib
from .potentials import parse_pot

# galpy's odeint codes (galpy/orbit/integratePlanarOrbit.py:690-709)
_ALIASES = {"leapfrog": 0, "rk4": 1, "rk6": 2, "symplec4": 3, "symplec6": 4, "dopr54": 5,
            "dop853": 6}
CUDA_METHODS = {f"{name}_cuda": code for name, code in _ALIASES.items()}
# precision forms (include/galpy_cuda.h): float64; float32 force with
# float64 state; float64 force with float32 tails of its table polynomials;
# that with the bulge term in float32; float32 force with a double-float
# state (the last three for MWPotential2014-type potentials)
PRECISIONS = {"fp64": _lib.FP64, "f32force": _lib.F32FORCE, "f64tail32": 2, "f32bulge": 3,
              "f32force_df": 4}
# the ODE system of a device launch: orbits, or surface-of-section states
# (3D rows (x, y, vx, vy, A, t, psi); planar rows (u, vu, A, t, psi) for the
# surface x = 0 or y = 0)
SYSTEMS = {"orbit": _lib.SYS_ORBIT, "sos": _lib.SYS_SOS, "sos_planar_x": _lib.SYS_SOS_PLANAR_X,
           "sos_planar_y": _lib.SYS_SOS_PLANAR_Y}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def parse_integrator(int_method):
    """galpy odeint code of a method name.  Unlike galpy's _parse_integrator
    (which maps unknown names to leapfrog), unknown names raise."""
    m = int_method.lower()
    if m in CUDA_METHODS:
        return CUDA_METHODS[m]
    for suffix in ("_cuda", "_c"):
        if m.endswith(suffix) and m[: -len(suffix)] in _ALIASES:
            return _ALIASES[m[: -len(suffix)]]
    if m in _ALIASES:
        return _ALIASES[m]
    raise ValueError(f"{int_method} is not a method of the CUDA engine")


def parse_tol(rtol, atol):
    """natural logs, default 1e-12 (galpy/orbit/integratePlanarOrbit.py:712-723)."""
    r = -12.0 * np.log(10.0) if rtol is None else np.log(rtol)
    a = -12.0 * np.log(10.0) if atol is None else np.log(atol)
    return float(r), float(a)


def _precision(p):
    if isinstance(p, int):
        return p
    return PRECISIONS[p.lower()]


def _integrate_c(planar, pot, yo, t, int_method, rtol, atol, progressbar, dt, precision,
                 max_attempts, return_nsteps, device, stream_rows=-1, devices=None):
    single_obj = yo.ndim == 1
    yo = np.atleast_2d(yo)
    nobj = len(yo)
    nv = 4 if planar else 6
    rtol, atol = parse_tol(rtol, atol)
    npot, pot_type, pot_args = parse_pot(pot, planar=planar)
    code = parse_integrator(int_method)
    dt = _lib.DT_SENTINEL if dt is None else float(dt)
    t = np.asarray(t)
    indiv_t = int(t.ndim > 1)
    nt = t.shape[-1]
    result = np.empty((nobj, nt, nv))
    err = np.zeros(nobj, dtype=np.int32)
    nsteps = np.zeros(nobj, dtype=np.int64) if return_nsteps else None
    yo = np.require(yo, dtype=np.float64, requirements=["C", "W"])
    t = np.require(t, dtype=np.float64, requirements=["C", "W"])
    opts = _lib.make_opts(precision=_precision(precision), device=device,
                          max_attempts=max_attempts, nsteps=nsteps, stream_rows=stream_rows,
                          devices=devices)
    cb = _lib.CALLBACK()
    pbar = None
    if progressbar and nobj > 1:
        try:
            import tqdm

            pbar = tqdm.tqdm(total=nobj, leave=False)
            cb = _lib.CALLBACK(pbar.update)
        except ImportError:  # pragma: no cover
            pass
    fn = _lib.lib().integratePlanarOrbit_cuda if planar else _lib.lib().integrateFullOrbit_cuda
    rc = fn(nobj, yo.ctypes.data_as(_dp), nt, t.ctypes.data_as(_dp), indiv_t, npot,
            pot_type.ctypes.data_as(_ip), pot_args.ctypes.data_as(_dp), None, dt, rtol, atol,
            result.ctypes.data_as(_dp), err.ctypes.data_as(_ip), code, cb, ctypes.byref(opts))
    if pbar is not None:
        pbar.close()
    _lib.check(rc)
    if np.any(err == -10):  # same behaviour as galpy (integrateFullOrbit.py:737-738)
        raise KeyboardInterrupt("Orbit integration interrupted by CTRL-C (SIGINT)")
    out = (result[0], err[0]) if single_obj else (result, err)
    if return_nsteps:
        out = out + ((nsteps[0] if single_obj else nsteps),)
    return out


def integrateFullOrbit_cuda(pot, yo, t, int_method, rtol=None, atol=None, progressbar=True,
                            dt=None, precision="fp64", max_attempts=0, return_nsteps=False,
                            device=-1, stream_rows=-1, devices=None):
    """Integrate 3D orbits on the GPU.

    Parameters mirror galpy's integrateFullOrbit_c: yo [N,6] or [6]
    cylindrical (R,vR,vT,z,vz,phi) -- overwritten in place with rectangular
    coordinates when it is a C-contiguous float64 array, as in galpy; t [nt]
    or [N,nt]; int_method one of 'leapfrog_cuda', 'rk4_cuda', 'rk6_cuda',
    'symplec4_cuda', 'symplec6_cuda', 'dopr54_cuda', 'dop853_cuda'.  Extra
    keywords: precision (a key of PRECISIONS), max_attempts (per-orbit
    step-attempt budget, 0 = none), return_nsteps, stream_rows (the result
    transfer: -1 automatic, 0 one copy after the kernel, 1 the rows of
    finished orbits copied while the kernel runs), devices (None: the one
    device `device`; a sequence of ordinals, or -1 for every visible device:
    the orbits are cut into contiguous ranges of equal estimated cost, one
    per device, integrated concurrently).

    Returns (result [N,nt,6] cylindrical, err [N]) like galpy (the leading
    axis is dropped for a single orbit), plus per-orbit accepted steps when
    return_nsteps."""
    return _integrate_c(False, pot, yo, t, int_method, rtol, atol, progressbar, dt, precision,
                        max_attempts, return_nsteps, device, stream_rows, devices)


def integratePlanarOrbit_cuda(pot, yo, t, int_method, rtol=None, atol=None, progressbar=True,
                              dt=None, precision="fp64", max_attempts=0, return_nsteps=False,
                              device=-1, stream_rows=-1, devices=None):
    """Planar counterpart of integrateFullOrbit_cuda: yo [N,4] (R,vR,vT,phi)."""
    return _integrate_c(True, pot, yo, t, int_method, rtol, atol, progressbar, dt, precision,
                        max_attempts, return_nsteps, device, stream_rows, devices)


def _integrate_sos(planar, pot, yo, psi, t0, int_method, surface, rtol, atol, progressbar,
                   dpsi, max_attempts, return_nsteps, device, devices=None):
    single_obj = np.ndim(yo) == 1
    yo = np.atleast_2d(yo)
    nobj = len(yo)
    nv = 5 if planar else 7
    rtol, atol = parse_tol(rtol, atol)
    npot, pot_type, pot_args = parse_pot(pot, planar=planar)
    code = parse_integrator(int_method)
    dpsi = _lib.DT_SENTINEL if dpsi is None else float(dpsi)
    t0 = np.atleast_1d(np.asarray(t0, dtype=np.float64))
    yoo = np.empty((nobj, nv))
    yoo[:, :nv - 1] = yo[:, :nv - 1]
    yoo[:, nv - 1] = t0[0] if len(t0) == 1 else t0
    psi = np.require(np.asarray(psi, dtype=np.float64), requirements=["C", "W"])
    indiv = int(psi.ndim > 1)
    npsi = psi.shape[-1]
    result = np.empty((nobj, npsi, nv))
    err = np.zeros(nobj, dtype=np.int32)
    nsteps = np.zeros(nobj, dtype=np.int64) if return_nsteps else None
    opts = _lib.make_opts(precision=_lib.FP64, device=device, max_attempts=max_attempts,
                          nsteps=nsteps, devices=devices)
    cb = _lib.CALLBACK()
    pbar = None
    if progressbar and nobj > 1:
        try:
            import tqdm

            pbar = tqdm.tqdm(total=nobj, leave=False)
            cb = _lib.CALLBACK(pbar.update)
        except ImportError:  # pragma: no cover
            pass
    args = [nobj, yoo.ctypes.data_as(_dp), npsi, psi.ctypes.data_as(_dp), indiv]
    if planar:  # galpy passes 1 for surface 'y', 0 otherwise (integratePlanarOrbit.py:1664)
        args.append(1 if surface == "y" else 0)
    args += [npot, pot_type.ctypes.data_as(_ip), pot_args.ctypes.data_as(_dp), None, dpsi, rtol,
             atol, result.ctypes.data_as(_dp), err.ctypes.data_as(_ip), code, cb,
             ctypes.byref(opts)]
    fn = _lib.lib().integratePlanarOrbit_sos_cuda if planar else \
        _lib.lib().integrateFullOrbit_sos_cuda
    rc = fn(*args)
    if pbar is not None:
        pbar.close()
    _lib.check(rc)
    if np.any(err == -10):
        raise KeyboardInterrupt("Orbit integration interrupted by CTRL-C (SIGINT)")
    out = (result[0], err[0]) if single_obj else (result, err)
    if return_nsteps:
        out = out + ((nsteps[0] if single_obj else nsteps),)
    return out


def integrateFullOrbit_sos_cuda(pot, yo, psi, t0, int_method, rtol=None, atol=None,
                                progressbar=True, dpsi=None, max_attempts=0,
                                return_nsteps=False, device=-1, devices=None):
    """Surface-of-section integration on the GPU (galpy's
    integrateFullOrbit_sos_c, galpy/orbit/integrateFullOrbit.py:1215-1355).

    yo [N,6] (R,vR,vT,z,vz,phi) or [6]; psi [npsi] or [N,npsi] increments of
    the angle psi = atan2(z, vz) at which the state is wanted; t0 the initial
    time (scalar or [N]); int_method 'rk4_cuda', 'rk6_cuda', 'dopr54_cuda' or
    'dop853_cuda'; dpsi the step (None: estimated).  Returns (y [N,npsi,7]
    with the time as the last column, err [N]); the leading axis is dropped
    for a single orbit.  devices: as for integrateFullOrbit_cuda (equal orbit
    counts per device)."""
    return _integrate_sos(False, pot, yo, psi, t0, int_method, None, rtol, atol, progressbar,
                          dpsi, max_attempts, return_nsteps, device, devices)


def integratePlanarOrbit_sos_cuda(pot, yo, psi, t0, int_method, surface="x", rtol=None,
                                  atol=None, progressbar=True, dpsi=None, max_attempts=0,
                                  return_nsteps=False, device=-1, devices=None):
    """Planar surface-of-section integration on the GPU (galpy's
    integratePlanarOrbit_sos_c, galpy/orbit/integratePlanarOrbit.py:1543-1693):
    yo [N,4] (R,vR,vT,phi); surface 'x' (x = 0, the default) or 'y' (y =
    0); returns (y [N,npsi,5] = (R,vR,vT,phi,t), err [N])."""
    return _integrate_sos(True, pot, yo, psi, t0, int_method, surface, rtol, atol, progressbar,
                          dpsi, max_attempts, return_nsteps, device, devices)


def _dxdv_single(planar, pot, yo, dyo, t, int_method, dt, rtol, atol, device):
    rtol, atol = parse_tol(rtol, atol)
    dt = _lib.DT_SENTINEL if dt is None else float(dt)
    npot, pot_type, pot_args = parse_pot(pot, planar=planar)
    code = parse_integrator(int_method)
    yo = np.require(np.concatenate((yo, dyo)), dtype=np.float64, requirements=["C", "W"])
    t = np.require(t, dtype=np.float64, requirements=["C", "W"])
    nv = 8 if planar else 12
    result = np.empty((len(t), nv))
    err = ctypes.c_int(0)
    opts = _lib.make_opts(device=device)
    L = _lib.lib()
    if planar:
        rc = L.integratePlanarOrbit_dxdv_cuda(
            yo.ctypes.data_as(_dp), len(t), t.ctypes.data_as(_dp), npot,
            pot_type.ctypes.data_as(_ip), pot_args.ctypes.data_as(_dp), None, dt, rtol, atol,
            result.ctypes.data_as(_dp), ctypes.byref(err), code, _lib.CALLBACK(),
            ctypes.byref(opts))
    else:
        rc = L.integrateFullOrbit_dxdv_cuda(
            yo.ctypes.data_as(_dp), len(t), t.ctypes.data_as(_dp), npot,
            pot_type.ctypes.data_as(_ip), pot_args.ctypes.data_as(_dp), None, dt, rtol, atol,
            result.ctypes.data_as(_dp), ctypes.byref(err), code, ctypes.byref(opts))
    _lib.check(rc)
    if int(err.value) == -10:
        raise KeyboardInterrupt("Orbit integration interrupted by CTRL-C (SIGINT)")
    return result, err.value


def integrateFullOrbit_dxdv_cuda(pot, yo, dyo, t, int_method, dt=None, rtol=None, atol=None,
                                 device=-1):
    """Mirror of galpy's integrateFullOrbit_dxdv_c: rectangular yo [6], dyo [6];
    returns (result [nt,12], err)."""
    return _dxdv_single(False, pot, yo, dyo, t, int_method, dt, rtol, atol, device)


def integratePlanarOrbit_dxdv_cuda(pot, yo, dyo, t, int_method, rtol=None, atol=None, dt=None,
                                   device=-1):
    """Mirror of galpy's integratePlanarOrbit_dxdv_c: rectangular yo [4],
    dyo [4]; returns (result [nt,8], err)."""
    return _dxdv_single(True, pot, yo, dyo, t, int_method, dt, rtol, atol, device)


def integrate_dxdv_batch(pot, w, t, int_method, planar=False, dt=None, rtol=None, atol=None,
                         device=-1, return_nsteps=False, devices=None):
    """Variational integration of many (orbit, deviation) pairs in one launch.

    w [N, 4*dim] rectangular (x, v, dx, dv); t [nt] or [N, nt].  Returns
    (result [N, nt, 4*dim], err [N]).  Build a state-transition matrix by
    passing the same orbit once per canonical deviation."""
    rtol, atol = parse_tol(rtol, atol)
    dt = _lib.DT_SENTINEL if dt is None else float(dt)
    npot, pot_type, pot_args = parse_pot(pot, planar=planar)
    code = parse_integrator(int_method)
    w = np.require(np.atleast_2d(w), dtype=np.float64, requirements=["C", "W"])
    t = np.require(t, dtype=np.float64, requirements=["C", "W"])
    nobj, nv = w.shape
    nt = t.shape[-1]
    result = np.empty((nobj, nt, nv))
    err = np.zeros(nobj, dtype=np.int32)
    nsteps = np.zeros(nobj, dtype=np.int64) if return_nsteps else None
    opts = _lib.make_opts(device=device, nsteps=nsteps, devices=devices)
    rc = _lib.lib().integrateOrbit_dxdv_batch_cuda(
        int(planar), nobj, w.ctypes.data_as(_dp), nt, t.ctypes.data_as(_dp), int(t.ndim > 1),
        npot, pot_type.ctypes.data_as(_ip), pot_args.ctypes.data_as(_dp), dt, rtol, atol,
        result.ctypes.data_as(_dp), err.ctypes.data_as(_ip), code, ctypes.byref(opts))
    _lib.check(rc)
    if np.any(err == -10):
        raise KeyboardInterrupt("Orbit integration interrupted by CTRL-C (SIGINT)")
    return (result, err, nsteps) if return_nsteps else (result, err)


def compile_potential(pot, planar=False, ngroup=1):
    """Compiled device records (bytes) of a potential, or of ngroup parameter
    groups when pot is (pot_type, pot_args) with ngroup argument blocks, and
    the number of records per group (the launches' ncomp)."""
    npot, pot_type, pot_args = parse_pot(pot, planar=planar)
    size = _lib.lib().galpy_cuda_comp_size()
    # records per group: one per component, plus an SCF expansion's
    # continuation records (the launch's ncomp)
    nrec = _lib.lib().galpy_cuda_comp_records(int(planar), npot, pot_type.ctypes.data_as(_ip),
                                              pot_args.ctypes.data_as(_dp))
    _lib.check(min(nrec, 0))
    buf = np.zeros(size * nrec * ngroup, dtype=np.uint8)
    rc = _lib.lib().galpy_cuda_compile_potential(
        int(planar), npot, pot_type.ctypes.data_as(_ip), pot_args.ctypes.data_as(_dp), ngroup,
        buf.ctypes.data_as(ctypes.c_void_p))
    _lib.check(rc)
    return buf, nrec


def signature(pot, planar=False):
    """Kernel specialisation of a potential (0 generic, 1 MWPotential2014-type)."""
    npot, pot_type, _ = parse_pot(pot, planar=planar)
    return _lib.lib().galpy_cuda_signature(npot, pot_type.ctypes.data_as(_ip))


def split_orbits(pot, w, t, nparts, planar=False, group=None, ngroup=1):
    """Contiguous orbit ranges of equal estimated cost (the cut a call with
    ``devices=`` makes), for spreading a batch over processes, one per
    device: part k is orbits [bounds[k], bounds[k+1]).

    w [N, nv] RECTANGULAR states, positions first (x, y[, z], ...); t [nt]
    or [N, nt]; for parameter groups, pot = (pot_type, pot_args) with
    ngroup argument blocks and group [N] each orbit's block.  The cost of an
    orbit is |t_end - t_0| * Omega(x_0), Omega^2 = |a.x| / |x|^2 in its
    group's potential.  Runs on the host; needs no GPU."""
    npot, pot_type, pot_args = parse_pot(pot, planar=planar)
    w = np.require(np.atleast_2d(w), dtype=np.float64, requirements=["C"])
    t = np.require(t, dtype=np.float64, requirements=["C"])
    if t.ndim > 1 and t.shape[0] != w.shape[0]:
        raise ValueError("per-orbit times need one row per orbit")
    gp = None
    if group is not None:
        group = np.require(group, dtype=np.int32, requirements=["C"])
        if group.shape != (w.shape[0],):
            raise ValueError("group needs one entry per orbit")
        gp = group.ctypes.data_as(_ip)
    bounds = np.zeros(int(nparts) + 1, dtype=np.int64)
    rc = _lib.lib().galpy_cuda_split_orbits(
        int(planar), w.shape[0], w.ctypes.data_as(_dp), w.shape[1], t.shape[-1],
        t.ctypes.data_as(_dp), int(t.ndim > 1), npot, pot_type.ctypes.data_as(_ip),
        pot_args.ctypes.data_as(_dp), int(ngroup), gp, int(nparts),
        bounds.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
    _lib.check(rc)
    return bounds


def shard_of(pot, w, t, rank, world, planar=False, group=None, ngroup=1):
    """This rank's orbit range (start, stop) of a batch spread over `world`
    processes by split_orbits.  The ranks share nothing but the inputs: each
    computes the same cut."""
    b = split_orbits(pot, w, t, world, planar=planar, group=group, ngroup=ngroup)
    return int(b[rank]), int(b[rank + 1])


def integrate_device(comps, ncomp, w0, t, out, err, int_method, planar=False, variational=False,
                     nsteps=None, group=None, in_layout="soa", out_layout="soa_rect",
                     out_row0=0, dt=None, rtol=None, atol=None, precision="fp64",
                     max_attempts=0, stream=None, block_size=0, grid_size=0, signature=0,
                     schedule="longest_first", variant=0, comps_host=None, tail_sms=-1,
                     system="orbit", abort_flag=None):
    """Asynchronous integration of device-resident torch tensors.

    comps: uint8 CUDA tensor of compiled records (compile_potential); w0
    float64 [nv, N] (in_layout 'soa') or [N, nv] ('aos'); t float64 [nt] or
    [N, nt]; out float64 sized for the layout ('soa_rect'/'soa_cyl':
    [nv, nt-out_row0, N], 'aos_rect'/'galpy': [N, nt-out_row0, nv]); err int32
    [N]; nsteps int64 [N] or None; group int32 [N] or None; signature from
    ``signature(pot)`` selects kernels specialised for the component list;
    system 'orbit' (default), or a surface-of-section system ('sos': 3D rows
    of 7, t holding the psi increments; 'sos_planar_x' / 'sos_planar_y':
    planar rows of 5, planar=True) with rk4/rk6/dopr54/dop853 in float64.
    Runs on `stream` (a torch.cuda.Stream, default: the current stream).
    abort_flag: optional int32 CUDA tensor (one element) that the kernel polls
    every 256 loop iterations; once it reads non-zero, the orbits in flight
    stop with err -10 and NaN rows after their last written one, and orbits
    not yet started get err -10 and NaN rows (the device form of galpy's
    SIGINT handling)."""
    import torch

    layouts_in = {"aos": _lib.IN_AOS, "soa": _lib.IN_SOA}
    layouts_out = {"galpy": _lib.OUT_GALPY, "aos_rect": _lib.OUT_AOS_RECT,
                   "soa_rect": _lib.OUT_SOA_RECT, "soa_cyl": _lib.OUT_SOA_CYL}
    for name, x, dt_ in (("w0", w0, torch.float64), ("t", t, torch.float64),
                         ("out", out, torch.float64), ("err", err, torch.int32)):
        if not (x.is_cuda and x.dtype == dt_ and x.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous CUDA tensor of {dt_}")
    nobj = err.shape[0]
    rtol, atol = parse_tol(rtol, atol)
    L = _lib.GalpyCudaLaunch()
    L.planar = int(planar)
    L.variational = int(variational)
    L.odeint_type = parse_integrator(int_method)
    L.precision = _precision(precision)
    L.nobj = nobj
    L.nt = t.shape[-1]
    L.indiv_t = int(t.dim() > 1)
    L.t = t.data_ptr()
    L.w0 = w0.data_ptr()
    L.in_layout = layouts_in[in_layout]
    L.out = out.data_ptr()
    L.out_layout = layouts_out[out_layout]
    L.out_row0 = out_row0
    L.err = err.data_ptr()
    L.nsteps = nsteps.data_ptr() if nsteps is not None else None
    L.comps = comps.data_ptr()
    L.ncomp = ncomp
    L.group = group.data_ptr() if group is not None else None
    L.dt = _lib.DT_SENTINEL if dt is None else float(dt)
    L.rtol = rtol
    L.atol = atol
    L.max_attempts = max_attempts
    if abort_flag is not None:
        if not (abort_flag.is_cuda and abort_flag.dtype == torch.int32):
            raise ValueError("abort_flag must be an int32 CUDA tensor")
        L.abort_flag = abort_flag.data_ptr()
    else:
        L.abort_flag = None
    s = stream if stream is not None else torch.cuda.current_stream(w0.device)
    L.stream = s.cuda_stream
    L.block_size = block_size
    L.grid_size = grid_size
    L.signature = int(signature)
    L.schedule = {"in_order": 0, "longest_first": 1}[schedule]
    L.variant = int(variant)
    # host copy of the records (numpy uint8 from compile_potential): lets a
    # single-potential launch pass its scalars as kernel parameters
    L.comps_host = comps_host.ctypes.data if comps_host is not None else None
    # SMs reserved for the longest orbits of a large longest-first batch
    L.size_ext = 2
    L.tail_sms = int(tail_sms)
    L.system = SYSTEMS[system] if isinstance(system, str) else int(system)
    _lib.check(_lib.lib().galpy_cuda_integrate_device(ctypes.byref(L)))


def accel_device(comps, ncomp, pos, acc, planar=False, signature=0, precision="fp64",
                 group=None, stream=None):
    """Accelerations [3, N] at positions pos [3, N] (float64 CUDA tensors,
    z ignored when planar) with the integration kernels' force code."""
    import torch

    for name, x in (("pos", pos), ("acc", acc)):
        if not (x.is_cuda and x.dtype == torch.float64 and x.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous CUDA tensor of float64")
    s = stream if stream is not None else torch.cuda.current_stream(pos.device)
    _lib.check(_lib.lib().galpy_cuda_accel_device(
        comps.data_ptr(), ncomp, group.data_ptr() if group is not None else None, int(planar),
        int(signature), _precision(precision), pos.data_ptr(), pos.shape[1], acc.data_ptr(),
        s.cuda_stream))


def energy_device(comps, ncomp, w, E, planar=False, layout="soa", group=None, stream=None):
    """E = v^2/2 + Phi(x) of device-resident rectangular states (torch).

    w: float64 CUDA tensor [nv, N] ('soa') or [N, nv] ('aos'), or any
    strided view with those two axes; E: float64 [N]."""
    import torch

    if layout == "soa":
        sc, so = w.stride(0), w.stride(1)
    else:
        so, sc = w.stride(0), w.stride(1)
    s = stream if stream is not None else torch.cuda.current_stream(w.device)
    _lib.check(_lib.lib().galpy_cuda_energy_device(
        comps.data_ptr(), ncomp, group.data_ptr() if group is not None else None, int(planar),
        w.data_ptr(), E.shape[0], sc, so, E.data_ptr(), s.cuda_stream))
