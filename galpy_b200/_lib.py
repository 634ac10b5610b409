"""Loader of libgalpy_cuda.so (the engine's C ABI, include/galpy_cuda.h).

Mirrors galpy/util/_load_extension_libs.py:64-111 (ctypes.CDLL of an
in-tree shared library) but fails loudly: there is no CPU fallback in this
package.  Any call that needs the library raises CudaLibraryMissing when the
library was not built, and CudaError when the CUDA runtime reports a failure.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgalpy_cuda.so")

OK = 0
ERR_ARG = -1
ERR_METHOD = -2
ERR_POTENTIAL = -3
ERR_CUDA = -4
ERR_NODEVICE = -5
ERR_INTERRUPTED = -10

FP64 = 0
F32FORCE = 1

IN_AOS, IN_SOA = 0, 1
OUT_GALPY, OUT_AOS_RECT, OUT_SOA_RECT, OUT_SOA_CYL = 0, 1, 2, 3

SYS_ORBIT, SYS_SOS, SYS_SOS_PLANAR_X, SYS_SOS_PLANAR_Y = 0, 1, 2, 3

DT_SENTINEL = -9999.99


class CudaLibraryMissing(RuntimeError):
    """libgalpy_cuda.so has not been built (run galpy_b200.build.build())."""


class CudaError(RuntimeError):
    """The engine returned an error status."""

    def __init__(self, code, msg):
        super().__init__(f"galpy_cuda error {code}: {msg}")
        self.code = code


class MethodNotSupported(CudaError):
    pass


class PotentialNotSupported(CudaError):
    pass


class GalpyCudaOpts(ctypes.Structure):
    _fields_ = [
        ("size", ctypes.c_int),
        ("device", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("block_size", ctypes.c_int),
        ("max_attempts", ctypes.c_longlong),
        ("nsteps", ctypes.POINTER(ctypes.c_longlong)),
        ("elapsed_ms", ctypes.POINTER(ctypes.c_double)),
        ("variant", ctypes.c_int),
        ("schedule", ctypes.c_int),
        ("stream_rows", ctypes.c_int),
        ("ndevices", ctypes.c_int),
        ("devices", ctypes.POINTER(ctypes.c_int)),
    ]


class GalpyCudaLaunch(ctypes.Structure):
    _fields_ = [
        ("planar", ctypes.c_int),
        ("variational", ctypes.c_int),
        ("odeint_type", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("nobj", ctypes.c_longlong),
        ("nt", ctypes.c_int),
        ("indiv_t", ctypes.c_int),
        ("t", ctypes.c_void_p),
        ("w0", ctypes.c_void_p),
        ("in_layout", ctypes.c_int),
        ("out", ctypes.c_void_p),
        ("out_layout", ctypes.c_int),
        ("out_row0", ctypes.c_int),
        ("err", ctypes.c_void_p),
        ("nsteps", ctypes.c_void_p),
        ("comps", ctypes.c_void_p),
        ("ncomp", ctypes.c_int),
        ("group", ctypes.c_void_p),
        ("dt", ctypes.c_double),
        ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("max_attempts", ctypes.c_longlong),
        ("abort_flag", ctypes.c_void_p),
        ("stream", ctypes.c_void_p),
        ("block_size", ctypes.c_int),
        ("grid_size", ctypes.c_int),
        ("signature", ctypes.c_int),
        ("schedule", ctypes.c_int),
        ("variant", ctypes.c_int),
        ("comps_host", ctypes.c_void_p),
        ("size_ext", ctypes.c_int),
        ("tail_sms", ctypes.c_int),
        ("system", ctypes.c_int),
    ]


class GalpyCudaAdjoint(ctypes.Structure):
    _fields_ = [
        ("size", ctypes.c_int),
        ("planar", ctypes.c_int),
        ("nobj", ctypes.c_longlong),
        ("t0", ctypes.c_double),
        ("tend", ctypes.c_double),
        ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("max_attempts", ctypes.c_longlong),
        ("comps", ctypes.c_void_p),
        ("ncomp", ctypes.c_int),
        ("group", ctypes.c_void_p),
        ("signature", ctypes.c_int),
        ("w0", ctypes.c_void_p),
        ("yT", ctypes.c_void_p),
        ("nsteps", ctypes.c_void_p),
        ("err", ctypes.c_void_p),
        ("ckpt", ctypes.c_void_p),
        ("ckpt_cap", ctypes.c_int),
        ("hrec", ctypes.c_void_p),
        ("hcap", ctypes.c_longlong),
        ("gyT", ctypes.c_void_p),
        ("gw0", ctypes.c_void_p),
        ("gparam", ctypes.c_void_p),
        ("stream", ctypes.c_void_p),
        ("block_size", ctypes.c_int),
        ("order", ctypes.c_void_p),
        ("variant", ctypes.c_int),
    ]


CALLBACK = ctypes.CFUNCTYPE(None)

_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_ci = ctypes.c_int
_cd = ctypes.c_double
_opts_p = ctypes.POINTER(GalpyCudaOpts)

# exported symbol -> (restype, argtypes); every symbol declared in include/galpy_cuda.h
SIGNATURES = {
    "galpy_cuda_abi_version": (_ci, []),
    "galpy_cuda_last_error": (ctypes.c_char_p, []),
    "galpy_cuda_device_count": (_ci, []),
    "galpy_cuda_comp_size": (_ci, []),
    "galpy_cuda_comp_records": (_ci, [_ci, _ci, _ip, _dp]),
    "galpy_cuda_signature": (_ci, [_ci, _ip]),
    "galpy_cuda_compile_potential": (_ci, [_ci, _ci, _ip, _dp, _ci, _vp]),
    "integrateFullOrbit_cuda": (
        _ci,
        [_ci, _dp, _ci, _dp, _ci, _ci, _ip, _dp, _vp, _cd, _cd, _cd, _dp, _ip, _ci, CALLBACK,
         _opts_p],
    ),
    "integrateFullOrbit_sos_cuda": (
        _ci,
        [_ci, _dp, _ci, _dp, _ci, _ci, _ip, _dp, _vp, _cd, _cd, _cd, _dp, _ip, _ci, CALLBACK,
         _opts_p],
    ),
    "integratePlanarOrbit_sos_cuda": (
        _ci,
        [_ci, _dp, _ci, _dp, _ci, _ci, _ci, _ip, _dp, _vp, _cd, _cd, _cd, _dp, _ip, _ci,
         CALLBACK, _opts_p],
    ),
    "integratePlanarOrbit_cuda": (
        _ci,
        [_ci, _dp, _ci, _dp, _ci, _ci, _ip, _dp, _vp, _cd, _cd, _cd, _dp, _ip, _ci, CALLBACK,
         _opts_p],
    ),
    "integrateFullOrbit_dxdv_cuda": (
        _ci, [_dp, _ci, _dp, _ci, _ip, _dp, _vp, _cd, _cd, _cd, _dp, _ip, _ci, _opts_p]),
    "integratePlanarOrbit_dxdv_cuda": (
        _ci, [_dp, _ci, _dp, _ci, _ip, _dp, _vp, _cd, _cd, _cd, _dp, _ip, _ci, CALLBACK, _opts_p]),
    "integrateOrbit_dxdv_batch_cuda": (
        _ci,
        [_ci, _ci, _dp, _ci, _dp, _ci, _ci, _ip, _dp, _cd, _cd, _cd, _dp, _ip, _ci, _opts_p],
    ),
    "galpy_cuda_integrate_device": (_ci, [ctypes.POINTER(GalpyCudaLaunch)]),
    "galpy_cuda_integrate_device_noalloc": (_ci, [ctypes.POINTER(GalpyCudaLaunch)]),
    "galpy_cuda_fp64_peak": (_ci, [_dp, _dp]),
    "galpy_cuda_energy_device": (
        _ci, [_vp, _ci, _vp, _ci, _vp, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong,
              _vp, _vp]),
    "galpy_cuda_adjoint_forward": (_ci, [ctypes.POINTER(GalpyCudaAdjoint)]),
    "galpy_cuda_adjoint_backward": (_ci, [ctypes.POINTER(GalpyCudaAdjoint)]),
    "galpy_cuda_adjoint_replay": (_ci, [ctypes.POINTER(GalpyCudaAdjoint)]),
    "galpy_cuda_adjoint_params": (_ci, [_ci, _ci, _ip, _dp, _ip]),
    "galpy_cuda_accel_device": (
        _ci, [_vp, _ci, _vp, _ci, _ci, _ci, _vp, ctypes.c_longlong, _vp, _vp]),
    "galpy_cuda_split_orbits": (
        _ci, [_ci, ctypes.c_longlong, _dp, _ci, _ci, _dp, _ci, _ci, _ip, _dp, _ci, _ip, _ci,
              ctypes.POINTER(ctypes.c_longlong)]),
    "galpy_cuda_orbit_interp_device": (
        _ci, [_ci, ctypes.c_longlong, _ci, _vp, _ci, _vp, _ci, _vp, _ci, _vp, _vp]),
    "galpy_cuda_trim_memory": (_ci, [_ci]),
    "galpy_cuda_jacobi_device": (
        _ci, [_vp, _ci, _vp, _ci, _vp, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong,
              _dp, _vp, _vp]),
}


def lib():
    """The loaded library (raises CudaLibraryMissing if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CudaLibraryMissing(
                f"{LIB_PATH} not found: build it with `python -c 'import galpy_b200.build as b; "
                "b.build()'` (needs nvcc); galpy_b200 has no CPU fallback")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def last_error():
    return lib().galpy_cuda_last_error().decode(errors="replace")


def check(code):
    """Raise the matching exception for a non-zero status."""
    if code == OK:
        return
    msg = last_error()
    if code == ERR_METHOD:
        raise MethodNotSupported(code, msg)
    if code == ERR_POTENTIAL:
        raise PotentialNotSupported(code, msg)
    if code == ERR_INTERRUPTED:
        raise KeyboardInterrupt("Orbit integration interrupted by CTRL-C (SIGINT)")
    raise CudaError(code, msg)


def make_opts(precision=FP64, device=-1, block_size=0, max_attempts=0, nsteps=None,
              elapsed=None, variant=0, schedule=1, stream_rows=-1, devices=None):
    """devices: None (one device, `device`), -1 (every visible device) or a
    sequence of device ordinals the call spreads its orbits over."""
    o = GalpyCudaOpts()
    o.size = ctypes.sizeof(GalpyCudaOpts)
    o.device = device
    o.precision = precision
    o.block_size = block_size
    o.max_attempts = max_attempts
    if nsteps is not None:
        o.nsteps = nsteps.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    if elapsed is not None:
        o.elapsed_ms = ctypes.pointer(elapsed)
    o.variant = variant
    o.schedule = schedule
    o.stream_rows = stream_rows
    if devices is None:
        o.ndevices = 0
    elif isinstance(devices, int):
        if devices != -1:
            raise ValueError("devices: -1 (every visible device) or a sequence of ordinals")
        o.ndevices = -1
    else:
        arr = (ctypes.c_int * len(devices))(*[int(d) for d in devices])
        o._devices_keep = arr  # the array lives as long as the opts
        o.ndevices = len(devices)
        o.devices = ctypes.cast(arr, ctypes.POINTER(ctypes.c_int))
    return o
