"""Launch-shape autotuner for the integration kernels.

The engine runs one orbit per thread in a persistent, work-stealing grid
(galpy_b200/csrc/galpy_cuda.cu).  What is left to choose per workload is the
launch shape, and the best choice differs between integrators, dimensions,
precisions and potentials (register pressure, shared-memory slot stores,
how ragged the step counts are):

* ``block_size`` -- orbits per block (64 or 128 for the fixed-step
  integrators; DOP853 runs 128: at its ~214 registers each SM sub-partition
  holds two warps whatever the block, and blocks of 96 -- which a sample of
  the batching workload preferred -- left 6 warps per SM and made the full
  batch 22 % slower);
* ``variant`` -- register budget: 0 = compiler default (up to 255 registers
  a thread), 1 = capped so that more blocks are resident per SM;
* ``schedule`` -- not tuned: always longest first by the estimated cost
  |t_end - t_0| * orbital frequency.  Its pre-pass costs about a millisecond,
  and what it prevents -- the longest orbits starting late and running alone
  at the end -- only shows on the whole batch: a subsample has shorter
  longest orbits and fewer orbits per thread, and once let a noisy in-order
  win on the sample cost the full batch 1.5x;
* ``threads_per_orbit`` -- 1 (the only form the kernels implement: every
  lane owns a whole orbit, so that each lane's force evaluation is the
  warp's single force call site).

``tune`` times every candidate with CUDA events on a random subsample of the
caller's batch (same initial conditions, times and potential) and keeps the
fastest; results are cached per device and workload key in a JSON file
(``$GALPY_B200_AUTOTUNE_CACHE``, default ``~/.cache/galpy_b200/autotune.json``)
so that later calls with the same key reuse them without timing.
"""
import json
import os
import threading

from . import _lib
from .integrate import integrate_device, parse_integrator

_lock = threading.Lock()
_memo = {}


def cache_path():
    return os.environ.get("GALPY_B200_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "galpy_b200",
                                       "autotune.json"))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key, cfg):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        data = _load()
        data[key] = cfg
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # an unwritable cache only costs a re-tune


def candidates(int_method):
    """Launch shapes to try for an integrator."""
    code = parse_integrator(int_method)
    shapes = []
    if code == 6:
        pairs = ((128, 0), (128, 1))
    else:
        pairs = tuple((b, v) for b in (64, 128) for v in (0, 1))
    for block, variant in pairs:
        shapes.append({"block_size": block, "variant": variant,
                       "schedule": "longest_first", "threads_per_orbit": 1})
    return shapes


def workload_key(device_name, int_method, planar, precision, signature, variational, nobj,
                 indiv_t, extra=""):
    """Cache key: the device, the kernel instantiation, and the batch size
    and time layout rounded to a power of two (the best shape depends on
    how many waves the batch fills and on how ragged it is)."""
    nb = max(int(nobj), 1).bit_length()
    try:  # a rebuilt library may want different shapes
        build = int(os.path.getmtime(_lib.LIB_PATH))
    except OSError:
        build = 0
    return (f"{device_name}|build={build}|{parse_integrator(int_method)}|planar={int(planar)}|"
            f"prec={precision}|sig={int(signature)}|var={int(variational)}|n~2^{nb}|"
            f"indiv_t={int(indiv_t)}|{extra}")


def tune(comps, ncomp, w0, t, out, err, int_method, planar=False, variational=False,
         precision="fp64", signature=0, group=None, out_row0=0, dt=None, rtol=None, atol=None,
         comps_host=None, sample=131072, seed=0, use_cache=True, key_extra="", verbose=False,
         out_layout="soa_rect"):
    """Best launch shape for this batch (dict of integrate_device keyword
    arguments, plus ``threads_per_orbit`` and the measured ``ms``).

    Arguments as for integrate_device with device tensors w0 [nv, N]
    (SoA), t [nt] or [N, nt], out [nv, nt - out_row0, N] (out_layout
    'soa_rect' / 'soa_cyl') or [N, nt - out_row0, nv] ('aos_rect' /
    'galpy') and err [N].  At most ``sample`` orbits, drawn at random, are
    timed per candidate."""
    import torch

    nobj = err.shape[0]
    dev = w0.device
    key = workload_key(torch.cuda.get_device_name(dev), int_method, planar, precision,
                       signature, variational, nobj, t.dim() > 1,
                       key_extra + ("" if out_layout == "soa_rect" else f"|out={out_layout}"))
    with _lock:
        if use_cache:
            if key in _memo:
                return dict(_memo[key])
            cached = _load().get(key)
            if cached:
                _memo[key] = cached
                return dict(cached)
    m = min(int(sample), nobj)
    g = torch.Generator(device="cpu").manual_seed(seed)
    idx = torch.randperm(nobj, generator=g)[:m].to(dev)
    w_s = w0[:, idx].contiguous()
    t_s = t[idx].contiguous() if t.dim() > 1 else t
    if out_layout in ("aos_rect", "galpy"):
        out_s = torch.empty((m, out.shape[1], out.shape[2]), dtype=out.dtype, device=dev)
    else:
        out_s = torch.empty((out.shape[0], out.shape[1], m), dtype=out.dtype, device=dev)
    err_s = torch.empty(m, dtype=torch.int32, device=dev)
    grp_s = group[idx].contiguous() if group is not None else None
    stream = torch.cuda.current_stream(dev)

    def run(cfg):
        integrate_device(comps, ncomp, w_s, t_s, out_s, err_s, int_method, planar=planar,
                         variational=variational, group=grp_s, out_row0=out_row0, dt=dt,
                         rtol=rtol, atol=atol, precision=precision, stream=stream,
                         signature=signature, comps_host=comps_host,
                         block_size=cfg["block_size"], variant=cfg["variant"],
                         schedule=cfg["schedule"], out_layout=out_layout)

    results = []
    cands = candidates(int_method)
    run(cands[0])  # warm-up: module load, first-touch of the buffers
    for cfg in cands:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        run(cfg)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        results.append((ms, cfg))
        if verbose:
            print(f"autotune {key}: {cfg} {ms:.3f} ms")
    ms, best = min(results, key=lambda r: r[0])
    best = dict(best, ms=ms, sample=m)
    with _lock:
        _memo[key] = best
        if use_cache:
            _store(key, best)
    return dict(best)


def launch_kwargs(cfg):
    """The integrate_device keyword arguments of a tuned shape."""
    return {k: cfg[k] for k in ("block_size", "variant", "schedule")}
