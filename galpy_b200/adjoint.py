"""Gradients of final orbit states with respect to initial conditions and
potential parameters (reverse mode, on the GPU).

galpy itself has no adjoint: its gradient information is the variational
integration ``Orbit.integrate_dxdv`` (galpy/orbit/Orbits.py:2445, C in
integratePlanarOrbit.c:940 / integrateFullOrbit.c:1234), which propagates one
tangent vector per input direction.  Here a loss on the final states is
differentiated with one backward sweep per orbit:

* forward: galpy's DOP853 from t0 to tend on the GPU (the step sequence of
  method 'dop853_c'/'dop853_cuda', y(tend) from its dense output), saving
  the state every 64 accepted steps with those steps' sizes (checkpoints);
* backward: each 64-step segment is recomputed from its checkpoint with the
  recorded step sizes and the exact adjoint of the Runge-Kutta stages is
  applied with the step sizes held fixed (tidal tensors for the state,
  analytic derivatives of the forces for the parameters).

``final_state`` wraps both passes in a ``torch.autograd.Function``::

    w0 = torch.tensor(..., dtype=torch.float64, device="cuda", requires_grad=True)
    pot_args = torch.tensor(galpy_pot_args, dtype=torch.float64, requires_grad=True)
    yT = final_state(w0, (pot_type, pot_args), tend=20.0, planar=True, rtol=1e-10)
    loss = ((yT - targets) ** 2).sum()
    loss.backward()   # w0.grad, pot_args.grad

Differentiable parameters (the other entries of pot_args get zero
gradient): PowerSphericalPotentialwCutoff amp and rc, MiyamotoNagai amp, a,
b, NFW amp and a, Hernquist amp and a, LogarithmicHalo amp, q and core^2.

When torch.distributed is initialised and the orbits are sharded over the
ranks, the potential-parameter gradient is summed over the ranks (one
all-reduce of a few doubles); initial-condition gradients stay sharded.
"""
import ctypes

import numpy as np

from . import _lib
from .integrate import parse_tol
from .potentials import parse_pot

CKPT_EVERY = 64

_ip = ctypes.POINTER(ctypes.c_int)


def adjoint_params(pot_type, planar=False, pot_args=None):
    """pot_args index of every differentiable parameter of a component list
    (pot_args is needed for the ellipsoidal types, whose argument count
    depends on their arguments)."""
    pt = np.ascontiguousarray(pot_type, dtype=np.int32)
    pa = None if pot_args is None else np.ascontiguousarray(pot_args, dtype=np.float64)
    pap = None if pa is None else pa.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    n = _lib.lib().galpy_cuda_adjoint_params(int(planar), len(pt), pt.ctypes.data_as(_ip), pap,
                                             None)
    if n < 0:
        _lib.check(n)
    idx = np.zeros(max(n, 1), dtype=np.int32)
    _lib.lib().galpy_cuda_adjoint_params(int(planar), len(pt), pt.ctypes.data_as(_ip), pap,
                                         idx.ctypes.data_as(_ip))
    return idx[:n]


def _require(name, x, dtype):
    import torch

    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == dtype and x.is_contiguous()):
        raise ValueError(f"{name} must be a contiguous CUDA tensor of {dtype}")


def _struct(planar, nobj, t0, tend, rtol, atol, comps, ncomp, group, signature, w0, stream,
            max_attempts=0, block_size=0):
    a = _lib.GalpyCudaAdjoint()
    a.size = ctypes.sizeof(_lib.GalpyCudaAdjoint)
    a.planar = int(planar)
    a.nobj = nobj
    a.t0 = float(t0)
    a.tend = float(tend)
    a.rtol = rtol
    a.atol = atol
    a.max_attempts = int(max_attempts)
    a.comps = comps.data_ptr()
    a.ncomp = int(ncomp)
    a.group = group.data_ptr() if group is not None else None
    a.signature = int(signature)
    a.w0 = w0.data_ptr()
    a.stream = stream.cuda_stream
    a.block_size = int(block_size)
    return a


def _cost_order(comps, ncomp, w0, planar, signature, group, stream):
    """Orbits by decreasing estimated cost, the local orbital frequency
    sqrt(|a . x|) / |x| at the initial point (the step count of an adaptive
    integration over a common interval grows with it), so that the lanes of
    a warp integrate orbits of similar length."""
    import torch

    from .integrate import accel_device

    nv, n = w0.shape
    d = nv // 2
    pos = torch.zeros((3, n), dtype=torch.float64, device=w0.device)
    pos[:d] = w0[:d]
    acc = torch.empty_like(pos)
    accel_device(comps, ncomp, pos, acc, planar=planar, signature=signature, group=group,
                 stream=stream)
    r2 = (pos * pos).sum(0)
    cost = torch.sqrt(torch.abs((acc * pos).sum(0))) / torch.sqrt(r2)
    return torch.argsort(cost, descending=True).to(torch.int32)


def adjoint_forward(comps, ncomp, w0, tend, t0=0.0, rtol=None, atol=None, planar=False,
                    signature=0, group=None, ckpt_cap=None, record_steps=0, max_attempts=0,
                    stream=None, block_size=0, sort=True):
    """Forward pass on device-resident tensors.

    comps: uint8 CUDA tensor of compiled records (compile_potential); w0:
    float64 CUDA tensor [nv, N] (SoA, rectangular).  Returns a dict with
    yT [nv, N], nsteps int64 [N], err int32 [N], ckpt, ckpt_cap and, with
    record_steps > 0, hrec [record_steps, N] (the accepted step sizes, for
    ``adjoint_replay``).  Checkpoints take (nv + 65) doubles per orbit and 64
    steps; by default the capacity starts at 512 steps and orbits that need
    more are re-run with 4x the capacity (up to twice).  sort: hand orbits to
    the GPU threads by decreasing estimated cost (the results do not
    depend on the order)."""
    import torch

    _require("w0", w0, torch.float64)
    nv, nobj = w0.shape
    if nv != (4 if planar else 6):
        raise ValueError("w0 must be [4, N] (planar) or [6, N]")
    rtol, atol = parse_tol(rtol, atol)
    s = stream if stream is not None else torch.cuda.current_stream(w0.device)
    dev = w0.device
    cap = int(ckpt_cap) if ckpt_cap else 8
    order = _cost_order(comps, ncomp, w0, planar, signature, group, s) if sort and nobj > 1 \
        else None
    for attempt in range(3):
        a = _struct(planar, nobj, t0, tend, rtol, atol, comps, ncomp, group, signature, w0, s,
                    max_attempts, block_size)
        yT = torch.empty((nv, nobj), dtype=torch.float64, device=dev)
        nsteps = torch.empty(nobj, dtype=torch.int64, device=dev)
        err = torch.empty(nobj, dtype=torch.int32, device=dev)
        ckpt = torch.empty((cap, nv + 1 + CKPT_EVERY, nobj), dtype=torch.float64, device=dev)
        hrec = (torch.empty((record_steps, nobj), dtype=torch.float64, device=dev)
                if record_steps else None)
        a.yT, a.nsteps, a.err, a.ckpt = (yT.data_ptr(), nsteps.data_ptr(), err.data_ptr(),
                                         ckpt.data_ptr())
        a.ckpt_cap = cap
        a.hrec = hrec.data_ptr() if hrec is not None else None
        a.hcap = record_steps
        a.order = order.data_ptr() if order is not None else None
        _lib.check(_lib.lib().galpy_cuda_adjoint_forward(ctypes.byref(a)))
        if ckpt_cap or max_attempts or record_steps:
            break
        over = (err == 2) & (nsteps == 0)
        if not bool(over.any()):
            break
        cap *= 4
    return {"yT": yT, "nsteps": nsteps, "err": err, "ckpt": ckpt, "ckpt_cap": cap,
            "hrec": hrec}


def adjoint_backward(comps, ncomp, fwd, gyT, tend, t0=0.0, rtol=None, atol=None, planar=False,
                     signature=0, group=None, nparam=None, stream=None, block_size=0, w0=None,
                     sort=True, variant=0):
    """Backward pass: (gw0 [nv, N], gparam [nparam, N]) for dL/dyT = gyT
    [nv, N], from the dict returned by adjoint_forward (same potential,
    interval and tolerances).  sort: hand the orbits to the GPU threads by
    decreasing step count (the forward pass's exact cost), so that the lanes
    of a warp do similar work and the longest orbits start first."""
    import torch

    gyT = gyT.contiguous()
    _require("gyT", gyT, torch.float64)
    nv, nobj = gyT.shape
    rtol, atol = parse_tol(rtol, atol)
    s = stream if stream is not None else torch.cuda.current_stream(gyT.device)
    a = _struct(planar, nobj, t0, tend, rtol, atol, comps, ncomp, group, signature,
                w0 if w0 is not None else gyT, s, 0, block_size)
    gw0 = torch.empty_like(gyT)
    gparam = torch.empty((max(int(nparam or 0), 1), nobj), dtype=torch.float64,
                         device=gyT.device)
    a.nsteps = fwd["nsteps"].data_ptr()
    a.err = fwd["err"].data_ptr()
    a.ckpt = fwd["ckpt"].data_ptr()
    a.ckpt_cap = fwd["ckpt_cap"]
    a.gyT = gyT.data_ptr()
    a.gw0 = gw0.data_ptr()
    a.gparam = gparam.data_ptr() if nparam else None
    a.variant = int(variant)
    order = None
    if sort:
        order = torch.argsort(fwd["nsteps"], descending=True).to(torch.int32)
        a.order = order.data_ptr()
    _lib.check(_lib.lib().galpy_cuda_adjoint_backward(ctypes.byref(a)))
    return gw0, (gparam[:nparam] if nparam else None)


def adjoint_replay(comps, ncomp, w0, hrec, nsteps, tend, t0=0.0, planar=False, signature=0,
                   group=None, stream=None):
    """y(tend) [nv, N] with the step sizes frozen at hrec [hcap, N] (nsteps
    [N] of them per orbit): the map whose exact derivative the backward pass
    computes."""
    import torch

    _require("w0", w0, torch.float64)
    nv, nobj = w0.shape
    s = stream if stream is not None else torch.cuda.current_stream(w0.device)
    a = _struct(planar, nobj, t0, tend, 0.0, 0.0, comps, ncomp, group, signature, w0, s)
    yT = torch.empty_like(w0)
    a.yT = yT.data_ptr()
    a.nsteps = nsteps.data_ptr()
    a.hrec = hrec.data_ptr()
    a.hcap = hrec.shape[0]
    _lib.check(_lib.lib().galpy_cuda_adjoint_replay(ctypes.byref(a)))
    return yT


def reduce_param_grad(g):
    """Sum a parameter gradient over the ranks of an initialised
    torch.distributed group (orbits sharded across ranks); identity
    otherwise."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(g, op=dist.ReduceOp.SUM)
    return g


def _compile(pot_type, pot_args_np, planar, device):
    import torch

    from .integrate import compile_potential, signature

    buf, n = compile_potential((pot_type, pot_args_np), planar=planar)
    return (torch.from_numpy(buf).to(device), n,
            signature((pot_type, pot_args_np), planar=planar))


def _autograd_function():
    import torch

    class FinalState(torch.autograd.Function):
        """y(tend) of orbits w0 [N, nv] in the potential (pot_type, pot_args);
        differentiable with respect to w0 and pot_args."""

        @staticmethod
        def forward(ctx, w0, pot_args, spec):
            planar, pot_type, t0, tend, rtol, atol, reduce = spec
            pa = pot_args.detach().to("cpu", torch.float64).numpy()
            # the parameter map first: a potential without gradients fails
            # before any device work
            idx = adjoint_params(pot_type, planar, pa)
            comps, ncomp, sig = _compile(pot_type, pa, planar, w0.device)
            w0s = w0.detach().t().contiguous()
            fwd = adjoint_forward(comps, ncomp, w0s, tend, t0=t0, rtol=rtol, atol=atol,
                                  planar=planar, signature=sig)
            ctx.spec = spec
            ctx.idx = idx
            ctx.state = (comps, ncomp, sig, fwd, w0s)
            ctx.pot_args_meta = (pot_args.shape, pot_args.device, pot_args.dtype)
            return fwd["yT"].t()

        @staticmethod
        def backward(ctx, gy):
            planar, pot_type, t0, tend, rtol, atol, reduce = ctx.spec
            comps, ncomp, sig, fwd, w0s = ctx.state
            idx = ctx.idx
            gw0, gparam = adjoint_backward(comps, ncomp, fwd, gy.t().contiguous(), tend, t0=t0,
                                           rtol=rtol, atol=atol, planar=planar, signature=sig,
                                           nparam=len(idx), w0=w0s)
            g_pa = None
            if ctx.needs_input_grad[1]:
                shape, device, dtype = ctx.pot_args_meta
                g = torch.zeros(int(np.prod(shape)), dtype=torch.float64, device=gw0.device)
                if len(idx):
                    g.index_add_(0, torch.from_numpy(idx.astype(np.int64)).to(gw0.device),
                                 gparam.sum(dim=1))
                if reduce:
                    reduce_param_grad(g)
                g_pa = g.reshape(shape).to(device=device, dtype=dtype)
            return gw0.t(), g_pa, None

    return FinalState


_FinalState = None


def final_state(w0, pot, tend, t0=0.0, rtol=None, atol=None, planar=None, reduce_params=True):
    """Differentiable y(tend) [N, nv] of the orbits w0 [N, nv] (float64 CUDA
    tensor, rectangular: (x, y, vx, vy) planar or (x, y, z, vx, vy, vz)).

    pot: (pot_type, pot_args) with pot_args a float64 torch tensor (CPU or
    CUDA; its gradient is returned on the same device), or any potential
    ``parse_pot`` accepts (then no parameter gradient is tracked).  rtol /
    atol as galpy's (default 1e-12 like galpy's C integrators)."""
    import torch

    global _FinalState
    if _FinalState is None:
        _FinalState = _autograd_function()
    if planar is None:
        planar = w0.shape[-1] == 4
    if isinstance(pot, tuple) and len(pot) == 2 and isinstance(pot[1], torch.Tensor):
        pot_type = tuple(int(t) for t in np.asarray(pot[0]).ravel())
        pot_args = pot[1]
    else:
        _, pt, pa = parse_pot(pot, planar=planar)
        pot_type = tuple(int(t) for t in pt)
        pot_args = torch.from_numpy(np.asarray(pa, dtype=np.float64))
    spec = (bool(planar), pot_type, float(t0), float(tend), rtol, atol, bool(reduce_params))
    return _FinalState.apply(w0, pot_args, spec)
