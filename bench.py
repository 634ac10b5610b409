#!/usr/bin/env python
"""Throughput of the batched orbit integrator: orbit-steps/s.

Workload (the batching configuration): 1,048,576 orbits per GPU in
MWPotential2014, DOP853 with rtol = atol = 1e-10, float64 state.  Initial
conditions from a seeded generator: R log-uniform in [0.05, 3], vR ~ N(0,
0.1), vT ~ 1 + N(0, 0.1), z ~ N(0, 0.05), vz ~ N(0, 0.05), phi ~ U(0, 2 pi);
every orbit has its own end time t_end ~ LogNormal(ln 50, 0.7) and keeps 101
snapshots (float64 on the device, one orbit's rows contiguous).  One "step" is one integration of the
whole batch; an orbit-step is one accepted DOP853 step of one orbit.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl galpy_b200|reference]

value: device-resident inputs, K launches timed with CUDA events on the
launching stream (max over ranks).  e2e: the same batch through the
galpy-facing C ABI (integrateFullOrbit_cuda) from pinned host buffers,
host<->device copies inside the timed region.  cpu_baseline / the reference
arm: the reference's own C integrators (oracle/_ref, built from the
reference's sources) -- or, where that build is absent, the CPU oracle -- on
a bounded sample of the same workload on all host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))

N_ORBITS = 1 << 20
NT = 101
RTOL = ATOL = 1e-10
F_STEP_DOP853 = 6500.0  # nominal float64 flops per accepted DOP853 step (MWPotential2014)
METRIC = "orbit-steps/s (MWPotential2014, dop853 rtol=atol=1e-10, ragged t_end, 1 B200)"
WORKLOAD = ("batching: 1,048,576 orbits/GPU in MWPotential2014, dop853 rtol=atol=1e-10, "
            "R log-uniform [0.05,3], t_end ~ LogNormal(ln 50, 0.7) per orbit, 101 snapshots "
            "float64")


def workload(n, seed):
    rng = np.random.default_rng(seed)
    R = np.exp(rng.uniform(np.log(0.05), np.log(3.0), n))
    vR = rng.normal(0, 0.1, n)
    vT = 1 + rng.normal(0, 0.1, n)
    z = rng.normal(0, 0.05, n)
    vz = rng.normal(0, 0.05, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    tend = np.exp(rng.normal(np.log(50.0), 0.7, n))
    ics = np.stack([R, vR, vT, z, vz, phi], 1)
    t = np.linspace(0.0, 1.0, NT)[None, :] * tend[:, None]
    return ics, t


def precision_workload(n, seed=2):
    """The precision configuration: config-0 style initial conditions,
    symplec4 with dt = 0.01 for 20,000 steps, final state only."""
    rng = np.random.default_rng(seed)
    R = rng.uniform(0.5, 2.0, n)
    ics = np.stack([R, rng.normal(0, 0.1, n), 1 + rng.normal(0, 0.1, n),
                    rng.normal(0, 0.05, n), rng.normal(0, 0.05, n),
                    rng.uniform(0, 2 * np.pi, n)], 1)
    return ics, np.array([0.0, 200.0])


def ragged_workload(seed=4, ngroup=512):
    """The ragged multi-potential configuration: 512 MWPotential2014 variants
    (MiyamotoNagai a, b, NFW a and the three amplitudes each scaled by
    U(0.8, 1.2)), U(1024, 16384) orbits per variant with config-0 initial
    conditions, DOP853 rtol = 1e-9, t in [0, 50], 51 snapshots."""
    import galpy_b200 as gb

    rng = np.random.default_rng(seed)
    _, pt, pa = gb.parse_pot(gb.MWPotential2014())
    args = np.tile(pa, (ngroup, 1))
    scale = rng.uniform(0.8, 1.2, (ngroup, 6))
    args[:, 6] *= scale[:, 0]  # MiyamotoNagai a
    args[:, 7] *= scale[:, 1]  # MiyamotoNagai b
    args[:, 9] *= scale[:, 2]  # NFW a
    args[:, 0] *= scale[:, 3]  # bulge amplitude
    args[:, 5] *= scale[:, 4]  # disk amplitude
    args[:, 8] *= scale[:, 5]  # halo amplitude
    counts = rng.integers(1024, 16385, ngroup)
    group = np.repeat(np.arange(ngroup), counts).astype(np.int32)
    ics, _ = precision_workload(len(group), seed=seed)
    return pt, args, group, ics, np.linspace(0.0, 50.0, 51)


def over_ranks(maxed, summed, pg, device):
    """Device times are reduced with MAX and work counts with SUM over the
    ranks of the process group (identity on one rank): the job's throughput is
    the work of all ranks over the slowest rank's time."""
    if pg is None:
        return [float(v) for v in maxed], [float(v) for v in summed]
    import torch

    mx = torch.tensor([float(v) for v in maxed], dtype=torch.float64, device=device)
    sm = torch.tensor([float(v) for v in summed], dtype=torch.float64, device=device)
    pg.all_reduce(mx, op=pg.ReduceOp.MAX)
    pg.all_reduce(sm, op=pg.ReduceOp.SUM)
    return mx.tolist(), sm.tolist()


def shard_seed(base, rank):
    """Seed of a rank's shard: every rank integrates its own orbits (weak
    scaling, no data exchange)."""
    return base + 1000 * rank


def differentiation_workload(n=65536, seed=3):
    """The differentiation configuration: n planar orbits in MWPotential2014
    (config-0 style initial conditions with z = vz = 0) as rectangular (x, y,
    vx, vy), DOP853 rtol = atol = 1e-10 over t in [0, 20], and seeded targets
    for L = sum |y(20) - target|^2."""
    def planar_rect(seed_):
        rng = np.random.default_rng(seed_)
        R = rng.uniform(0.5, 2.0, n)
        vR = rng.normal(0, 0.1, n)
        vT = 1 + rng.normal(0, 0.1, n)
        rng.normal(0, 0.05, n)  # z and vz of the 3D generator: zero in the plane
        rng.normal(0, 0.05, n)
        phi = rng.uniform(0, 2 * np.pi, n)
        c, s = np.cos(phi), np.sin(phi)
        return np.stack([R * c, R * s, vR * c - vT * s, vR * s + vT * c], 1)

    return planar_rect(seed), planar_rect(seed + 100)


def stats(x):
    x = np.asarray(x)
    return {"median": float(np.median(x)), "p99": float(np.quantile(x, 0.99)),
            "max": float(np.max(x))}


def mw14_args():
    import galpy_b200 as gb

    _, pt, pa = gb.parse_pot(gb.MWPotential2014())
    return pt, pa


def cyl_to_rect(v):
    R, vR, vT, z, vz, phi = v.T
    c, s = np.cos(phi), np.sin(phi)
    return np.stack([R * c, R * s, z, vR * c - vT * s, vR * s + vT * c, vz], 1)


# ---------------------------------------------------------------- clocks --
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.dev)], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        loaded = [s for s in sm if s > 0.5 * smax] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows
                                                         if r[3].replace(".", "").isdigit())}


# ----------------------------------------------------------- CPU baseline --
def cpu_reference_rate(ics, t, pt, pa, target_s=10.0, min_orbits=512, method="dop853",
                       rtol=RTOL, atol=ATOL, dt=None, planar=False):
    """orbit-steps/s of the reference's C (oracle/_ref) or the oracle, all cores."""
    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    n = min_orbits
    rng = np.random.default_rng(123)
    while True:
        idx = rng.choice(len(ics), size=min(n, len(ics)), replace=False)
        sub_ics, sub_t = ics[idx], (t[idx] if t.ndim > 1 else t)
        t0 = time.perf_counter()
        O.integrate(sub_ics, sub_t, pt, pa, method, rtol=rtol, atol=atol, dt=dt, planar=planar,
                    impl=("ref" if kind == "reference" else "port"), nthreads=cores)
        el = time.perf_counter() - t0
        if el >= 0.4 * target_s or n >= len(ics):
            break
        n = int(n * min(8.0, max(2.0, 0.5 * target_s / max(el, 1e-3))))
    # accepted steps of the same sample (the oracle is bit-identical to the
    # reference's C, so its counts are the reference's)
    _, _, ns, _ = O.integrate(sub_ics, sub_t, pt, pa, method, rtol=rtol, atol=atol, dt=dt,
                              planar=planar, nthreads=cores)
    steps = int(ns.sum())
    return {"value": steps / el, "unit": "orbit-steps/s", "cores": cores, "kind": kind,
            "sample": f"{len(idx)} random orbits of the workload ({steps} accepted steps, "
                      f"{el:.1f} s), OMP threads = {cores}"}


def cpu_reference_rate_groups(pt, args, group, ics, t, target_s=10.0, ngroups=8, rtol=1e-9,
                              atol=1e-9):
    """The reference's C on the ragged multi-potential workload: it takes one
    potential per call, so a random sample of the parameter groups is
    integrated group by group (all cores inside each call)."""
    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    rng = np.random.default_rng(321)
    gsel = rng.choice(len(args), size=ngroups, replace=False)
    per = 64
    while True:
        el, steps, norb = 0.0, 0, 0
        for g in gsel:
            idx = np.flatnonzero(group == g)
            idx = rng.choice(idx, size=min(per, len(idx)), replace=False)
            t0 = time.perf_counter()
            O.integrate(ics[idx], t, pt, args[g], "dop853", rtol=rtol, atol=atol,
                        impl=("ref" if kind == "reference" else "port"), nthreads=cores)
            el += time.perf_counter() - t0
            _, _, ns, _ = O.integrate(ics[idx], t, pt, args[g], "dop853", rtol=rtol, atol=atol,
                                      nthreads=cores)
            steps += int(ns.sum())
            norb += len(idx)
        if el >= 0.4 * target_s or per >= 16384:
            break
        per = int(per * min(8.0, max(2.0, 0.5 * target_s / max(el, 1e-3))))
    return {"value": steps / el, "unit": "orbit-steps/s", "cores": cores, "kind": kind,
            "sample": f"{norb} random orbits of {ngroups} random parameter groups, one call per "
                      f"group ({steps} accepted steps, {el:.1f} s), OMP threads = {cores}"}


def cpu_reference_gradient_rate(w0, tgt, pt, pa, idx, target_s=10.0):
    """What the reference needs for the same gradients on a sample of the
    differentiation workload: dL/d(initial state) from its variational
    integrator (integratePlanarOrbit_dxdv, one call per orbit and deviation
    direction: the 4 columns of the state-transition matrix), and
    dL/d(parameters) by central differences (2 integrations of every orbit
    per parameter).  Threads over orbits for the single-orbit dxdv calls
    (ctypes releases the interpreter lock); the batched calls use OpenMP.
    Returns orbit-steps/s in the differentiation leg's unit: accepted
    forward steps of the sample over that time."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    impl = "ref" if kind == "reference" else "port"
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    t = np.array([0.0, 20.0])
    rng = np.random.default_rng(77)

    def cyl(w):
        x, y, vx, vy = w.T
        phi = np.arctan2(y, x)
        c, s = np.cos(phi), np.sin(phi)
        return np.stack([np.hypot(x, y), vx * c + vy * s, -vx * s + vy * c, phi], 1)

    n = 32
    while True:
        sel = rng.choice(len(w0), size=min(n, len(w0)), replace=False)
        w, ics = w0[sel], cyl(w0[sel])
        t0 = time.perf_counter()
        # state-transition matrix columns: one variational run per direction
        rows = [np.concatenate([w[i], np.eye(4)[k]]) for i in range(len(w)) for k in range(4)]

        def one(r):
            return O.integrate_dxdv(r[None], t, pt, pa, "dop853", planar=True, rtol=1e-10,
                                    atol=1e-10, impl=impl)[0]

        with ThreadPoolExecutor(max_workers=cores) as ex:
            list(ex.map(one, rows))
        # parameters: central differences of the whole sample's loss
        for j in idx:
            for sgn in (1, -1):
                p = np.array(pa, float)
                p[j] += sgn * 1e-6 * abs(pa[j])
                O.integrate(ics, t, pt, p, "dop853", planar=True, rtol=1e-10, atol=1e-10,
                            impl=impl, nthreads=cores)
        el = time.perf_counter() - t0
        if el >= 0.4 * target_s or n >= len(w0):
            break
        n = int(n * min(8.0, max(2.0, 0.5 * target_s / max(el, 1e-3))))
    _, _, ns, _ = O.integrate(ics, t, pt, pa, "dop853", planar=True, rtol=1e-10, atol=1e-10,
                              nthreads=cores)
    steps = int(ns.sum())
    return {"value": steps / el, "unit": "orbit-steps/s (forward + backward)", "cores": cores,
            "kind": kind,
            "sample": f"{len(sel)} random orbits: 4 variational dop853 runs per orbit "
                      f"(integratePlanarOrbit_dxdv, {cores} threads over orbits) and "
                      f"{2 * len(idx)} perturbed integrations of the sample for the "
                      f"{len(idx)} parameters (central differences), {steps} accepted forward "
                      f"steps, {el:.1f} s"}


# ------------------------------------------------------------------ main --
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="galpy_b200", choices=["galpy_b200", "reference"])
    ap.add_argument("--orbits", type=int, default=N_ORBITS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--mixed-orbits", type=int, default=1 << 22)
    ap.add_argument("--no-ragged", action="store_true")
    ap.add_argument("--no-grad", action="store_true")
    ap.add_argument("--no-interp", action="store_true",
                    help="skip the orbit-interpolation leg (Orbit.__call__ between times)")
    ap.add_argument("--interp-only", action="store_true",
                    help="run only the orbit-interpolation leg (with --interp-orbits "
                         "orbits, --steps timed calls after --warmup)")
    ap.add_argument("--interp-orbits", type=int, default=1 << 20)
    ap.add_argument("--grad-only", action="store_true",
                    help="run only the differentiation leg (with --grad-orbits orbits)")
    ap.add_argument("--grad-orbits", type=int, default=65536)
    ap.add_argument("--methods-only", action="store_true",
                    help="run only the integrator comparison leg: all seven integrators "
                         "on the same batch, each beside the reference's C on a sample")
    ap.add_argument("--profile", default=None,
                    help="profiling case (for ncu): METHOD[:KIND], KIND one of plain, "
                         "groups, variational, sos; runs one warm-up and one launch of that "
                         "kernel on a small batch (--orbits, default 65,536) and prints its "
                         "time, nothing else")
    ap.add_argument("--variant", type=int, default=None,
                    help="pin the register variant of the headline kernel (0 compiler "
                         "budget, 1 capped) instead of the autotuner's choice")
    ap.add_argument("--block", type=int, default=None,
                    help="pin the headline kernel's orbits per block (DOP853: 128 or 96) "
                         "instead of the autotuner's choice")
    ap.add_argument("--out-layout", default="aos_rect", choices=["soa_rect", "aos_rect"],
                    help="snapshot layout of the headline and --profile runs: [N][nt][6] "
                         "(aos_rect, galpy's row order: one orbit's rows are contiguous, so "
                         "its partial 32-byte sectors merge in L2; the default) or "
                         "[6][nt][N] (soa_rect: four orbits share each sector, written at "
                         "different times, 4.7x the DRAM traffic)")
    ap.add_argument("--case", default="batching",
                    choices=["batching", "uniform", "longest", "bulk"],
                    help="uniform: R ~ U(0.5, 2), shared t in [0, 50] (101 snapshots) "
                         "(a throughput-bound case for profiling the same kernel); longest: "
                         "only the --orbits longest orbits of the batching workload (by "
                         "t_end / r0), the tail that bounds its step time; bulk: the "
                         "batching workload without its --orbits longest orbits")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, world, rank)

    import torch

    from galpy_b200 import _lib
    from galpy_b200 import build as gbuild
    import galpy_b200 as gb

    gbuild.build()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
        pg = dist

    if args.profile:
        n = args.orbits if args.orbits != N_ORBITS else 65536
        print(json.dumps(profile_leg(gb, torch, dev, args.profile, n, args.out_layout)),
              flush=True)
        return

    if args.grad_only:
        peak = ctypes_fp64_peak(_lib)
        res = differentiation_leg(gb, torch, dev, torch.cuda.current_stream(dev), pg, peak,
                                  n=args.grad_orbits)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        if rank == 0:
            print(json.dumps(res), flush=True)
        return

    if args.interp_only:
        res = interp_leg(gb, torch, dev, torch.cuda.current_stream(dev), pg,
                         n=args.interp_orbits, K=args.steps, W=args.warmup,
                         cpu=rank == 0 and not args.no_cpu_baseline)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        if rank == 0:
            print(json.dumps(res), flush=True)
        return

    if args.methods_only:
        res = methods_leg(gb, torch, dev, torch.cuda.current_stream(dev), pg,
                          ctypes_fp64_peak(_lib), rank, not args.no_cpu_baseline)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        if rank == 0:
            print(json.dumps(res), flush=True)
        return

    pt, pa = mw14_args()
    if args.case == "uniform":
        ics, _ = precision_workload(args.orbits, seed=shard_seed(1, rank))
        t = np.repeat(np.linspace(0.0, 50.0, NT)[None, :], len(ics), axis=0)
    elif args.case == "longest":
        ics, t = workload(N_ORBITS, seed=shard_seed(1, rank))
        r0 = np.sqrt(ics[:, 0] ** 2 + ics[:, 3] ** 2)
        keep = np.argsort(-t[:, -1] / r0)[:args.orbits]
        ics, t = ics[keep], t[keep]
    elif args.case == "bulk":
        ics, t = workload(N_ORBITS, seed=shard_seed(1, rank))
        r0 = np.sqrt(ics[:, 0] ** 2 + ics[:, 3] ** 2)
        keep = np.sort(np.argsort(-t[:, -1] / r0)[args.orbits:])
        ics, t = ics[keep], t[keep]
    else:
        ics, t = workload(args.orbits, seed=shard_seed(1, rank))
    n = len(ics)
    comps, ncomp = gb.compile_potential((pt, pa))
    sig = gb.signature((pt, pa))
    comps_d = torch.tensor(comps, device=dev)
    w0 = torch.tensor(cyl_to_rect(ics).T.copy(), device=dev)
    t_d = torch.tensor(t, device=dev)
    aos = args.out_layout == "aos_rect"
    out = torch.empty((n, NT, 6) if aos else (6, NT, n), dtype=torch.float64, device=dev)
    err = torch.empty(n, dtype=torch.int32, device=dev)
    nsteps = torch.empty(n, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)

    # launch shape chosen by the autotuner on a subsample of this batch, then
    # the whole integration (queue sort + persistent kernel) captured once in
    # a CUDA graph: every timed step is one graph launch
    from galpy_b200 import autotune
    from galpy_b200.graph import IntegrationGraph

    tuned = autotune.tune(comps_d, ncomp, w0, t_d, out, err, "dop853_cuda", rtol=RTOL,
                          atol=ATOL, signature=sig, comps_host=comps,
                          out_layout=args.out_layout)
    if args.variant is not None:
        tuned = dict(tuned, variant=args.variant, pinned_variant=True)
    if args.block is not None:
        tuned = dict(tuned, block_size=args.block, pinned_block=True)
    graph = IntegrationGraph(comps_d, ncomp, w0, t_d, out, err, "dop853_cuda", nsteps=nsteps,
                             rtol=RTOL, atol=ATOL, precision="fp64", signature=sig,
                             comps_host=comps, out_layout=args.out_layout,
                             **autotune.launch_kwargs(tuned))

    def run(precision="fp64"):
        graph.replay()

    def timed(precision, K, W):
        for _ in range(W):
            run(precision)
        torch.cuda.synchronize()
        steps = int(nsteps.sum().item())
        nbad = int((err != 0).sum().item())
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            run(precision)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if pg:
            pg.barrier()
        (ms,), (steps, nbad) = over_ranks([ms], [steps, nbad], pg, dev)
        return ms, steps, nbad

    clocks = ClockSampler(local)
    clocks.start()
    ms, steps, nbad = timed("fp64", args.steps, args.warmup)
    clk = clocks.stop()
    value = steps * args.steps / (ms * 1e-3)

    peak = ctypes_fp64_peak(_lib)
    achieved = value / world * F_STEP_DOP853 / 1e12  # per GPU
    result = {
        "metric": METRIC,
        "value": value,
        "unit": "orbit-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded initial conditions of the batching configuration)",
        "config": {"workload": WORKLOAD, "orbits_per_gpu": n, "snapshots": NT,
                   "accepted_steps_per_gpu_step": steps / world,
                   "orbits_with_err": nbad,
                   "launch": {"graph": "CUDA graph replay (cost pass, queue sort, persistent "
                                       "work-stealing kernel)",
                              **{k: tuned[k] for k in ("block_size", "variant", "schedule",
                                                       "threads_per_orbit")},
                              "autotune_sample_orbits": tuned.get("sample")},
                   "l2": "no flush: inputs (0.85 GB times) and outputs (5.1 GB snapshots) "
                         "exceed the 126 MB L2"},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     # DRAM read + write of a 65,536-orbit capture of this kernel
                     # with 101 snapshots per orbit (AoS rows: 0.549 GB; SoA rows:
                     # 3.833 GB), scaled by orbits x snapshots to this launch
                     "traffic": (0.549170e9 if aos else 3.833354e9) * n / 65536,
                     "traffic_algorithmic": n * NT * 6 * 8 + t.size * 8 + n * 6 * 8,
                     "traffic_source": "ncu capture of 65,536 orbits (uniform case, "
                                       f"{args.out_layout} snapshots), scaled by orbits x "
                                       "snapshots",
                     "out_layout": args.out_layout,
                     "kernel": "orbit_kernel<Dop853Machine<3,false>,3,0,false>",
                     "flops_per_unit": F_STEP_DOP853,
                     "peak_source": "measured in-process: float64 FMA-chain kernel "
                                    "(galpy_cuda_fp64_peak); MEASURED_PEAKS.json has no FP64 "
                                    "figure"},
        "clocks": clk,
        "gpu_launches": 2 * args.steps,  # cost_kernel + orbit_kernel per graph replay
    }

    # energy drift of the headline run (initial state vs final snapshot)
    E0 = torch.empty(n, dtype=torch.float64, device=dev)
    E1 = torch.empty(n, dtype=torch.float64, device=dev)
    gb.energy_device(comps_d, ncomp, w0, E0, stream=stream)
    gb.energy_device(comps_d, ncomp, out[:, NT - 1, :], E1, layout="aos" if aos else "soa",
                     stream=stream)
    torch.cuda.synchronize()
    result["energy_rel_err"] = stats((torch.abs(E1 / E0 - 1)).cpu().numpy())

    if not args.no_mixed:
        result["mixed"] = mixed_leg(gb, torch, dev, stream, comps_d, ncomp, sig, pt, pa, pg,
                                    args.mixed_orbits, comps,
                                    cpu=rank == 0 and not args.no_cpu_baseline)
        result["gpu_launches"] += 4
        # the FP32-force form of the batching workload's DOP853, on a sample
        result["f32force_sample"] = f32force_dop853_sample(gb, torch, dev, stream, "batching")
        result["gpu_launches"] += 4

    if not args.no_ragged:
        result["ragged"] = ragged_leg(gb, torch, dev, stream, pg,
                                      cpu=rank == 0 and not args.no_cpu_baseline)
        result["gpu_launches"] += result["ragged"]["gpu_launches"]

    if not args.no_grad:
        result["differentiation"] = differentiation_leg(
            gb, torch, dev, stream, pg, peak, n=args.grad_orbits,
            cpu=rank == 0 and not args.no_cpu_baseline)
        result["gpu_launches"] += 4

    if not args.no_e2e:
        result["e2e"] = e2e(gb, ics, t, pt, pa, args.steps, pg, dev, steps)
        result["gpu_launches"] += args.steps

    if not args.no_interp:
        result["interp"] = interp_leg(gb, torch, dev, stream, pg,
                                      cpu=rank == 0 and not args.no_cpu_baseline)
        result["gpu_launches"] += result["interp"]["gpu_launches"]

    if rank == 0 and not args.no_cpu_baseline:
        try:
            result["cpu_baseline"] = cpu_reference_rate(ics, t, pt, pa)
        except Exception as exc:  # report, do not hide
            result["cpu_baseline"] = {"value": None, "error": repr(exc)}
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


F_STEP_DOP853_PLANAR = 6200.0  # 15 planar force evaluations (280) + 2000 stage flops
F_GRAD_STEP = 3 * F_STEP_DOP853_PLANAR  # forward + backward (2 x forward: Hessian-vector products)


def interp_leg(gb, torch, dev, stream, pg, n=1 << 20, nt=NT, nq=NT - 1, K=3, W=3, cpu=False):
    """Orbits between their stored rows (galpy's Orbit.__call__ at times
    between the integration times): n orbits with nt galpy-layout rows on a
    shared grid t in [0, 50], evaluated at the nq midpoints of the grid, on
    the device (galpy_cuda_orbit_interp_device: not-a-knot cubic splines of
    x, y and the other components per orbit).  HBM bound: the algorithmic
    bytes are the rows read once and the outputs written once.  cpu: galpy's
    own route (scipy's RectBivariateSpline per component over (t, orbit
    index), then evaluation) on a sample, one host thread."""
    from galpy_b200.orbit_quantities import interpolate_device

    rng = np.random.default_rng(7)
    t = np.linspace(0.0, 50.0, nt)
    tq = 0.5 * (t[1:] + t[:-1])[:nq]
    # smooth synthetic rows of the batching workload's shape (the cost does
    # not depend on the values)
    f = rng.uniform(0.2, 2.0, (n, 1))
    ph = rng.uniform(0, 2 * np.pi, (n, 1))
    rows_h = np.empty((n, nt, 6))
    rows_h[..., 0] = 1.0 + 0.3 * np.sin(f * t[None, :] + ph)
    rows_h[..., 1] = 0.3 * f * np.cos(f * t[None, :] + ph)
    rows_h[..., 2] = 1.0 + 0.1 * np.cos(f * t[None, :])
    rows_h[..., 3] = 0.05 * np.sin(2 * f * t[None, :] + ph)
    rows_h[..., 4] = 0.1 * f * np.cos(2 * f * t[None, :] + ph)
    rows_h[..., 5] = np.mod(f * t[None, :] + ph, 2 * np.pi) - np.pi
    rows = torch.from_numpy(rows_h).to(dev)
    t_d = torch.from_numpy(t).to(dev)
    tq_d = torch.from_numpy(tq).to(dev)
    out = torch.empty((n, nq, 6), dtype=torch.float64, device=dev)
    for _ in range(W):
        interpolate_device(rows, t_d, tq_d, out, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        interpolate_device(rows, t_d, tq_d, out, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    (ms,), _ = over_ranks([ms], [], pg, dev)
    algo_bytes = n * (nt + nq) * 6 * 8
    res = {"workload": f"interpolation: {n} orbits x {nt} rows (6 components, shared t in "
                       f"[0, 50]) at the {nq} midpoints",
           "value": n * nq / (ms * 1e-3), "unit": "interpolated rows/s", "ms": ms,
           "algorithmic_bytes": algo_bytes,
           "achieved_GBs": algo_bytes / (ms * 1e-3) / 1e9,
           "gpu_launches": 4 * K}  # transpose, sweep, moments, evaluation
    if cpu:
        try:
            from scipy import interpolate as si

            m = 4096
            sub = rows_h[:m]
            c0 = time.perf_counter()
            x = sub[..., 0] * np.cos(sub[..., 5])
            y = sub[..., 0] * np.sin(sub[..., 5])
            comps = [x, sub[..., 1], sub[..., 2], sub[..., 3], sub[..., 4], y]
            idx = np.arange(m)
            vals = [si.RectBivariateSpline(t, idx, c.T, ky=1, s=0.0)(tq, idx) for c in comps]
            el = time.perf_counter() - c0
            ref = np.stack([np.sqrt(vals[0] ** 2 + vals[5] ** 2), vals[1], vals[2], vals[3],
                            vals[4], np.arctan2(vals[5], vals[0])], -1).transpose(1, 0, 2)
            got = out[:m].cpu().numpy()
            d = np.abs(got - ref)
            d[..., 5] = np.abs(np.mod(got[..., 5] - ref[..., 5] + np.pi, 2 * np.pi) - np.pi)
            res["cpu_baseline"] = {"value": m * nq / el, "unit": "interpolated rows/s",
                                   "cores": 1, "kind": "reference",
                                   "sample": f"{m} orbits through galpy's route (scipy "
                                             "RectBivariateSpline(kx=3, ky=1, s=0) per "
                                             f"component), {el:.2f} s",
                                   "max_abs_diff_vs_device": float(d.max())}
        except ImportError:
            res["cpu_baseline"] = {"unavailable": "scipy not importable"}
    return res


def differentiation_leg(gb, torch, dev, stream, pg, peak, n=65536, cpu=False):
    """Gradient of L = sum |y(20) - target|^2 over 65,536 planar orbits
    with respect to the initial conditions and the MiyamotoNagai (amp, a,
    b), NFW (amp, a) and bulge (amp, rc) parameters: adjoint forward +
    backward on the GPU, timed with CUDA events; the parameter gradient is
    checked against central differences (h = 1e-6 relative) of the loss with
    the forward pass's step sizes frozen."""
    from galpy_b200 import adjoint as adj

    _, pt, pa = gb.parse_pot(gb.MWPotential2014(), planar=True)
    w0, tgt = differentiation_workload(n, seed=shard_seed(3, pg.get_rank() if pg else 0))
    comps, ncomp = gb.compile_potential((pt, pa), planar=True)
    sig = gb.signature((pt, pa), planar=True)
    comps_d = torch.tensor(comps, device=dev)
    w = torch.tensor(w0.T.copy(), device=dev)
    tg = torch.tensor(tgt.T.copy(), device=dev)
    idx = adj.adjoint_params(pt, planar=True)
    times = []
    for rep in range(3):  # two warm-ups, one timed
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(stream)
        f = adj.adjoint_forward(comps_d, ncomp, w, 20.0, rtol=1e-10, atol=1e-10, planar=True,
                                signature=sig, ckpt_cap=16, stream=stream)
        ev[1].record(stream)
        gw, gp = adj.adjoint_backward(comps_d, ncomp, f, 2 * (f["yT"] - tg), 20.0, rtol=1e-10,
                                      atol=1e-10, planar=True, signature=sig, nparam=len(idx),
                                      stream=stream)
        gsum = gp.sum(dim=1)
        ev[2].record(stream)
        torch.cuda.synchronize()
        times.append((ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])))
    fwd_ms, bwd_ms = times[-1]
    steps = float(f["nsteps"].sum().item())
    nbad = int((f["err"] != 0).sum().item())
    # frozen-step central differences of the total loss
    fr = adj.adjoint_forward(comps_d, ncomp, w, 20.0, rtol=1e-10, atol=1e-10, planar=True,
                             signature=sig, ckpt_cap=16, record_steps=int(f["nsteps"].max()),
                             stream=stream)

    def loss(p):
        c = torch.tensor(gb.compile_potential((pt, p), planar=True)[0], device=dev)
        y = adj.adjoint_replay(c, ncomp, w, fr["hrec"], fr["nsteps"], 20.0, planar=True,
                               signature=sig, stream=stream)
        return float(((y - tg) ** 2).sum().item())

    fd = []
    for j in idx:
        h = 1e-6 * abs(pa[j])
        pp, pm = pa.copy(), pa.copy()
        pp[j] += h
        pm[j] -= h
        fd.append((loss(pp) - loss(pm)) / (2 * h))
    fd = np.array(fd)
    g = gsum.cpu().numpy()
    (ms_tot,), (steps_all, nbad_all) = over_ranks([fwd_ms + bwd_ms], [steps, nbad], pg, dev)
    value = steps_all / (ms_tot * 1e-3)
    achieved = value / (pg.get_world_size() if pg else 1) * F_GRAD_STEP / 1e12
    names = ["bulge amp", "bulge rc", "disk amp", "disk a", "disk b", "halo amp", "halo a"]
    res = {"workload": f"differentiation: {n} planar orbits in MWPotential2014, dop853 "
                       "rtol=atol=1e-10, t in [0,20], L = sum |y(20) - target|^2, gradient "
                       "w.r.t. initial conditions and 7 potential parameters",
           "value": value, "unit": "orbit-steps/s (forward + backward)",
           "forward_ms": fwd_ms, "backward_ms": bwd_ms, "accepted_steps": steps,
           "max_steps_per_orbit": int(f["nsteps"].max().item()), "orbits_with_err": nbad_all,
           "param_grad": dict(zip(names, g.tolist())),
           "param_grad_rel_err_vs_fd": float(np.max(np.abs(g - fd) / np.abs(fd))),
           "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak,
                        "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                        "flops_per_unit": F_GRAD_STEP,
                        "unit_of_work": "accepted forward step (forward + backward flops)"}}
    if cpu:
        try:
            res["cpu_baseline"] = cpu_reference_gradient_rate(w0, tgt, pt, pa, idx)
        except Exception as exc:  # report, do not hide
            res["cpu_baseline"] = {"value": None, "error": repr(exc)}
    return res


# Nominal float64 flops per step of each integrator in MWPotential2014 (3D,
# F_force = 300): kicks/drifts or stage combinations on top of the force
# evaluations per step (dopr54 and dop853: per accepted step).
METHOD_FLOPS = {"leapfrog": 318.0, "symplec4": 942.0, "symplec6": 2200.0, "rk4": 1260.0,
                "rk6": 2250.0, "dopr54": 2050.0, "dop853": F_STEP_DOP853}
METHODS_WORKLOAD = ("131,072 orbits/GPU in MWPotential2014, config-0 initial conditions "
                    "(R ~ U(0.5, 2)), t in [0, 100] with 101 snapshots, galpy's default "
                    "tolerances (rtol = atol = 1e-12) and estimated step, SoA float64 output")


def methods_leg(gb, torch, dev, stream, pg, peak, rank, cpu=True, n=131072, K=3, W=3):
    """Every integrator on the same batch: orbit-steps/s on the device (CUDA
    events, max over ranks) and the reference's C on a sample of the same
    orbits on all host cores."""
    pt, pa = mw14_args()
    ics, _ = precision_workload(n, seed=shard_seed(0, rank))
    t = np.linspace(0.0, 100.0, 101)
    comps, ncomp = gb.compile_potential((pt, pa))
    sig = gb.signature((pt, pa))
    comps_d = torch.tensor(comps, device=dev)
    w0 = torch.tensor(cyl_to_rect(ics).T.copy(), device=dev)
    t_d = torch.tensor(t, device=dev)
    out = torch.empty((6, len(t), n), dtype=torch.float64, device=dev)
    err = torch.empty(n, dtype=torch.int32, device=dev)
    nsteps = torch.empty(n, dtype=torch.int64, device=dev)
    world = pg.get_world_size() if pg else 1
    res = {"workload": METHODS_WORKLOAD, "n_gpus": world, "steps": K, "warmup": W,
           "per_method": {}}
    from galpy_b200 import autotune

    for m, flops in METHOD_FLOPS.items():
        # launch shape (orbits per block, register budget) from the autotuner,
        # as for the headline
        tuned = autotune.tune(comps_d, ncomp, w0, t_d, out, err, m + "_cuda", signature=sig,
                              comps_host=comps)
        kw = autotune.launch_kwargs(tuned)

        def run():
            gb.integrate_device(comps_d, ncomp, w0, t_d, out, err, m + "_cuda", nsteps=nsteps,
                                signature=sig, comps_host=comps, stream=stream, **kw)

        for _ in range(W):
            run()
        torch.cuda.synchronize()
        steps = int(nsteps.sum().item())
        nbad = int((err != 0).sum().item())
        if pg:
            pg.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            run()
        e1.record(stream)
        torch.cuda.synchronize()
        (ms,), (steps, nbad) = over_ranks([e0.elapsed_time(e1)], [steps, nbad], pg, dev)
        rate = steps * K / (ms * 1e-3)
        entry = {"value": rate, "unit": "orbit-steps/s", "ms_per_step": ms / K,
                 "steps_per_batch": steps, "orbits_with_err": nbad,
                 "launch": {k: tuned[k] for k in ("block_size", "variant")},
                 "flops_per_step": flops,
                 "fp64_frac_of_measured_peak": rate / world * flops / 1e12 / peak if peak
                 else None}
        if cpu and rank == 0:
            try:
                c = cpu_reference_rate(ics, t, pt, pa, target_s=4.0, min_orbits=64, method=m,
                                       rtol=None, atol=None)
                entry["cpu_reference"] = c
                entry["vs_cpu_reference"] = rate / c["value"]
            except Exception as exc:  # report, do not hide
                entry["cpu_reference"] = {"value": None, "error": repr(exc)}
        res["per_method"][m] = entry
    # cost pass + orbit kernel per timed or warm-up run (the autotuner's trial
    # launches come before)
    res["gpu_launches"] = 2 * (K + W) * len(METHOD_FLOPS)
    return res


def scf_expansion_args(N=8, L=6, a=1.1, seed=3):
    """galpy's SCFPotential arguments (a, isNonAxi, N, L, M, Nt = 0, Acos,
    Asin, 11 cache slots) of a seeded non-axisymmetric expansion: the
    (0, 0, 0) term 1, the m <= l others ~N(0, 0.05)."""
    rng = np.random.default_rng(seed)
    Acos = rng.normal(size=(N, L, L)) * 0.05
    Asin = rng.normal(size=(N, L, L)) * 0.05
    Acos[0, 0, 0] = 1.0
    for l in range(L):
        Acos[:, l, l + 1:] = 0.0
        Asin[:, l, l + 1:] = 0.0
    Asin[:, :, 0] = 0.0
    return np.concatenate([[a, 1.0, N, L, L, 0.0], Acos.ravel(), Asin.ravel(),
                           [-1.0] + [0.0] * 10])


def profile_leg(gb, torch, dev, spec, n, out_layout="soa_rect"):
    """One warm-up and one timed launch of a single kernel on a small batch,
    for profiler captures (`ncu -k regex:<machine> -s 1 -c 1`):

      plain        config-0 initial conditions (R ~ U(0.5, 2)), t in [0, 20]
                   with 101 snapshots, galpy's default tolerances 1e-12 and
                   estimated step, MWPotential2014 (compile-time list)
      groups       the same orbits split over 64 MWPotential2014 variants of
                   the ragged configuration (parameter-group kernel), dop853
                   rtol = atol = 1e-9
      variational  3D variational integration (12-D state, one unit
                   deviation per orbit), t in [0, 20], 21 rows
      sos          3D surface of section, psi in [0, 20 pi] with 21 rows
      uniform      R ~ U(0.5, 2) (seed 1), per-orbit copies of t in [0, 50]
                   with 101 snapshots, rtol = atol = 1e-10: the batching
                   workload's kernel on orbits of similar length
      bar          as plain, in MWPotential2014 plus a rotating
                   DehnenBarPotential (the full run-time list, whose force
                   reads the time)
      scf          as plain, in a non-axisymmetric SCF expansion (N = 8,
                   L = 6) plus MWPotential2014's disk (full run-time list)

    A third field selects the register variant and a fourth the orbits per
    block (METHOD:KIND:VARIANT[:BLOCK]).  out_layout: the snapshot layout
    ('soa_rect' or 'aos_rect')."""
    method, _, rest = spec.partition(":")
    kind, _, variant = rest.partition(":")
    variant, _, block = variant.partition(":")
    kind = kind or "plain"
    stream = torch.cuda.current_stream(dev)
    pt, pa = mw14_args()
    if kind == "bar":
        pt = np.append(pt, 1).astype(np.int32)
        pa = np.concatenate([pa, [0.01, -2.0, 3.0, 0.8, 1.85, 0.4]])
    elif kind == "scf":
        pt = np.array([24, 5], np.int32)
        pa = np.concatenate([scf_expansion_args(), pa[5:8]])
    ics, _ = precision_workload(n, seed=1 if kind == "uniform" else 5)
    kw = {"variant": int(variant or 0), "block_size": int(block or 0)}
    group = None
    if kind == "groups":
        pt, args, _, _, _ = ragged_workload(ngroup=512)
        args = args[:64]
        comps, ncomp = gb.compile_potential((pt, args.ravel()), ngroup=len(args))
        group = torch.tensor(np.arange(n, dtype=np.int32) % len(args), device=dev)
        sig = gb.signature((pt, args[0]))
        kw.update(rtol=1e-9, atol=1e-9)
    else:
        comps, ncomp = gb.compile_potential((pt, pa))
        sig = gb.signature((pt, pa))
        if kind in ("plain", "uniform"):
            kw["comps_host"] = comps
    comps_d = torch.tensor(comps, device=dev)
    w = cyl_to_rect(ics)
    nv = 6
    t = np.linspace(0.0, 20.0, 101)
    if kind == "uniform":
        t = np.repeat(np.linspace(0.0, 50.0, NT)[None, :], n, axis=0)
        kw.update(rtol=RTOL, atol=ATOL)
    elif kind == "variational":
        w = np.concatenate([w, np.zeros((n, 6))], 1)
        w[np.arange(n), 6 + np.arange(n) % 6] = 1.0
        nv, t = 12, np.linspace(0.0, 20.0, 21)
        kw["variational"] = True
        sig = 0
    elif kind == "sos":
        # (x, y, vx, vy, A, t, psi) from the cylindrical initial conditions
        R, vR, vT, z, vz, phi = ics.T
        c, s = np.cos(phi), np.sin(phi)
        w = np.stack([R * c, R * s, vR * c - vT * s, vR * s + vT * c, np.hypot(z, vz),
                      np.zeros(n), np.arctan2(z, vz)], 1)
        nv, t = 7, np.linspace(0.0, 20 * np.pi, 21)
        kw["system"] = "sos"
        sig = 0
    w0 = torch.tensor(np.ascontiguousarray(w.T), device=dev)
    t_d = torch.tensor(t, device=dev)
    shape = (n, t.shape[-1], nv) if out_layout == "aos_rect" else (nv, t.shape[-1], n)
    out = torch.empty(shape, dtype=torch.float64, device=dev)
    kw["out_layout"] = out_layout
    err = torch.empty(n, dtype=torch.int32, device=dev)
    ns = torch.empty(n, dtype=torch.int64, device=dev)
    ms = []
    for rep in range(2):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        gb.integrate_device(comps_d, ncomp, w0, t_d, out, err, method + "_cuda", nsteps=ns,
                            group=group, signature=sig, stream=stream, **kw)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return {"profile": spec, "orbits": n, "ms": ms[-1],
            "accepted_steps": float(ns.sum().item()),
            "orbits_with_err": int((err != 0).sum().item())}


def ragged_leg(gb, torch, dev, stream, pg, K=3, W=2, cpu=False):
    """One launch over 512 potential-parameter groups (about 4.3 M orbits):
    the launch shape from the autotuner (on a subsample, parameter groups
    included), the integration captured in a CUDA graph, W warm-up and K
    timed replays (CUDA events, max over ranks).  Also: the FP32-force
    variant on a sample of 8 groups, and the reference's C on a sample of
    groups (cpu)."""
    from galpy_b200 import autotune
    from galpy_b200.graph import IntegrationGraph

    pt, args, group, ics, t = ragged_workload()
    n = len(group)
    comps, ncomp = gb.compile_potential((pt, args.ravel()), ngroup=len(args))
    comps_d = torch.tensor(comps, device=dev)
    sig = gb.signature((pt, args[0]))
    w0 = torch.tensor(cyl_to_rect(ics).T.copy(), device=dev)
    t_d = torch.tensor(t, device=dev)
    g_d = torch.tensor(group, device=dev)
    out = torch.empty((6, len(t), n), dtype=torch.float64, device=dev)
    err = torch.empty(n, dtype=torch.int32, device=dev)
    ns = torch.empty(n, dtype=torch.int64, device=dev)
    tuned = autotune.tune(comps_d, ncomp, w0, t_d, out, err, "dop853_cuda", rtol=1e-9, atol=1e-9,
                          signature=sig, group=g_d)
    graph = IntegrationGraph(comps_d, ncomp, w0, t_d, out, err, "dop853_cuda", nsteps=ns,
                             group=g_d, rtol=1e-9, atol=1e-9, signature=sig,
                             **autotune.launch_kwargs(tuned))
    for _ in range(W):
        graph.replay()
    torch.cuda.synchronize()
    steps = float(ns.sum().item())
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    (ms,), (steps_all,) = over_ranks([e0.elapsed_time(e1) / K], [steps], pg, dev)
    E0 = torch.empty(n, dtype=torch.float64, device=dev)
    E1 = torch.empty(n, dtype=torch.float64, device=dev)
    gb.energy_device(comps_d, ncomp, w0, E0, group=g_d, stream=stream)
    gb.energy_device(comps_d, ncomp, out[:, len(t) - 1, :], E1, group=g_d, stream=stream)
    torch.cuda.synchronize()
    rel = torch.abs(E1 / E0 - 1).cpu().numpy()
    E0h = E0.cpu().numpy()
    res = {"workload": f"ragged: {len(args)} MWPotential2014 variants, {n} orbits, dop853 "
                       "rtol=atol=1e-9, t in [0,50], 51 snapshots, one launch",
           "value": steps_all / (ms * 1e-3), "unit": "orbit-steps/s", "ms": ms, "steps": K,
           "warmup": W, "launch": {"graph": "CUDA graph replay",
                                   **autotune.launch_kwargs(tuned)},
           "accepted_steps": steps, "orbits_with_err": int((err != 0).sum().item()),
           "energy_rel_err": stats(rel),
           # the largest relative drifts belong to orbits whose energy is
           # close to zero (|E0| small makes |E1/E0 - 1| large for the same
           # absolute error): the absolute drift of the worst orbits
           "energy_worst": {"rel": float(rel.max()), "E0": float(E0h[rel.argmax()]),
                            "abs_err_max": float(np.abs(rel * E0h).max())},
           "gpu_launches": 2 * (K + W)}
    res["f32force_sample"] = f32force_dop853_sample(gb, torch, dev, stream, "ragged")
    if cpu:
        try:
            res["cpu_baseline"] = cpu_reference_rate_groups(pt, args, group, ics, t)
        except Exception as exc:  # report, do not hide
            res["cpu_baseline"] = {"value": None, "error": repr(exc)}
    graph.reset()
    return res


# the precision forms of the engine (include/galpy_cuda.h), in the order
# the mixed leg reports them; the first is the plain float64 reference form
PRECISION_FORMS = ("fp64", "f32force", "f64tail32", "f32bulge", "f32force_df")


def mixed_leg(gb, torch, dev, stream, comps_d, ncomp, sig, pt, pa, pg, n, comps_host=None,
              cpu=False):
    """The precision forms on the precision configuration (symplec4, dt =
    0.01, 20,000 steps, final state only), each at its own autotuned launch
    shape: throughput and its ratio to the plain float64 kernel, the
    per-orbit relative energy drift, and the final phase-space difference
    from the float64 kernel and from the float64 oracle (on a sample).
    Forms: fp64 (float64 force and state), f32force (float32 force, float64
    state), f64tail32 (float64 force with float32 tails of its table
    polynomials), f32bulge (f64tail32 with the bulge term in float32),
    f32force_df (float32 force, double-float state)."""
    ics, t = precision_workload(n)
    w0 = torch.tensor(cyl_to_rect(ics).T.copy(), device=dev)
    t_d = torch.tensor(t, device=dev)
    E0 = torch.empty(n, dtype=torch.float64, device=dev)
    gb.energy_device(comps_d, ncomp, w0, E0, stream=stream)
    from galpy_b200 import autotune

    res = {}
    outs = {}
    for prec in PRECISION_FORMS:
        out = torch.empty((6, 1, n), dtype=torch.float64, device=dev)
        err = torch.empty(n, dtype=torch.int32, device=dev)
        ns = torch.empty(n, dtype=torch.int64, device=dev)
        # each form at its own best launch shape
        tuned = autotune.tune(comps_d, ncomp, w0, t_d, out, err, "symplec4_cuda", dt=0.01,
                              out_row0=1, precision=prec, signature=sig, comps_host=comps_host)
        ms_list = []
        for rep in range(2):  # warm-up + timed
            if pg:
                pg.barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            gb.integrate_device(comps_d, ncomp, w0, t_d, out, err, "symplec4_cuda", nsteps=ns,
                                dt=0.01, out_row0=1, precision=prec, stream=stream,
                                signature=sig, comps_host=comps_host,
                                **autotune.launch_kwargs(tuned))
            e1.record(stream)
            torch.cuda.synchronize()
            ms_list.append(e0.elapsed_time(e1))
        E1 = torch.empty(n, dtype=torch.float64, device=dev)
        gb.energy_device(comps_d, ncomp, out[:, 0, :], E1, stream=stream)
        torch.cuda.synchronize()
        steps = float(ns.sum().item())
        (ms,), (steps,) = over_ranks([ms_list[-1]], [steps], pg, dev)
        res[prec] = {"value": steps / (ms * 1e-3), "unit": "orbit-steps/s", "ms": ms,
                     "launch": autotune.launch_kwargs(tuned),
                     "energy_rel_err": stats(torch.abs(E1 / E0 - 1).cpu().numpy()),
                     "orbits_with_err": int((err != 0).sum().item())}
        outs[prec] = out[:, 0, :]
    scale = torch.abs(outs["fp64"]).max(dim=0).values
    for prec in PRECISION_FORMS[1:]:
        d = torch.abs(outs[prec] - outs["fp64"]).max(dim=0).values
        res[prec]["phase_space_rel_err_vs_fp64"] = stats((d / scale).cpu().numpy())
        res[prec]["speedup_vs_fp64"] = res[prec]["value"] / res["fp64"]["value"]
    res["speedup_f32force_vs_fp64"] = res["f32force"]["speedup_vs_fp64"]
    res["workload"] = (f"precision: {n} orbits in MWPotential2014 (config-0 initial "
                       "conditions), symplec4 dt=0.01, 20,000 steps, final state only")
    # every form against the FP64 oracle (the reference's arithmetic) on a
    # sample: final phase-space difference and the oracle's own energy drift
    from oracle import oracle as O

    m = min(n, 1024)
    ref, eref, _, _ = O.integrate(ics[:m], t, pt, pa, "symplec4", dt=0.01)
    ref_rect = cyl_to_rect(ref[:, -1])
    for prec in PRECISION_FORMS:
        g = outs[prec][:, :m].cpu().numpy().T
        dd = np.abs(g - ref_rect).max(axis=1) / np.abs(ref_rect).max(axis=1)
        res[prec]["phase_space_rel_err_vs_oracle"] = stats(dd)
    e0 = O.energy_cyl(ics[:m, None], pt, pa)[:, 0]
    e1 = O.energy_cyl(ref[:, -1:], pt, pa)[:, 0]
    res["oracle_sample"] = {"orbits": m, "energy_rel_err": stats(np.abs(e1 / e0 - 1)),
                            "kind": "oracle (C restatement of galpy's symplec4, bit-identical "
                                    "to the reference's C)"}
    if cpu:  # the reference's C symplec4 (float64) on a sample, all cores
        try:
            res["cpu_baseline"] = cpu_reference_rate(ics, t, pt, pa, method="symplec4",
                                                     dt=0.01, min_orbits=64)
        except Exception as exc:  # report, do not hide
            res["cpu_baseline"] = {"value": None, "error": repr(exc)}
    return res


def rect_to_cyl(w):
    x, y, z, vx, vy, vz = w.T
    phi = np.arctan2(y, x)
    c, s = np.cos(phi), np.sin(phi)
    return np.stack([np.hypot(x, y), vx * c + vy * s, -vx * s + vy * c, z, vz, phi], 1)


def f32force_dop853_sample(gb, torch, dev, stream, kind, n_sample=4096, budget=2_000_000):
    """The precision forms of DOP853 beside float64 on a random sample of the
    batching (kind "batching": rtol = atol = 1e-10) or ragged ("ragged":
    1e-9, 8 parameter groups) workload: f32force (float32 force; DOP853's
    error estimate sees the single-precision force rounding, so its step
    count grows), f64tail32 and f32bulge.  Per form: the accepted-step ratio
    and speed ratio to float64, the relative energy drift and the final
    phase-space difference.  A per-orbit attempt budget bounds the run;
    orbits that exhaust it (err 2) in any form are counted and left out of
    the error statistics."""
    rng = np.random.default_rng(99)
    group_d = None
    if kind == "batching":
        pt, pa = mw14_args()
        ics, t = workload(N_ORBITS, seed=1)
        sel = rng.choice(len(ics), size=n_sample, replace=False)
        ics, t = ics[sel], t[sel]
        comps, ncomp = gb.compile_potential((pt, pa))
        sig = gb.signature((pt, pa))
        tol = RTOL
        last = NT - 1
    else:
        pt, args, group, ics_all, t = ragged_workload()
        gsel = rng.choice(len(args), size=8, replace=False)
        idx = np.concatenate([rng.choice(np.flatnonzero(group == g),
                                         size=n_sample // 8, replace=False) for g in gsel])
        ics = ics_all[idx]
        slot_of = {int(g): k for k, g in enumerate(gsel)}
        grp = np.array([slot_of[int(g)] for g in group[idx]], np.int32)
        comps, ncomp = gb.compile_potential((pt, args[gsel].ravel()), ngroup=len(gsel))
        sig = gb.signature((pt, args[0]))
        group_d = torch.tensor(grp, device=dev)
        tol = 1e-9
        last = len(t) - 1
    n = len(ics)
    comps_d = torch.tensor(comps, device=dev)
    w0 = torch.tensor(cyl_to_rect(ics).T.copy(), device=dev)
    t_d = torch.tensor(t, device=dev)
    E0 = torch.empty(n, dtype=torch.float64, device=dev)
    gb.energy_device(comps_d, ncomp, w0, E0, group=group_d, stream=stream)
    res, fin, steps, errs, ms = {}, {}, {}, {}, {}
    forms = ("fp64", "f32force", "f64tail32", "f32bulge")
    for prec in forms:
        out = torch.empty((6, 1, n), dtype=torch.float64, device=dev)
        err = torch.empty(n, dtype=torch.int32, device=dev)
        ns = torch.empty(n, dtype=torch.int64, device=dev)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        gb.integrate_device(comps_d, ncomp, w0, t_d, out, err, "dop853_cuda", nsteps=ns,
                            group=group_d, out_row0=last, rtol=tol, atol=tol, precision=prec,
                            max_attempts=budget, signature=sig, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms[prec] = e0.elapsed_time(e1)
        fin[prec] = out[:, 0, :]
        steps[prec] = ns.cpu().numpy()
        errs[prec] = err.cpu().numpy()
    ok = np.logical_and.reduce([errs[p] == 0 for p in forms])
    for prec in forms:
        E1 = torch.empty(n, dtype=torch.float64, device=dev)
        gb.energy_device(comps_d, ncomp, fin[prec], E1, group=group_d, stream=stream)
        torch.cuda.synchronize()
        rel = torch.abs(E1 / E0 - 1).cpu().numpy()
        res[prec] = {"accepted_steps": float(steps[prec].sum()), "ms": ms[prec],
                     "orbits_with_err": int((errs[prec] != 0).sum()),
                     "energy_rel_err": stats(rel[ok]) if ok.any() else None}
        if prec == "fp64":
            continue
        d = (torch.abs(fin[prec] - fin["fp64"]).max(dim=0).values /
             torch.abs(fin["fp64"]).max(dim=0).values).cpu().numpy()
        res[prec]["phase_space_rel_err_vs_fp64"] = stats(d[ok]) if ok.any() else None
        res[prec]["accepted_step_ratio_vs_fp64"] = float(
            steps[prec][ok].sum() / max(1, steps["fp64"][ok].sum()))
        res[prec]["speed_ratio_vs_fp64_orbits_per_s"] = ms["fp64"] / ms[prec]
    res["accepted_step_ratio_f32force_vs_fp64"] = res["f32force"]["accepted_step_ratio_vs_fp64"]
    res["sample"] = (f"{n} random orbits of the {kind} workload" +
                     (" (8 random parameter groups)" if kind == "ragged" else "") +
                     f", dop853 rtol = atol = {tol:g}, attempt budget {budget} per orbit")
    return res


def e2e(gb, ics, t, pt, pa, K, pg, dev, steps_total):
    """The galpy-facing C ABI from pinned host memory (copies timed)."""
    import torch

    n = len(ics)
    yo_pin = torch.empty((n, 6), dtype=torch.float64, pin_memory=True).numpy()
    t_pin = torch.empty(t.shape, dtype=torch.float64, pin_memory=True).numpy()
    res_pin = torch.empty((n, NT, 6), dtype=torch.float64, pin_memory=True).numpy()
    t_pin[:] = t
    import ctypes

    from galpy_b200 import _lib

    L = _lib.lib()
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    err = np.zeros(n, np.int32)
    pti = np.ascontiguousarray(pt, np.int32)
    pad = np.ascontiguousarray(pa, np.float64)
    r, a = float(np.log(RTOL)), float(np.log(ATOL))
    kernel_ms = ctypes.c_double(0.0)
    opts = _lib.make_opts(device=dev.index, elapsed=kernel_ms)
    times, kernel = [], []
    for k in range(K + 1):
        yo_pin[:] = ics  # galpy's call overwrites yo with rectangular coordinates
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        rc = L.integrateFullOrbit_cuda(n, yo_pin.ctypes.data_as(dp), NT, t_pin.ctypes.data_as(dp),
                                       1, len(pti), pti.ctypes.data_as(ip), pad.ctypes.data_as(dp),
                                       None, -9999.99, r, a, res_pin.ctypes.data_as(dp),
                                       err.ctypes.data_as(ip), 6, _lib.CALLBACK(),
                                       ctypes.byref(opts))
        el = time.perf_counter() - t0
        _lib.check(rc)
        if k > 0:  # first call is a warm-up
            times.append(el)
            kernel.append(kernel_ms.value * 1e-3)
    (el,), _ = over_ranks([max(times)], [], pg, dev)
    # the same call with pageable numpy arrays, as galpy passes them
    # (integrateFullOrbit.py:708-712)
    yo_pg = np.empty((n, 6))
    t_pg = np.ascontiguousarray(t, dtype=np.float64)
    res_pg = np.empty((n, NT, 6))
    ptimes = []
    for k in range(K + 1):
        yo_pg[:] = ics
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        rc = L.integrateFullOrbit_cuda(n, yo_pg.ctypes.data_as(dp), NT, t_pg.ctypes.data_as(dp),
                                       1, len(pti), pti.ctypes.data_as(ip), pad.ctypes.data_as(dp),
                                       None, -9999.99, r, a, res_pg.ctypes.data_as(dp),
                                       err.ctypes.data_as(ip), 6, _lib.CALLBACK(),
                                       ctypes.byref(opts))
        pel = time.perf_counter() - t0
        _lib.check(rc)
        if k > 0:
            ptimes.append(pel)
    (pel,), _ = over_ranks([max(ptimes)], [], pg, dev)
    return {"value": steps_total / el, "unit": "orbit-steps/s", "seconds_per_step": el,
            "kernel_seconds_per_step": max(kernel),
            "h2d_bytes_per_step": int(yo_pin.nbytes + t_pin.nbytes),
            "d2h_bytes_per_step": int(res_pin.nbytes + err.nbytes),
            "api": "integrateFullOrbit_cuda (galpy layout, pinned host buffers)",
            "pageable": {"value": steps_total / pel, "seconds_per_step": pel,
                         "api": "integrateFullOrbit_cuda (galpy layout, pageable numpy "
                                "arrays as galpy passes them)"}}


def ctypes_fp64_peak(_lib):
    import ctypes

    tf, ms = ctypes.c_double(0), ctypes.c_double(0)
    rc = _lib.lib().galpy_cuda_fp64_peak(ctypes.byref(tf), ctypes.byref(ms))
    return tf.value if rc == 0 else None


def run_reference(args, world, rank):
    if rank != 0:
        return
    pt, pa = mw14_args()
    ics, t = workload(args.orbits, seed=1)
    vals = []
    base = None
    for k in range(args.warmup + args.steps):
        b = cpu_reference_rate(ics, t, pt, pa, target_s=10.0)
        if k >= args.warmup:
            vals.append(b["value"])
            base = b
    value = statistics.mean(vals)
    base = dict(base)
    base["value"] = value
    print(json.dumps({
        "metric": METRIC, "impl": "reference", "value": value, "unit": "orbit-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded initial conditions of the batching configuration)",
        "config": {"workload": WORKLOAD, "orbits_per_gpu": args.orbits, "snapshots": NT},
        "cpu_baseline": base,
        "e2e": {"value": value, "unit": "orbit-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


if __name__ == "__main__":
    main()
