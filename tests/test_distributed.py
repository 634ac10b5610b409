"""The multi-GPU plumbing on CPU: world_size-2 process groups over gloo.

Orbits shard across ranks with no data exchange in the integration; the
only collectives are the bench's reductions (MAX of device time, SUM of
work) and the sum of the potential-parameter gradient after the backward
pass (galpy_b200.adjoint.reduce_param_grad)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from galpy_b200.adjoint import reduce_param_grad

        # bench aggregation: slowest rank's time, all ranks' work
        (ms,), (steps, nbad) = bench.over_ranks([10.0 + rank], [100.0 * (rank + 1), rank], dist,
                                                "cpu")
        # shards: distinct seeds, hence distinct orbits
        ics, _ = bench.workload(4, seed=bench.shard_seed(1, rank))
        gathered = [torch.zeros(4, 6, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, torch.from_numpy(ics))
        distinct = not torch.equal(gathered[0], gathered[1])
        # parameter gradient: summed over ranks; IC gradients stay local
        g = torch.full((7,), float(rank + 1), dtype=torch.float64)
        reduce_param_grad(g)
        q.put((rank, ms, steps, nbad, distinct, g.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions_over_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, steps, nbad, distinct, g in out:
        assert ms == 11.0 and steps == 300.0 and nbad == 1.0
        assert distinct
        assert g == [3.0] * 7


def test_single_process_reductions_are_identity():
    import sys

    sys.path.insert(0, ROOT)
    import bench
    from galpy_b200.adjoint import reduce_param_grad

    assert bench.over_ranks([2.5], [7, 1], None, "cpu") == ([2.5], [7.0, 1.0])
    g = torch.ones(3, dtype=torch.float64)
    assert reduce_param_grad(g) is g and g.tolist() == [1.0] * 3
    with pytest.raises(Exception):
        bench.over_ranks([1.0], [1.0], object(), "cpu")


# --- orbit ranges of equal estimated cost (galpy_cuda_split_orbits) -------
# The multi-device call (opts.ndevices) and processes that share a batch
# (shard_of) cut it with the same host-side estimate; the cut needs no GPU.

def _sorted_batch(golden, n=20000, seed=5):
    """A batch ordered by radius (a grid of orbits in energy, as users make
    them), with ragged per-orbit end times: equal orbit counts per part
    would load the parts very unevenly."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import cyl_to_rect, seeded_ics

    ics = seeded_ics(n, seed, r_range=(0.05, 20.0), log_r=True)
    ics = ics[np.argsort(ics[:, 0])]
    rng = np.random.default_rng(seed)
    tend = np.exp(rng.normal(np.log(50.0), 0.5, n))
    t = np.linspace(0, 1, 11)[None, :] * tend[:, None]
    return cyl_to_rect(ics), t, (golden["mw14_type"], golden["mw14_args"])


def _oracle_costs(w, t, pot, oracle):
    """|t_end - t_0| * Omega(x_0) + 1e-3 with Omega^2 = |a.x| / |x|^2, from
    the oracle's forces (a.x = F_R R + F_z z: the azimuthal force is normal
    to x)."""
    R = np.hypot(w[:, 0], w[:, 1])
    z = w[:, 2]
    phi = np.arctan2(w[:, 1], w[:, 0])
    f = oracle.forces(R, z, phi, pot[0], pot[1])
    ax = f[:, 0] * R + f[:, 1] * z
    om = np.sqrt(np.abs(ax) / (R * R + z * z))
    return np.abs(t[:, -1] - t[:, 0]) * om + 1e-3


@pytest.mark.parametrize("nparts", [2, 3, 8])
def test_split_orbits_equal_cost(golden, oracle, nparts):
    import galpy_b200 as gb

    w, t, pot = _sorted_batch(golden)
    b = gb.split_orbits(pot, w, t, nparts)
    assert b[0] == 0 and b[-1] == len(w) and (np.diff(b) >= 0).all()
    cost = _oracle_costs(w, t, pot, oracle)
    share = np.array([cost[b[k]:b[k + 1]].sum() for k in range(nparts)])
    # each cut lands within half an orbit's cost of its target
    assert np.abs(share - cost.sum() / nparts).max() <= cost.max() * (1 + 1e-6)
    # the sorted batch is what the cost weighting is for: equal counts are
    # far from equal cost here
    eq = np.linspace(0, len(w), nparts + 1).astype(int)
    share_eq = np.array([cost[eq[k]:eq[k + 1]].sum() for k in range(nparts)])
    assert share_eq.max() / share_eq.min() > 2.0
    assert share.max() / share.min() < 1.01


def test_split_orbits_edges(golden):
    import galpy_b200 as gb
    from galpy_b200 import _lib

    w, t, pot = _sorted_batch(golden, n=50)
    # shared time grid, more parts than orbits, one part, empty batch
    b = gb.split_orbits(pot, w, t[0], 64)
    assert b[0] == 0 and b[-1] == 50 and (np.diff(b) >= 0).all()
    assert list(gb.split_orbits(pot, w, t, 1)) == [0, 50]
    assert list(gb.split_orbits(pot, w[:0], t[0], 4)) == [0] * 5
    # a single dominant orbit takes a part to itself
    t2 = t.copy()
    t2[17] *= 1e6
    b = gb.split_orbits(pot, w, t2, 2)
    assert b[1] in (17, 18)
    with pytest.raises(_lib.CudaError):
        gb.split_orbits(pot, w, t, 0)
    with pytest.raises(ValueError):
        gb.split_orbits(pot, w, t[:3], 2)


def _shard_worker(rank, world, port, q):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import galpy_b200 as gb

        golden = dict(np.load(os.path.join(ROOT, "tests", "golden", "golden.npz")))
        w, t, pot = _sorted_batch(golden, n=6000)
        start, stop = gb.shard_of(pot, w, t, rank, world)
        ranges = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(ranges, torch.tensor([start, stop], dtype=torch.int64))
        q.put((rank, [r.tolist() for r in ranges], gb.split_orbits(pot, w, t, world).tolist()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_a_batch_by_cost():
    """Each rank computes its own range from the same inputs with no
    exchange; the ranges tile the batch without overlap."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ranges, bounds in out:
        assert ranges == [[bounds[k], bounds[k + 1]] for k in range(world)]
        assert ranges[0][0] == 0 and ranges[-1][1] == 6000 and ranges[0][1] == ranges[1][0]
    assert out[0][1] == out[1][1]


def test_split_orbits_parameter_groups(oracle):
    """Parameter groups: each orbit's cost is taken in its own group's
    potential (here the halo amplitude differs by a factor 16 between the
    two halves of the groups, so the orbital frequencies differ by 4)."""
    import sys

    import galpy_b200 as gb

    sys.path.insert(0, ROOT)
    import bench

    pt, args, group, ics, t = bench.ragged_workload(seed=9, ngroup=8)
    args = args.copy()
    args[4:, 8] *= 16.0  # halo amplitude of groups 4..7
    order = np.argsort(group, kind="stable")
    group, ics = group[order], ics[order]
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import cyl_to_rect

    w = cyl_to_rect(ics)
    b = gb.split_orbits((pt, args.ravel()), w, t, 4, group=group, ngroup=len(args))
    cost = np.empty(len(w))
    for g in range(len(args)):
        sel = group == g
        cost[sel] = _oracle_costs(w[sel], np.broadcast_to(t, (sel.sum(), len(t))), (pt, args[g]),
                                  oracle)
    share = np.array([cost[b[k]:b[k + 1]].sum() for k in range(4)])
    assert np.abs(share - cost.sum() / 4).max() <= cost.max() * (1 + 1e-6)
    # the cut follows the costs, not the counts: the heavy groups get fewer orbits
    assert b[2] - b[0] > b[4] - b[2]
    with pytest.raises(gb.CudaError):
        gb.split_orbits((pt, args.ravel()), w, t, 4, group=group, ngroup=4)
