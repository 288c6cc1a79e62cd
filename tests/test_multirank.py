"""The multi-rank path of the batched workload on the CPU: two gloo ranks (127.0.0.1) shard a
batch of bunches with the package's ShardedBatch (assignment computed identically on every
rank, no communication), solve their bunches with the oracle's deposit + space_charge_3d +
interpolate_field, and gather the fields to rank 0 with ShardedBatch.gather; the result
must equal a single-rank solve of every bunch in the batch's particle order, the shards must
partition the batch, and the job time is the maximum over ranks."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GAMMA = 9.784756683727565


def make_bunches(nb=6, seed=3):
    from openspacecharge_b200.bunch import gendist
    rng = np.random.default_rng(seed)
    grids, counts, parts = [], [], []
    for b in range(nb):
        grids.append(tuple(int(rng.choice((12, 16))) for _ in range(3)))
        n = int(rng.integers(500, 3000))
        counts.append(n)
        parts.append(gendist(n, sigma=tuple(rng.uniform(0.5e-3, 2e-3, 3)), seed=100 + b))
    return grids, counts, parts


def solve(oracle, grid, xyz):
    x, y, z = xyz
    om = oracle.make_mesh((1, 1, 1), grid, (1, 1, 1), (0, 0, 0), (0, 0, 0), (0, 0, 0), GAMMA)
    rho, _ = oracle.deposit_particles(x, y, z, om, total_charge=1e-9, resize_mesh=True)
    ef, _ = oracle.space_charge_3d(om, rho)
    E, _, _ = oracle.interpolate_field(om, ef, x, y, z)
    return E


def worker(rank, ws, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle
        from openspacecharge_b200 import Mesh3D
        from openspacecharge_b200.multirank import ShardedBatch, max_over_ranks
        oracle.set_threads(1)
        grids, counts, parts = make_bunches()
        meshes = [Mesh3D(nlo=(1, 1, 1), nhi=g, gamma=GAMMA) for g in grids]
        sb = ShardedBatch(meshes, counts, rank=rank, world_size=ws)
        full = [np.concatenate([p[d] for p in parts]) for d in range(3)]
        xl, yl, zl = (sb.select(a) for a in full)
        rows, o = [], 0
        for b in sb.mine:  # this rank's bunches, in the order select() concatenates them
            sl = slice(o, o + counts[b])
            rows.append(solve(oracle, grids[b], (xl[sl], yl[sl], zl[sl])))
            o += counts[b]
        E_local = torch.from_numpy(np.concatenate(rows) if rows else np.zeros((0, 3)))
        E_full = sb.gather(E_local, dst=0)
        t = max_over_ranks(1.0 + rank)
        if rank == 0:
            out.put((E_full.numpy(), t, sb.shards))
        else:
            assert E_full is None
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_batch_matches_single_rank(oracle):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    E_full, t, shards = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    grids, counts, parts = make_bunches()
    assert sorted(shards[0] + shards[1]) == list(range(len(grids))) and not set(shards[0]) & set(shards[1])
    assert shards[0] and shards[1]
    assert t == 2.0  # the maximum over ranks
    ref = np.concatenate([solve(oracle, grids[b], parts[b]) for b in range(len(grids))])
    assert np.array_equal(E_full, ref)


def test_shard_balance():
    from openspacecharge_b200.multirank import bunch_cost, shard_bunches
    rng = np.random.default_rng(1)
    grids = [tuple(int(rng.choice((32, 48, 64, 96))) for _ in range(3)) for _ in range(256)]
    counts = [int(np.exp(rng.uniform(np.log(1e4), np.log(1e6)))) for _ in range(256)]
    cost = [bunch_cost(g, n) for g, n in zip(grids, counts)]
    for ws in (2, 4, 8):
        shards = [shard_bunches(grids, counts, r, ws) for r in range(ws)]
        assert sorted(sum(shards, [])) == list(range(256))
        loads = [sum(cost[b] for b in s) for s in shards]
        assert max(loads) <= 1.05 * sum(cost) / ws
    with pytest.raises(ValueError):
        shard_bunches(grids, counts, 2, 2)


def test_sharded_batch_single_rank_is_the_whole_batch():
    from openspacecharge_b200 import Mesh3D
    from openspacecharge_b200.multirank import ShardedBatch, max_over_ranks
    grids, counts, _ = make_bunches()
    sb = ShardedBatch([Mesh3D(nlo=(1, 1, 1), nhi=g) for g in grids], counts, rank=0, world_size=1)
    assert sb.mine == list(range(len(grids)))
    assert np.array_equal(sb.particle_index(), np.arange(sum(counts)))
    assert max_over_ranks(3.5) == 3.5  # no process group: the value itself
