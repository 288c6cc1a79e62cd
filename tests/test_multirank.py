"""The multi-rank path of the batched workload on the CPU: two gloo ranks (127.0.0.1) shard a
batch of bunches with bench.shard_bunches (no communication), solve their bunches with the
oracle's deposit + space_charge_3d + interpolate_field, and all-gather the fields; the
result must equal a single-rank solve of every bunch, the shards must partition the batch,
and the job time is the maximum over ranks."""
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
        import bench
        from oracle import oracle
        oracle.set_threads(1)
        grids, counts, parts = make_bunches()
        mine = bench.shard_bunches(grids, counts, rank, ws)
        local = {b: solve(oracle, grids[b], parts[b]) for b in mine}
        gathered = [None] * ws
        dist.all_gather_object(gathered, local)
        t = bench.max_over_ranks(1.0 + rank, dist)
        if rank == 0:
            merged = {}
            for d in gathered:
                merged.update(d)
            out.put((sorted(merged), {b: merged[b] for b in merged}, t,
                     [bench.shard_bunches(grids, counts, r, ws) for r in range(ws)]))
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
    keys, fields, t, shards = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    grids, counts, parts = make_bunches()
    assert keys == list(range(len(grids)))
    assert sorted(shards[0] + shards[1]) == list(range(len(grids))) and not set(shards[0]) & set(shards[1])
    assert t == 2.0  # the maximum over ranks
    for b in range(len(grids)):
        ref = solve(oracle, grids[b], parts[b])
        assert np.array_equal(fields[b], ref)


def test_shard_balance():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(1)
    grids = [tuple(int(rng.choice((32, 48, 64, 96))) for _ in range(3)) for _ in range(256)]
    counts = [int(np.exp(rng.uniform(np.log(1e4), np.log(1e6)))) for _ in range(256)]
    cost = [g[0] * g[1] * g[2] + 0.35 * n for g, n in zip(grids, counts)]
    for ws in (2, 4, 8):
        loads = [sum(cost[b] for b in bench.shard_bunches(grids, counts, r, ws)) for r in range(ws)]
        assert max(loads) <= 1.05 * sum(cost) / ws
