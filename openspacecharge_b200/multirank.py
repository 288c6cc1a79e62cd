"""Batched bunches sharded over ranks: one process per GPU, no data-path collective.

The batched step (``osc_batch_space_charge_step_dev``) solves many independent bunches,
each with its own mesh.  Bunches share nothing, so a job over several GPUs partitions them:
every rank computes the same assignment from the bunch sizes alone (no communication),
solves its own bunches on its own GPU, and the fields are gathered to one rank only when
the caller wants them in one place.  The reference solves one bunch per call
(space_charge_3d, code/open_spacecharge_mod.f90:431-489); a tracking code with many
bunches loops over them, which this replaces.
"""
from __future__ import annotations

import numpy as np

from .mesh import Mesh3D, batch_space_charge_step_dev
from .native import PREC_FP32

# Estimated cost of a bunch: grid nodes plus 0.35 per particle, the measured ratio of the
# field work per node to the particle work per particle of the FP32 batched step.
PARTICLE_COST = 0.35


def bunch_cost(grid, npart) -> float:
    return float(grid[0] * grid[1] * grid[2]) + PARTICLE_COST * float(npart)


def shard_bunches(grids, counts, rank: int, world_size: int) -> list[int]:
    """Indices of the bunches rank `rank` solves: longest-processing-time assignment by
    estimated cost (largest first, each to the least loaded rank, ties to the lower rank),
    identical on every rank."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} of world size {world_size}")
    cost = [bunch_cost(g, n) for g, n in zip(grids, counts)]
    load = [0.0] * world_size
    owner = [0] * len(cost)
    for b in sorted(range(len(cost)), key=lambda i: (-cost[i], i)):
        r = min(range(world_size), key=lambda k: (load[k], k))
        owner[b] = r
        load[r] += cost[b]
    return [b for b in range(len(cost)) if owner[b] == rank]


class ShardedBatch:
    """This rank's share of a batch of bunches.

    ``meshes`` (Mesh3D per bunch), ``counts`` (particles per bunch, concatenated in bunch
    order in the full arrays) and ``total_charges`` describe the whole batch on every rank.
    """

    def __init__(self, meshes, counts, total_charges=None, rank: int = 0, world_size: int = 1):
        self.meshes_all = list(meshes)
        self.counts_all = [int(c) for c in counts]
        self.charges_all = None if total_charges is None else [float(q) for q in total_charges]
        self.rank, self.world_size = rank, world_size
        self.offsets_all = np.concatenate([[0], np.cumsum(self.counts_all)]).astype(np.int64)
        grids = [tuple(int(v) for v in m.shape) for m in self.meshes_all]
        self.shards = [shard_bunches(grids, self.counts_all, r, world_size) for r in range(world_size)]
        self.mine = self.shards[rank]
        self.meshes = [self.meshes_all[b] for b in self.mine]
        self.counts = [self.counts_all[b] for b in self.mine]
        self.charges = None if self.charges_all is None else [self.charges_all[b] for b in self.mine]
        self.rows = [sum(self.counts_all[b] for b in s) for s in self.shards]

    def particle_index(self, rank: int | None = None) -> np.ndarray:
        """Rows of the full particle arrays that belong to `rank`'s bunches, in its order."""
        s = self.shards[self.rank if rank is None else rank]
        if not s:
            return np.zeros(0, dtype=np.int64)
        return np.concatenate([np.arange(self.offsets_all[b], self.offsets_all[b + 1]) for b in s])

    def select(self, a) -> np.ndarray:
        """This rank's particles from a full per-particle host array."""
        return np.ascontiguousarray(np.asarray(a)[self.particle_index()])

    def step_dev(self, ctx, x, y, z, E, qa=None, resize_mesh=True, precision=PREC_FP32) -> None:
        """The batched step over this rank's bunches (device tensors holding its particles,
        as ``select`` orders them)."""
        if not self.mine:
            return
        batch_space_charge_step_dev(ctx, self.meshes, x, y, z, self.counts, E, qa=qa, total_charges=self.charges,
                                    resize_mesh=resize_mesh, precision=precision)

    def gather(self, E_local, dst: int = 0, group=None):
        """Every rank's rows of E gathered on `dst` in the full batch's particle order (one
        padded all-gather; tensors on the device the process group's backend uses).
        Returns the full (total, 3) tensor on `dst`, None elsewhere."""
        import torch
        import torch.distributed as dist
        nmax = max(self.rows) if self.rows else 0
        pad = torch.zeros((nmax, 3), dtype=E_local.dtype, device=E_local.device)
        pad[: E_local.shape[0]] = E_local
        parts = [torch.empty_like(pad) for _ in range(self.world_size)]
        dist.all_gather(parts, pad, group=group)
        if dist.get_rank(group) != dst:
            return None
        full = torch.empty((int(self.offsets_all[-1]), 3), dtype=E_local.dtype, device=E_local.device)
        for r in range(self.world_size):
            idx = torch.from_numpy(self.particle_index(r)).to(E_local.device)
            full[idx] = parts[r][: self.rows[r]]
        return full


def max_over_ranks(v: float, group=None) -> float:
    """The largest of the ranks' values (a job's time is its slowest rank's); v itself
    without an initialised process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(v)
    t = torch.tensor([float(v)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


__all__ = ["bunch_cost", "shard_bunches", "ShardedBatch", "max_over_ranks", "Mesh3D"]
