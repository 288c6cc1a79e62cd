"""One grid solved over several GPUs by z slabs (FP32): the multi-GPU counterpart of the
reference's multi-rank prototype, which moves the doubled grid between rank layouts with MPI
all-to-alls (mpi_devel/code/open_spacecharge_mod.f90:722-990, movetodoublesizer2c and
movetosinglesizec2r; the Plimpton remap under it, mpi_devel/code/fft/remap_3d.c:64-108).

Rank r of P owns the z planes [z0_r, z0_{r+1}) of the nx x ny x nz grid and the
half-spectrum columns [c0_r, c0_{r+1}) (column ky*(nx+1) + kx), both split as evenly as the
counts allow.  One step, for the particles each rank owns (``owner_of``):

1. deposit into a quad grid of the rank's planes plus one ghost plane, whose sums are
   added into the next rank's first plane (halo sum, one plane);
2. x and y transforms of the rank's planes;
3. all-to-all: every rank receives its columns of every rank's planes;
4. the z pass of its columns (forward z transform, Green product, inverse);
5. all-to-all back: every rank receives its planes of every rank's columns;
6. inverse y and x transforms into the rank's x-pair E grid;
7. halo: the plane below and the plane above the slab from the neighbours;
8. the gather at the rank's particles.

The exchanges go through an ``Exchange``: ``DistExchange`` (torch.distributed, NCCL or
gloo; one rank per process) or ``LocalExchange`` (all ranks in one process, for running the
decomposition on one GPU).  The stages go through a backend: ``CudaSlabBackend`` calls the
library's ``osc_slab_*`` entry points; the CPU tests substitute a numpy backend with the same
array shapes to check the decomposition and the exchanges on gloo ranks.

Inputs and outputs of a step are per rank: ``{rank: (x, y, z, q)}`` -> ``{rank: E}`` (E rows
in the rank's particle order).  Results equal the one-GPU FP32 step to FP32 round-off.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .mesh import Mesh3D, _ctx, _tp


def split(count: int, world: int) -> list[int]:
    """Boundaries of `count` items over `world` ranks: rank r owns [b[r], b[r+1])."""
    return [r * count // world for r in range(world + 1)]


def deposit_cell(mesh: Mesh3D, z) -> np.ndarray:
    """0-based z cell of each particle under the deposit's formula floor((z - zmin) *
    (1/dz) + 1) - nlo (code/open_spacecharge_mod.f90:259-262), the product and the sum each
    rounded, as the deposit kernel evaluates them."""
    z = np.asarray(z, dtype=np.float64)
    dzi = 1.0 / float(mesh.delta[2])
    return (np.floor((z - float(mesh.min[2])) * dzi + 1.0) - 1.0).astype(np.int64)


def owner_of(mesh: Mesh3D, z, world: int) -> np.ndarray:
    """Rank owning each particle: the slab holding its deposit cell, clamped into
    [0, nz - 2] for particles beyond the mesh (they stay with the first or last rank, whose
    gather clamps them as the one-GPU gather does)."""
    nz = int(mesh.nhi[2]) - int(mesh.nlo[2]) + 1
    k = np.clip(deposit_cell(mesh, z), 0, nz - 2)
    bounds = np.asarray(split(nz, world))
    return np.searchsorted(bounds, k, side="right") - 1


@dataclass
class SlabPlan:
    """The static decomposition of an nx x ny x nz grid over `world` ranks."""

    n: tuple[int, int, int]
    world: int

    def __post_init__(self):
        nx, ny, nz = self.n
        if self.world < 1 or self.world > nz:
            raise ValueError(f"{self.world} ranks for {nz} planes")
        self.z0 = split(nz, self.world)
        self.ncols = (nx + 1) * 2 * ny
        self.c0 = split(self.ncols, self.world)

    def planes(self, r: int) -> tuple[int, int]:
        return self.z0[r], self.z0[r + 1] - self.z0[r]

    def columns(self, r: int) -> tuple[int, int]:
        return self.c0[r], self.c0[r + 1] - self.c0[r]

    def gather_planes(self, r: int) -> tuple[int, int]:
        """Planes [p0, p0 + count) of the rank's gather grid: its own, the one below
        (previous rank) and the one above (next rank) where they exist."""
        z0, nzl = self.planes(r)
        lo = 1 if r > 0 else 0
        hi = 1 if r < self.world - 1 else 0
        return z0 - lo, nzl + lo + hi


# ---- exchanges --------------------------------------------------------------------------
class LocalExchange:
    """All ranks in this process: sends[r][s] (rank r to rank s) becomes recvs[s][r]."""

    def __init__(self, world: int):
        self.world = world
        self.ranks = list(range(world))

    def all_to_all(self, sends: dict) -> dict:
        return {s: [sends[r][s] for r in self.ranks] for s in self.ranks}

    def sum(self, values: dict) -> float:
        return sum(values.values())


class DistExchange:
    """One rank per process over a torch.distributed group (NCCL for CUDA tensors, gloo
    for CPU ones): all_to_all_single on the concatenated, flattened sends."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.ranks = [dist.get_rank(group)]

    def all_to_all(self, sends: dict) -> dict:
        import torch

        (r,) = self.ranks
        parts = sends[r]
        ins = [int(t.numel()) for t in parts]
        # the receive sizes: every rank tells every other how much it sends
        ref = parts[0]
        cnt = torch.tensor(ins, dtype=torch.int64, device=ref.device)
        got = torch.empty_like(cnt)
        self.dist.all_to_all_single(got, cnt, group=self.group)
        outs = [int(v) for v in got.tolist()]
        send = torch.cat([t.reshape(-1) for t in parts]) if sum(ins) else ref.new_empty(0)
        recv = ref.new_empty(sum(outs))
        self.dist.all_to_all_single(recv, send, output_split_sizes=outs, input_split_sizes=ins, group=self.group)
        return {r: list(torch.split(recv, outs))}

    def sum(self, values: dict) -> float:
        import torch

        (r,) = self.ranks
        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([float(values[r])], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())


# ---- backends ---------------------------------------------------------------------------
class CudaSlabBackend:
    """The stages on this process's GPU through the osc_slab_* entry points (FP32); grids
    and spectra are float32 tensors (complex values as pairs in a trailing dimension).  The
    exchanges and the halo additions are torch operations, so the context is put on torch's
    current stream: every stage and every copy between them is ordered on that one stream
    (torch.distributed orders its collectives after it)."""

    def __init__(self, ctx, mesh: Mesh3D):
        import torch

        self.torch = torch
        self.ctx = _ctx(ctx)
        self.mesh = mesh
        self.m = mesh.to_c()
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.ctx.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def empty(self, shape):
        return self.torch.empty(shape, dtype=self.torch.float32, device=self.device)

    def empty_rows(self, n):
        return self.torch.empty((n, 3), dtype=self.torch.float64, device=self.device)

    def deposit(self, z0, nzl, x, y, z, q, charge1, quad):
        self.ctx.call("osc_slab_deposit_dev", ctypes.byref(self.m), int(z0), int(nzl), ctypes.c_int64(x.numel()),
                      _tp(x), _tp(y), _tp(z), _tp(q), ctypes.c_double(charge1), _tp(quad), None)

    def forward(self, z0, nzl, quad, X2):
        self.ctx.call("osc_slab_forward_dev", ctypes.byref(self.m), int(z0), int(nzl), _tp(quad), _tp(X2))

    def zpass(self, c0, ncols, zin, zout):
        self.ctx.call("osc_slab_zpass_dev", ctypes.byref(self.m), int(c0), int(ncols), _tp(zin), _tp(zout))

    def inverse(self, z0, nzl, X3, e8):
        self.ctx.call("osc_slab_inverse_dev", ctypes.byref(self.m), int(z0), int(nzl), _tp(X3), _tp(e8))

    def interp(self, p0, count, x, y, z, e8, E):
        self.ctx.call("osc_slab_interp_dev", ctypes.byref(self.m), int(p0), int(count), ctypes.c_int64(x.numel()),
                      _tp(x), _tp(y), _tp(z), _tp(e8), _tp(E))


# ---- the solver -------------------------------------------------------------------------
class SlabSolver:
    """The space-charge step of one mesh (fixed geometry; free space, FP32) over the ranks of
    `exchange`, each rank's stages on `backend` (``CudaSlabBackend`` by default)."""

    def __init__(self, ctx, mesh: Mesh3D, exchange, backend=None):
        self.mesh = mesh
        self.n = tuple(int(h) - int(l) + 1 for l, h in zip(mesh.nlo, mesh.nhi))
        self.ex = exchange
        self.plan = SlabPlan(self.n, exchange.world)
        self.be = backend if backend is not None else CudaSlabBackend(ctx, mesh)

    def step(self, parts: dict, total_charge: float | None = None) -> dict:
        """parts: {rank: (x, y, z, q or None)} for the ranks of this process; with q None
        every particle carries total_charge / (particles over all ranks)."""
        P, be, ex = self.plan, self.be, self.ex
        nx, ny, nz = self.n
        nxh, Ny = nx + 1, 2 * ny
        ranks = ex.ranks
        charge1 = 0.0
        if any(parts[r][3] is None for r in ranks):
            if total_charge is None:
                raise ValueError("q or total_charge must be given")
            npt = ex.sum({r: int(parts[r][0].numel()) for r in ranks})
            charge1 = float(total_charge) / npt
        plane = ny * nx
        # 1. deposit with a ghost plane; halo sum into the next rank's first plane
        quad = {}
        for r in ranks:
            z0, nzl = P.planes(r)
            x, y, z, q = parts[r]
            quad[r] = be.empty((nzl + 1, plane, 4))
            be.deposit(z0, nzl, x, y, z, q, charge1, quad[r])
        empty = {r: quad[r][:0] for r in ranks}
        sends = {r: [quad[r][-1] if s == r + 1 else empty[r] for s in range(P.world)] for r in ranks}
        got = ex.all_to_all(sends)
        for r in ranks:
            if r > 0:
                quad[r][0] += got[r][r - 1].reshape(plane, 4)
        # 2. x and y transforms of each rank's planes
        X2 = {}
        for r in ranks:
            z0, nzl = P.planes(r)
            X2[r] = be.empty((nzl, Ny * nxh, 2))
            be.forward(z0, nzl, quad[r], X2[r])
        # 3. columns of every rank's planes to the rank owning them
        sends = {r: [X2[r][:, P.c0[s]:P.c0[s + 1]].contiguous() for s in range(P.world)] for r in ranks}
        got = ex.all_to_all(sends)
        # 4. the z pass of each rank's columns
        zout = {}
        for s in ranks:
            c0, nc = P.columns(s)
            zin = be.torch.cat([got[s][r].reshape(P.z0[r + 1] - P.z0[r], nc, 2) for r in range(P.world)])
            zout[s] = be.empty((3, nc, nz, 2))
            be.zpass(c0, nc, zin, zout[s])
        # 5. every rank's planes of the columns back
        sends = {r: [zout[r][:, :, P.z0[s]:P.z0[s + 1]].contiguous() for s in range(P.world)] for r in ranks}
        got = ex.all_to_all(sends)
        # 6. inverse transforms into the x-pair grid of the gather planes
        e8 = {}
        for s in ranks:
            z0, nzl = P.planes(s)
            X3 = be.torch.cat([got[s][r].reshape(3, P.c0[r + 1] - P.c0[r], nzl, 2) for r in range(P.world)], dim=1)
            p0, cnt = P.gather_planes(s)
            e8[s] = be.empty((cnt, plane, 8))
            be.inverse(z0, nzl, X3.contiguous(), e8[s][z0 - p0:])
        # 7. halo planes of E: own first plane down, own last plane up
        sends = {}
        for r in ranks:
            z0, nzl = P.planes(r)
            p0, cnt = P.gather_planes(r)
            lo, hi = z0 - p0, z0 - p0 + nzl - 1
            sends[r] = [e8[r][lo] if s == r - 1 else e8[r][hi] if s == r + 1 else e8[r][:0] for s in range(P.world)]
        got = ex.all_to_all(sends)
        for r in ranks:
            p0, cnt = P.gather_planes(r)
            if r > 0:
                e8[r][0] = got[r][r - 1].reshape(plane, 8)
            if r < P.world - 1:
                e8[r][cnt - 1] = got[r][r + 1].reshape(plane, 8)
        # 8. the gather
        out = {}
        for r in ranks:
            x, y, z, _ = parts[r]
            p0, cnt = P.gather_planes(r)
            out[r] = be.empty_rows(x.numel())
            be.interp(p0, cnt, x, y, z, e8[r], out[r])
        return out
