"""The z-slab decomposition of one grid (openspacecharge_b200.slab) on the CPU.

The plan (plane and column splits, the gather's halo planes), the particle ownership by the
deposit's cell formula, and the exchanges: a toy backend with the same array shapes as the
CUDA stages (a linear deposit with a z-linear stencil into quad planes, real/complex FFTs
along x and y, a z-FFT product with random column spectra, the inverse transforms and a
z-linear gather) runs on two and three gloo ranks through DistExchange and must give what
the same backend gives on one rank, and LocalExchange runs the same decomposition in one
process."""
import datetime
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from openspacecharge_b200 import Mesh3D  # noqa: E402
from openspacecharge_b200 import slab  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N = (6, 5, 12)


class ToyBackend:
    """The stages' array shapes and exchanges of CudaSlabBackend with numpy arithmetic:
    nearest node in x and y, linear in z (deposit and gather), unpadded FFTs along x and y on
    the doubled lengths, and per-column random spectra along z."""

    torch = torch

    def __init__(self, mesh, n=N, seed=4):
        self.mesh = mesh
        self.n = n
        nx, ny, nz = n
        rng = np.random.default_rng(seed)
        ncols = (nx + 1) * 2 * ny
        self.G = rng.normal(size=(3, 2 * nz, ncols)) + 1j * rng.normal(size=(3, 2 * nz, ncols))

    def empty(self, shape):
        return torch.zeros(shape, dtype=torch.float32)

    def empty_rows(self, n):
        return torch.zeros((n, 3), dtype=torch.float64)

    def _ij(self, x, y):
        m, (nx, ny, _) = self.mesh, self.n
        i = np.clip(np.rint((x.numpy() - m.min[0]) / m.delta[0]).astype(int), 0, nx - 1)
        j = np.clip(np.rint((y.numpy() - m.min[1]) / m.delta[1]).astype(int), 0, ny - 1)
        return i, j

    def deposit(self, z0, nzl, x, y, z, q, charge1, quad):
        nx, ny, nz = self.n
        i, j = self._ij(x, y)
        k = slab.deposit_cell(self.mesh, z.numpy())
        w = (z.numpy() - self.mesh.min[2]) / self.mesh.delta[2] - k
        qq = q.numpy() if q is not None else np.full(len(k), charge1)
        a = quad.numpy()
        top = nzl if z0 + nzl < nz else nzl - 1
        for kk, ww in ((k - z0, 1 - w), (k + 1 - z0, w)):
            ok = (kk >= 0) & (kk <= top)
            np.add.at(a[:, :, 0], (kk[ok], j[ok] * nx + i[ok]), (qq * ww)[ok])

    def forward(self, z0, nzl, quad, X2):
        nx, ny, _ = self.n
        rho = quad.numpy()[:nzl, :, 0].reshape(nzl, ny, nx).astype(np.float64)
        F = np.fft.fft(np.fft.rfft(rho, n=2 * nx, axis=2), n=2 * ny, axis=1)
        X2.numpy()[...] = np.stack([F.real, F.imag], -1).reshape(X2.shape)

    def zpass(self, c0, nc, zin, zout):
        nz = self.n[2]
        a = zin.numpy().astype(np.float64)
        A = np.fft.fft(a[..., 0] + 1j * a[..., 1], n=2 * nz, axis=0)
        for c in range(3):
            b = np.fft.ifft(A * self.G[c][:, c0:c0 + nc], axis=0)[:nz].T
            zout.numpy()[c] = np.stack([b.real, b.imag], -1)

    def inverse(self, z0, nzl, X3, e8):
        nx, ny, _ = self.n
        a = X3.numpy().astype(np.float64).reshape(3, 2 * ny, nx + 1, nzl, 2)
        S = np.moveaxis(a[..., 0] + 1j * a[..., 1], 3, 1)  # [c][z][ky][kx]
        E = np.fft.irfft(np.fft.ifft(S, axis=2)[:, :, :ny], n=2 * nx, axis=3)[..., :nx]
        out = e8.numpy()
        for c in range(3):
            out[:nzl, :, c] = E[c].reshape(nzl, ny * nx)

    def interp(self, p0, cnt, x, y, z, e8, E):
        nx = self.n[0]
        i, j = self._ij(x, y)
        f = (z.numpy() - self.mesh.min[2]) / self.mesh.delta[2]
        k = np.clip(np.floor(f).astype(int), p0, p0 + cnt - 2)
        w = f - k
        a = e8.numpy()
        node = j * nx + i
        E.numpy()[...] = ((1 - w)[:, None] * a[k - p0, node, :3] + w[:, None] * a[k + 1 - p0, node, :3])


def toy_problem(seed=7, npart=3000):
    rng = np.random.default_rng(seed)
    nx, ny, nz = N
    m = Mesh3D(nlo=(1, 1, 1), nhi=N, min=np.zeros(3), max=np.array([nx - 1, ny - 1, nz - 1], float),
               delta=np.ones(3))
    x = rng.uniform(0, nx - 1, npart)
    y = rng.uniform(0, ny - 1, npart)
    z = rng.uniform(0, nz - 1.001, npart)
    q = rng.uniform(0.5, 1.5, npart)
    return m, x, y, z, q


def solve(world, exchange, m, x, y, z, q, use_q=True):
    own = slab.owner_of(m, z, world)
    parts = {}
    for r in exchange.ranks:
        idx = np.nonzero(own == r)[0]
        parts[r] = tuple(torch.from_numpy(a[idx].copy()) for a in (x, y, z)) + (
            torch.from_numpy(q[idx].copy()) if use_q else None,)
    out = slab.SlabSolver(None, m, exchange, backend=ToyBackend(m)).step(parts, total_charge=2.5)
    return own, out


def test_plan_splits_and_halo_planes():
    p = slab.SlabPlan((8, 6, 10), 3)
    assert p.z0 == [0, 3, 6, 10] and p.c0 == [0, 36, 72, 108] and p.ncols == 108
    assert [p.gather_planes(r) for r in range(3)] == [(0, 4), (2, 5), (5, 5)]
    assert slab.SlabPlan((8, 6, 10), 1).gather_planes(0) == (0, 10)
    with pytest.raises(ValueError):
        slab.SlabPlan((8, 6, 4), 5)


def test_owner_follows_the_deposit_cell_and_clamps():
    m = Mesh3D(nlo=(1, 1, 3), nhi=(4, 4, 14), min=np.zeros(3), max=np.array([3.0, 3.0, 2.2]),
               delta=np.array([1.0, 1.0, 0.2]))
    z = np.array([-5.0, 0.0, 0.19999999999999998, 0.2, 0.7, 1.1, 1.999, 2.2, 9.0])
    k = slab.deposit_cell(m, z)
    assert list(k) == list(np.floor(z * (1 / 0.2) + 1.0) - 1.0)
    own = slab.owner_of(m, z, 3)  # 12 planes: [0,4) [4,8) [8,12), cells clamped to [0,10]
    assert list(own) == [0, 0, 0, 0, 0, 1, 2, 2, 2]


@pytest.mark.parametrize("use_q", [True, False])
def test_local_exchange_matches_one_rank(use_q):
    m, x, y, z, q = toy_problem()
    _, ref = solve(1, slab.LocalExchange(1), m, x, y, z, q, use_q)
    for world in (2, 3, 4):
        own, out = solve(world, slab.LocalExchange(world), m, x, y, z, q, use_q)
        E = np.zeros((len(x), 3))
        for r in range(world):
            E[own == r] = out[r].numpy()
        np.testing.assert_allclose(E, ref[0].numpy(), rtol=0, atol=2e-5 * np.abs(ref[0].numpy()).max())


def worker(rank, ws, port, queue):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        m, x, y, z, q = toy_problem()
        own, out = solve(ws, slab.DistExchange(), m, x, y, z, q)
        queue.put((rank, np.nonzero(own == rank)[0], out[rank].numpy()))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("ws", [2, 3])
def test_gloo_ranks_match_one_rank(ws):
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, ws, port, queue)) for r in range(ws)]
    for p in procs:
        p.start()
    got = [queue.get(timeout=300) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m, x, y, z, q = toy_problem()
    _, ref = solve(1, slab.LocalExchange(1), m, x, y, z, q)
    E = np.full((len(x), 3), np.nan)
    for r, idx, Er in got:
        E[idx] = Er
    assert not np.isnan(E).any()
    np.testing.assert_allclose(E, ref[0].numpy(), rtol=0, atol=2e-5 * np.abs(ref[0].numpy()).max())
