"""One grid over z slabs (osc_slab_* and openspacecharge_b200.slab) on one GPU: P ranks
emulated in this process, their exchanges made in process (LocalExchange), must give the
fields of the one-GPU FP32 step on the same particles and mesh (FP32 reductions reorder,
hence 2e-6 normwise), for 1, 2 and 3 slabs, with and without per-particle charges and with
particles beyond the mesh in z; one case is also checked against the oracle's
deposit_particles + space_charge_3d + interpolate_field chain
(code/open_spacecharge_mod.f90:156-489) at the FP32 tolerance."""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200 import slab
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GAMMA = 9.784756683727565
Q = 1e-9


def problem(ctx, n, npart=120000, seed=3):
    x, y, z = gendist(npart, sigma=(1e-3, 1.3e-3, 2e-3), seed=seed)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=GAMMA)
    osc.space_charge_step(ctx, m, x, y, z, total_charge=Q, resize_mesh=True)  # fits the mesh
    # a few particles beyond the mesh in z: not deposited, clamped by the gather
    z = z.copy()
    z[:5] = m.min[2] - 3 * m.delta[2] * np.arange(1, 6)
    z[5:10] = m.max[2] + 3 * m.delta[2] * np.arange(1, 6)
    q = np.random.default_rng(seed).uniform(0.5, 1.5, npart) * (Q / npart)
    return m, x, y, z, q


def run_slabs(ctx, m, x, y, z, q, world):
    dev = torch.device("cuda", 0)
    own = slab.owner_of(m, z, world)
    parts = {}
    for r in range(world):
        idx = np.nonzero(own == r)[0]
        parts[r] = tuple(torch.from_numpy(a[idx].copy()).to(dev) for a in (x, y, z)) + (
            torch.from_numpy(q[idx].copy()).to(dev) if q is not None else None,)
    out = slab.SlabSolver(ctx, m, slab.LocalExchange(world)).step(parts, total_charge=Q)
    E = np.zeros((len(x), 3))
    for r in range(world):
        E[own == r] = out[r].cpu().numpy()
    return E


@pytest.mark.parametrize("n", [(32, 24, 48), (20, 30, 64), (16, 16, 96)])
@pytest.mark.parametrize("world", [1, 2, 3])
@pytest.mark.parametrize("use_q", [False, True])
def test_slab_step_matches_one_gpu_step(ctx, n, world, use_q):
    m, x, y, z, q = problem(ctx, n)
    qa = q if use_q else None
    dev = torch.device("cuda", 0)
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    tq = torch.from_numpy(q).to(dev) if use_q else None
    E1 = torch.empty((len(x), 3), dtype=torch.float64, device=dev)
    ms = osc.Mesh3D(nlo=m.nlo, nhi=m.nhi, min=m.min.copy(), max=m.max.copy(), delta=m.delta.copy(), gamma=GAMMA)
    osc.space_charge_step_dev(ctx, ms, tx, ty, tz, E1, qa=tq, total_charge=None if use_q else Q)
    E = run_slabs(ctx, m, x, y, z, qa, world)
    mx, rm = field_err(E, E1.cpu().numpy())
    assert mx <= 2e-6, (n, world, use_q, mx, rm)


def test_slab_step_matches_oracle(ctx, oracle):
    n = (20, 30, 64)
    m, x, y, z, _ = problem(ctx, n, npart=60000, seed=5)
    E = run_slabs(ctx, m, x, y, z, None, 2)
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), m.min, m.max, m.delta, GAMMA)
    rho, _ = oracle.deposit_particles(x, y, z, om, total_charge=Q, resize_mesh=False)
    ef, _ = oracle.space_charge_3d(om, rho)
    E0, _, _ = oracle.interpolate_field(om, ef, x, y, z)
    mx, rm = field_err(E, E0)
    assert mx <= 1e-5, (mx, rm)


def test_slab_entry_points_reject_bad_ranges(ctx):
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=(16, 16, 20), min=np.zeros(3), max=np.ones(3), delta=np.full(3, 1 / 15),
                   gamma=GAMMA)
    be = slab.CudaSlabBackend(ctx, m)
    quad = be.empty((21, 256, 4))
    with pytest.raises(osc.OscError) as ei:
        be.forward(15, 8, quad, be.empty((8, 32 * 17, 2)))  # planes [15, 23) of 20
    assert ei.value.code == osc.native.OSC_E_INVALID
    with pytest.raises(osc.OscError) as ei:  # doubled z length 40 has no warp z pass
        be.zpass(0, 8, be.empty((20, 8, 2)), be.empty((3, 8, 20, 2)))
    assert ei.value.code == osc.native.OSC_E_UNSUPPORTED
    m2 = osc.Mesh3D(nlo=(1, 1, 1), nhi=(16, 16, 48), min=np.zeros(3), max=np.ones(3), delta=np.full(3, 1 / 15),
                    gamma=GAMMA)
    be2 = slab.CudaSlabBackend(ctx, m2)
    with pytest.raises(osc.OscError) as ei:  # columns beyond the 17 x 32
        be2.zpass(17 * 32 - 4, 8, be2.empty((48, 8, 2)), be2.empty((3, 8, 48, 2)))
    assert ei.value.code == osc.native.OSC_E_INVALID
