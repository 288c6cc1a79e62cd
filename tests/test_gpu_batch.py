"""Batched steps (osc_batch_space_charge_step): many bunches with their own meshes in one call.
Every bunch must get the fields that a single step of that bunch gives (same mesh refit,
same Green spectra, same pipeline; FP32 atomics reorder, hence 2e-6), and one bunch is
checked against the oracle's deposit_particles + space_charge_3d + interpolate_field chain
(code/open_spacecharge_mod.f90:156-489) at the FP32 tolerance."""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu

GAMMA = 9.784756683727565


def make_bunches(nb, edges, seed, np_range=(2000, 30000)):
    rng = np.random.default_rng(seed)
    meshes, xs, ys, zs, counts, charges = [], [], [], [], [], []
    for b in range(nb):
        n = tuple(int(rng.choice(edges)) for _ in range(3))
        npart = int(np.exp(rng.uniform(np.log(np_range[0]), np.log(np_range[1]))))
        sig = tuple(rng.uniform(0.2e-3, 2e-3, 3))
        x, y, z = gendist(npart, sigma=sig, seed=seed * 1000 + b)
        meshes.append(osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=GAMMA))
        xs.append(x), ys.append(y), zs.append(z)
        counts.append(npart)
        charges.append(rng.uniform(0.1e-9, 2e-9))
    return meshes, np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), counts, charges


@pytest.mark.parametrize("prec", [osc.PREC_FP32, osc.PREC_FP64])
def test_batch_matches_single_steps(ctx, prec):
    meshes, x, y, z, counts, charges = make_bunches(9, (16, 24, 32), seed=5)
    E, nout = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges, precision=prec)
    assert nout == [0] * len(meshes)
    off = 0
    for b, m in enumerate(meshes):
        sl = slice(off, off + counts[b])
        ms = osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA)
        Es, _ = osc.space_charge_step(ctx, ms, x[sl], y[sl], z[sl], total_charge=charges[b], resize_mesh=True,
                                      precision=prec)
        assert np.array_equal(ms.min, m.min) and np.array_equal(ms.delta, m.delta)
        assert ms.charge == m.charge
        mx, _ = field_err(E[sl], Es)
        assert mx <= (2e-6 if prec == osc.PREC_FP32 else 1e-12), (b, m.nhi, mx)
        off += counts[b]


def test_batch_with_charges_and_fixed_meshes(ctx):
    meshes, x, y, z, counts, _ = make_bunches(5, (16, 32), seed=6)
    q = np.random.default_rng(9).uniform(0.5, 1.5, len(x)) * 1e-15
    osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, qa=q, resize_mesh=True)
    # shift every mesh by 3 cells: some particles fall outside and are counted per bunch
    for m in meshes:
        m.min = m.min + 3 * m.delta
        m.max = m.max + 3 * m.delta
    E, nout = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, qa=q, resize_mesh=False)
    off = 0
    for b, m in enumerate(meshes):
        sl = slice(off, off + counts[b])
        ms = osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA, min=m.min.copy(), max=m.max.copy(),
                        delta=m.delta.copy())
        Es, _ = osc.space_charge_step(ctx, ms, x[sl], y[sl], z[sl], qa=q[sl], resize_mesh=False)
        assert abs(ms.charge / m.charge - 1) < 1e-12
        nref = osc.deposit_particles(ctx, x[sl], y[sl], z[sl],
                                     osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, min=m.min.copy(), max=m.max.copy(),
                                                delta=m.delta.copy()), qa=q[sl], resize_mesh=False)
        assert nout[b] == nref > 0
        mx, _ = field_err(E[sl], Es)
        assert mx <= 2e-6, (b, mx)
        off += counts[b]


def test_batch_bunch_matches_oracle(ctx, oracle):
    meshes, x, y, z, counts, charges = make_bunches(4, (24,), seed=7, np_range=(40000, 60000))
    E, _ = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges)
    b = 2
    off = sum(counts[:b])
    sl = slice(off, off + counts[b])
    n = tuple(meshes[b].nhi)
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), (0, 0, 0), (0, 0, 0), (0, 0, 0), GAMMA)
    rho, _ = oracle.deposit_particles(x[sl], y[sl], z[sl], om, total_charge=charges[b], resize_mesh=True)
    ef, _ = oracle.space_charge_3d(om, rho)
    E0, _, _ = oracle.interpolate_field(om, ef, x[sl], y[sl], z[sl])
    assert np.array_equal(meshes[b].delta, np.array(om.delta[:]))
    mx, rm = field_err(E[sl], E0)
    assert mx <= 1e-5, (mx, rm)


def test_batch_dev_matches_host(ctx):
    torch = pytest.importorskip("torch")
    meshes, x, y, z, counts, charges = make_bunches(6, (16, 24, 32, 48), seed=8)
    E1, _ = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges)
    dev = torch.device("cuda", 0)
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    E = torch.empty((len(x), 3), dtype=torch.float64, device=dev)
    meshes2 = [osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA) for m in meshes]
    osc.batch_space_charge_step_dev(ctx, meshes2, tx, ty, tz, counts, E, total_charges=charges)
    ctx.synchronize()
    for m1, m2 in zip(meshes, meshes2):
        assert np.array_equal(m1.delta, m2.delta)
    mx, _ = field_err(E.cpu().numpy(), E1)
    assert mx < 2e-6
