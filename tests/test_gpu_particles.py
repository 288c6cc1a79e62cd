"""GPU parity of deposition, mesh sizing and interpolation against the FP64 oracle.

Deposition uses FP64 atomics on the host-facing entry points, so results equal the oracle
up to summation order (relative 1e-13 of the largest node).  Interpolation follows the
reference's order of operations (1e-13)."""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist

pytestmark = pytest.mark.gpu


def test_get_mesh_quantities_bit_exact(ctx, oracle):
    x, y, z = gendist(30000, seed=4)
    for isetzmin in (0, 1):
        d0, u0 = oracle.get_mesh_quantities(x, y, z + 2e-3, (1, 1, 1), (20, 22, 24), isetzmin)
        d1, u1 = osc.get_mesh_quantities(ctx, x, y, z + 2e-3, (1, 1, 1), (20, 22, 24), isetzmin)
        assert np.array_equal(d0, d1) and np.array_equal(u0, u1)


@pytest.mark.parametrize("resize", [True, False])
@pytest.mark.parametrize("use_q", [True, False])
def test_deposit_particles_matches_oracle(ctx, oracle, resize, use_q):
    x, y, z = gendist(200000, sigma=(1e-3, 2e-3, 0.5e-3), seed=8)
    n = (24, 20, 28)
    q = np.random.default_rng(1).uniform(0.5, 1.5, len(x)) * 1e-15 if use_q else None
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    umax = umin + (np.array(n) - 1) * delta
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umax, delta, 1.0)
    rho_ref, nout_ref = oracle.deposit_particles(x, y, z, om, qa=q, total_charge=None if use_q else 1e-9,
                                                 resize_mesh=resize)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin.copy(), max=umax.copy(), delta=delta.copy())
    nout = osc.deposit_particles(ctx, x, y, z, m, qa=q, total_charge=None if use_q else 1e-9, resize_mesh=resize)
    assert nout == nout_ref == 0
    assert np.array_equal(m.delta, np.array(om.delta[:])) and np.array_equal(m.min, np.array(om.min[:]))
    assert abs(m.charge / om.charge - 1) < 1e-12
    assert np.abs(m.rho - rho_ref).max() <= 1e-13 * np.abs(rho_ref).max()


def test_deposit_counts_particles_outside(ctx, oracle):
    x, y, z = gendist(50000, seed=12)
    n = (16, 16, 16)
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    umin2 = umin + 4 * delta  # shift the mesh so part of the bunch falls outside
    umax2 = umin2 + (np.array(n) - 1) * delta
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin2, umax2, delta, 1.0)
    rho_ref, nout_ref = oracle.deposit_particles(x, y, z, om, total_charge=1e-9, resize_mesh=False)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin2.copy(), max=umax2.copy(), delta=delta.copy())
    nout = osc.deposit_particles(ctx, x, y, z, m, total_charge=1e-9, resize_mesh=False)
    assert nout == nout_ref > 0
    assert np.abs(m.rho - rho_ref).max() <= 1e-13 * np.abs(rho_ref).max()


def test_deposit_without_charge_prints_and_returns(ctx, capsys):
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=(8, 8, 8))
    osc.deposit_particles(ctx, [0.0, 1.0], [0.0, 1.0], [0.0, 1.0], m)
    assert "must specify qa or total_charge" in capsys.readouterr().out


def test_depose_rho_scalar_with_lost_flags(ctx, oracle):
    x, y, z = gendist(80000, seed=13)
    n = (20, 20, 20)
    lost = (np.random.default_rng(2).uniform(size=len(x)) < 0.1).astype(float)
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    r0, f0 = oracle.depose_rho_scalar(x, y, z, 1e-14, (1, 1, 1), n, delta, umin, lostflag=lost)
    r1, f1 = osc.depose_rho_scalar(ctx, x, y, z, 1e-14, (1, 1, 1), n, delta, umin, lostflag=lost)
    assert f0 == f1
    assert np.abs(r1 - r0).max() <= 1e-13 * np.abs(r0).max()


def test_interpolate_matches_oracle(ctx, oracle):
    n = (10, 12, 14)
    rng = np.random.default_rng(5)
    ef = np.asfortranarray(rng.standard_normal(n + (3,)))
    bf = np.asfortranarray(rng.standard_normal(n + (3,)))
    delta = np.array([0.1, 0.2, 0.3])
    umin = np.array([-1.0, 0.5, 2.0])
    umax = umin + (np.array(n) - 1) * delta
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umax, delta, 1.0)
    npts = 20000
    pts = umin - 0.3 * delta + rng.uniform(size=(npts, 3)) * (umax - umin + 0.6 * delta)  # some outside
    E0, B0, c0 = oracle.interpolate_field(om, ef, pts[:, 0], pts[:, 1], pts[:, 2], bfield=bf)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umax, delta=delta)
    m.efield, m.bfield = ef, bf
    E1, B1, c1 = osc.interpolate_field(ctx, pts[:, 0], pts[:, 1], pts[:, 2], m, E=True, B=True)
    assert c0 == c1 > 0
    assert np.abs(E1 - E0).max() <= 1e-13 * np.abs(E0).max()
    assert np.abs(B1 - B0).max() <= 1e-13 * np.abs(B0).max()
