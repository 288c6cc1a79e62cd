"""Deterministic deposition (OSC_DEPOSIT_DETERMINISTIC): 64-bit fixed-point atomics make rho,
and everything computed from it, bit-identical for any order of the particles.  The
fixed-point sum is checked against the FP64 oracle (deposit_particles,
code/open_spacecharge_mod.f90:257-283) to 1e-13 of the largest node."""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist

pytestmark = pytest.mark.gpu


@pytest.fixture()
def det_ctx():
    c = osc.Context(0)
    c.set_option(osc.OPT_DEPOSIT_MODE, osc.DEPOSIT_DETERMINISTIC)
    yield c
    c.close()


def _mesh(oracle, x, y, z, n):
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    umax = umin + (np.array(n) - 1) * delta
    return delta, umin, umax


@pytest.mark.parametrize("use_q", [False, True])
def test_fixed_point_deposit_is_order_independent(det_ctx, oracle, use_q):
    x, y, z = gendist(300000, sigma=(1e-3, 1.5e-3, 0.6e-3), seed=21)
    n = (22, 26, 30)
    rng = np.random.default_rng(3)
    q = rng.uniform(0.2, 2.0, len(x)) * 1e-15 if use_q else None
    delta, umin, umax = _mesh(oracle, x, y, z, n)
    perm = rng.permutation(len(x))
    rhos = []
    for order in (np.arange(len(x)), perm, perm[::-1]):
        m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin.copy(), max=umax.copy(), delta=delta.copy())
        osc.deposit_particles(det_ctx, x[order], y[order], z[order], m, qa=None if q is None else q[order],
                              total_charge=None if use_q else 1e-9, resize_mesh=False)
        rhos.append(m.rho.copy())
    assert np.array_equal(rhos[0], rhos[1]) and np.array_equal(rhos[0], rhos[2])
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umax, delta, 1.0)
    ref, _ = oracle.deposit_particles(x, y, z, om, qa=q, total_charge=None if use_q else 1e-9, resize_mesh=False)
    assert np.abs(rhos[0] - ref).max() <= 1e-13 * np.abs(ref).max()


def test_fixed_point_depose_rho_scalar(det_ctx, oracle):
    x, y, z = gendist(60000, seed=22)
    n = (18, 18, 18)
    lost = (np.random.default_rng(4).uniform(size=len(x)) < 0.05).astype(float)
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    r0, f0 = oracle.depose_rho_scalar(x, y, z, 1e-14, (1, 1, 1), n, delta, umin, lostflag=lost)
    r1, f1 = osc.depose_rho_scalar(det_ctx, x, y, z, 1e-14, (1, 1, 1), n, delta, umin, lostflag=lost)
    assert f0 == f1
    assert np.abs(r1 - r0).max() <= 1e-13 * np.abs(r0).max()


@pytest.mark.parametrize("precision", [osc.PREC_FP32, osc.PREC_FP64])
def test_step_is_bit_reproducible_under_permutation(det_ctx, precision):
    x, y, z = gendist(200000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=23)
    perm = np.random.default_rng(5).permutation(len(x))
    out = []
    for order in (np.arange(len(x)), perm):
        m = osc.Mesh3D(nlo=(1, 1, 1), nhi=(32, 32, 48), gamma=9.785)
        E, _ = osc.space_charge_step(det_ctx, m, x[order], y[order], z[order], total_charge=1e-9,
                                     resize_mesh=True, precision=precision)
        inv = np.empty_like(order)
        inv[order] = np.arange(len(order))
        out.append(E[inv])
    assert np.array_equal(out[0], out[1])
