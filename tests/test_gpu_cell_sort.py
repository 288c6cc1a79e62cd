"""Cell-sorted particles: the counting sort by deposit cell, the run-aggregated deposits and
the step in every particle-order mode, against the FP64 oracle.

The reference deposits and gathers in the caller's order (deposit_particles,
code/open_spacecharge_mod.f90:257-283; interpolate_field, :311-390); the sorted modes must
give the same fields.  Tolerances: FP32 paths 1e-5 normwise per component against the
oracle; the fixed-point modes are compared bit for bit with each other.
"""
import ctypes

import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu

GAMMA = 9.784756683727565


def _torch():
    return pytest.importorskip("torch")


def _mesh(oracle, x, y, z, n, shrink=1.0):
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    delta = delta * shrink
    umax = umin + (np.array(n) - 1) * delta
    return osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umax, delta=delta, gamma=GAMMA)


@pytest.mark.parametrize("use_q", [False, True])
def test_sort_orders_by_cell_and_returns_a_permutation(ctx, oracle, use_q):
    torch = _torch()
    x, y, z = gendist(300_000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=41)
    n = (24, 20, 40)
    m = _mesh(oracle, x, y, z, n, shrink=0.9)  # the tails fall outside and sort last
    x[:7] = np.nan
    q = np.random.default_rng(1).uniform(0.5, 1.5, len(x)) if use_q else None
    t = [torch.from_numpy(a).cuda() for a in (x, y, z)]
    tq = torch.from_numpy(q).cuda() if use_q else None
    xs, ys, zs, qs, perm, nout = osc.sort_particles_dev(ctx, m, *t, q=tq)
    p = perm.cpu().numpy()
    assert np.array_equal(np.sort(p), np.arange(len(x)))
    assert np.array_equal(xs.cpu().numpy(), x[p], equal_nan=True)
    assert np.array_equal(ys.cpu().numpy(), y[p]) and np.array_equal(zs.cpu().numpy(), z[p])
    if use_q:
        assert np.array_equal(qs.cpu().numpy(), q[p])
    keys = osc.cell_keys(m, x, y, z)
    ks = keys[p]
    assert np.all(np.diff(ks) >= 0)
    N = n[0] * n[1] * n[2]
    assert nout == int((keys == N).sum()) and nout >= 7
    # the empty call and the aliasing check
    e = torch.zeros(0, dtype=torch.float64, device="cuda")
    assert osc.sort_particles_dev(ctx, m, e, e, e)[5] == 0
    ptrs = [ctypes.c_void_p(a.data_ptr()) for a in t]
    with pytest.raises(osc.OscError):  # sorted copies may not alias the inputs
        ctx.call("osc_sort_particles_dev", ctypes.byref(m.to_c()), ctypes.c_int64(len(x)), *ptrs, None, *ptrs,
                 None, None, None)


def _oracle_step(oracle, m, x, y, z, qtot=1e-9, at_cathode=False):
    om = oracle.make_mesh((1, 1, 1), m.nhi, (1, 1, 1), m.min, m.max, m.delta, GAMMA)
    rho, nout = oracle.deposit_particles(x, y, z, om, total_charge=qtot, resize_mesh=False)
    ef, _ = oracle.space_charge_3d(om, rho, at_cathode=at_cathode)
    E, _, _ = oracle.interpolate_field(om, ef, x, y, z)
    return E


@pytest.mark.parametrize("order", [osc.ORDER_SORT, osc.ORDER_CELL_SORTED, osc.ORDER_ANY])
@pytest.mark.parametrize("presorted", [False, True])
def test_fp32_step_in_every_order_mode_matches_oracle(oracle, order, presorted):
    x, y, z = gendist(400_000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=42)
    n = (32, 32, 48)
    with osc.Context(0) as c:
        m = _mesh(oracle, x, y, z, n)
        if presorted:
            p = np.argsort(osc.cell_keys(m, x, y, z), kind="stable")
            x, y, z = (np.ascontiguousarray(a[p]) for a in (x, y, z))
        E0 = _oracle_step(oracle, m, x, y, z)
        c.set_option(osc.OPT_PARTICLE_ORDER, order)
        assert c.get_option(osc.OPT_PARTICLE_ORDER) == order
        E1, _ = osc.space_charge_step(c, m, x, y, z, total_charge=1e-9, resize_mesh=False, precision=osc.PREC_FP32)
        mx, rm = field_err(E1, E0)
        assert mx <= 1e-5 and rm <= 1e-5, (mx, rm)


def test_sorted_step_with_b_and_cathode(oracle):
    x, y, z = gendist(200_000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=43, centroid=(0, 0, 3e-3))
    n = (24, 24, 32)
    with osc.Context(0) as c:
        c.set_option(osc.OPT_PARTICLE_ORDER, osc.ORDER_SORT)
        m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=GAMMA)
        E1, B1 = osc.space_charge_step(c, m, x, y, z, total_charge=1e-9, resize_mesh=True, at_cathode=True,
                                       precision=osc.PREC_FP32, want_b=True)
        c.set_option(osc.OPT_PARTICLE_ORDER, osc.ORDER_ANY)
        m2 = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=GAMMA)
        E2, B2 = osc.space_charge_step(c, m2, x, y, z, total_charge=1e-9, resize_mesh=True, at_cathode=True,
                                       precision=osc.PREC_FP32, want_b=True)
    E0 = _oracle_step(oracle, m, x, y, z, at_cathode=True)
    assert field_err(E1, E0)[0] <= 1e-5
    assert field_err(E1, E2)[0] <= 1e-6
    for comp in range(2):
        assert np.abs(B1[:, comp] - B2[:, comp]).max() <= 1e-6 * np.abs(B2[:, comp]).max()


@pytest.mark.parametrize("precision", [osc.PREC_FP32, osc.PREC_FP64])
def test_sorted_segment_deposit_is_bit_identical_to_fixed_point(oracle, precision):
    x, y, z = gendist(300_000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=44)
    q = np.random.default_rng(6).uniform(0.2, 2.0, len(x)) * 1e-15
    perm = np.random.default_rng(7).permutation(len(x))
    n = (32, 32, 48)
    rhos, Es = [], []
    with osc.Context(0) as c:
        m = _mesh(oracle, x, y, z, n)
        for mode, order in [(osc.DEPOSIT_DETERMINISTIC, osc.ORDER_ANY), (osc.DEPOSIT_SORTED_SEGMENT, osc.ORDER_ANY),
                            (osc.DEPOSIT_SORTED_SEGMENT, osc.ORDER_SORT)]:
            c.set_option(osc.OPT_DEPOSIT_MODE, mode)
            c.set_option(osc.OPT_PARTICLE_ORDER, order)
            for idx in (np.arange(len(x)), perm):
                mm = _mesh(oracle, x, y, z, n)
                osc.deposit_particles(c, x[idx], y[idx], z[idx], mm, qa=q[idx], resize_mesh=False)
                rhos.append(mm.rho.copy())
                E, _ = osc.space_charge_step(c, mm, x[idx], y[idx], z[idx], qa=q[idx], resize_mesh=False,
                                             precision=precision)
                inv = np.empty_like(idx)
                inv[idx] = np.arange(len(idx))
                Es.append(E[inv])
    for r in rhos[1:]:
        assert np.array_equal(r, rhos[0])
    for e in Es[1:]:
        assert np.array_equal(e, Es[0])
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), m.min, m.max, m.delta, GAMMA)
    ref, _ = oracle.deposit_particles(x, y, z, om, qa=q, resize_mesh=False)
    assert np.abs(rhos[0] - ref).max() <= 1e-13 * np.abs(ref).max()


def test_run_deposit_with_cell_order_promise_broken_is_still_correct(oracle):
    """ORDER_CELL_SORTED on random input: every particle is its own run."""
    x, y, z = gendist(300_000, sigma=(1e-3, 1e-3, 1e-3), seed=45)
    n = (20, 20, 20)
    with osc.Context(0) as c:
        c.set_option(osc.OPT_PARTICLE_ORDER, osc.ORDER_CELL_SORTED)
        m = _mesh(oracle, x, y, z, n)
        E1, _ = osc.space_charge_step(c, m, x, y, z, total_charge=1e-9, resize_mesh=False, precision=osc.PREC_FP32)
    E0 = _oracle_step(oracle, m, x, y, z)
    assert field_err(E1, E0)[0] <= 1e-5
