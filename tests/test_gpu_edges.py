"""Edge cases of the GPU path against the FP64 oracle: particles exactly on cell planes and on
the top face of the mesh (the cell index is bit-exact: code/open_spacecharge_mod.f90:259-261
and :320-322 evaluate floor((x-min)*dxi+1) without a fused multiply-add), the largest FFT
length the solver accepts (doubled grid 2048) and the first length past it, non-finite
coordinates, empty and inconsistent inputs (error codes, no crash)."""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200 import native
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu


def plane_particles(n, umin, delta, seed):
    """Every particle has at least one coordinate exactly on a node plane, including the top
    face (index n-1, outside the deposit stencil) and the bottom face (index 0)."""
    rng = np.random.default_rng(seed)
    m = 4000
    idx = np.stack([rng.integers(0, n[d], m) for d in range(3)], 1)
    pos = umin + idx * delta
    frac = rng.uniform(0.0, 1.0, (m, 3)) * delta
    on = rng.integers(0, 2, (m, 3)).astype(bool)
    on[:, 0] |= ~on.any(1)
    pos = np.where(on, pos, np.minimum(pos + frac, umin + (np.array(n) - 1) * delta))
    return pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()


@pytest.fixture(scope="module")
def plane_case():
    n = (16, 20, 24)
    umin = np.array([-1.1e-3, -0.73e-3, -2.3e-3])
    delta = np.array([1.37e-4, 0.71e-4, 2.09e-4])
    return n, umin, delta, plane_particles(n, umin, delta, 61)


def test_plane_particles_deposit_matches_oracle(ctx, oracle, plane_case):
    n, umin, delta, (x, y, z) = plane_case
    umax = umin + (np.array(n) - 1) * delta
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin.copy(), max=umax.copy(), delta=delta.copy())
    nout = osc.deposit_particles(ctx, x, y, z, m, total_charge=1e-9, resize_mesh=False)
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umax, delta, 1.0)
    ref, nref = oracle.deposit_particles(x, y, z, om, total_charge=1e-9, resize_mesh=False)
    assert nout == nref > 0  # the top-face particles are outside, identically
    assert np.abs(m.rho - ref).max() <= 1e-13 * np.abs(ref).max()


def test_plane_particles_interpolation_matches_oracle(ctx, oracle, plane_case):
    n, umin, delta, (x, y, z) = plane_case
    umax = umin + (np.array(n) - 1) * delta
    ef = np.asfortranarray(np.random.default_rng(62).normal(size=tuple(n) + (3,)))
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin.copy(), max=umax.copy(), delta=delta.copy())
    m.efield = ef
    E, _, ncl = osc.interpolate_field(ctx, x, y, z, m)
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umax, delta, 1.0)
    E0, _, ncl0 = oracle.interpolate_field(om, ef, x, y, z)
    assert ncl == ncl0 > 0
    assert np.abs(E - E0).max() <= 1e-13 * np.abs(E0).max()


@pytest.mark.parametrize("prec", [osc.PREC_FP64, osc.PREC_FP32])
def test_largest_fft_length(ctx, oracle, prec):
    """nz = 1024: the doubled z length 2048 is the largest the solver takes."""
    n = (8, 8, 1024)
    x, y, z = gendist(100000, sigma=(1e-3, 1e-3, 20e-3), seed=63)
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    umax = umin + (np.array(n) - 1) * delta
    rho, _ = oracle.depose_rho_scalar(x, y, z, 1e-9 / len(x), (1, 1, 1), n, delta, umin)
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umax, delta, 9.785)
    e0, _ = oracle.space_charge_3d(om, rho)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umax, delta=delta, gamma=9.785)
    m.rho = rho
    osc.space_charge_3d(ctx, m, precision=prec)
    mx, _ = field_err(m.efield, e0)
    assert mx <= (1e-10 if prec == osc.PREC_FP64 else 1e-5), mx


def test_fft_length_past_the_largest_is_an_error(ctx):
    n = (8, 8, 1200)  # doubled 2400 = 2^5 3 5^2: a valid radix mix, but above 2048
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=np.zeros(3), max=np.array([7e-3, 7e-3, 1.199]),
                   delta=np.full(3, 1e-3), gamma=2.0)
    m.rho = np.zeros(n, order="F")
    with pytest.raises(osc.OscError) as ei:
        osc.space_charge_3d(ctx, m)
    assert ei.value.code == native.OSC_E_FFT_SIZE


def test_nonfinite_coordinates(ctx):
    x, y, z = gendist(20000, seed=64)
    x[17] = np.nan
    z[123] = np.inf
    n = (16, 16, 16)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n)
    osc.deposit_particles(ctx, x[200:], y[200:], z[200:], m, total_charge=1e-9, resize_mesh=True)  # finite part
    fixed = dict(min=m.min.copy(), max=m.max.copy(), delta=m.delta.copy())
    # default: non-finite particles fall outside the mesh and are skipped and counted
    m1 = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, **fixed)
    nout = osc.deposit_particles(ctx, x, y, z, m1, total_charge=1e-9, resize_mesh=False)
    assert nout >= 2 and np.isfinite(m1.rho).all()
    # OSC_OPT_CHECK_FINITE: the deposit reports them
    c2 = osc.Context(0)
    c2.set_option(osc.OPT_CHECK_FINITE, 1)
    m2 = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, **fixed)
    with pytest.raises(osc.OscError) as ei:
        osc.deposit_particles(c2, x, y, z, m2, total_charge=1e-9, resize_mesh=False)
    assert ei.value.code == native.OSC_E_NAN
    c2.close()


def test_empty_and_inconsistent_inputs(ctx):
    n = (16, 16, 16)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=2.0)
    e = np.zeros(0)
    with pytest.raises(osc.OscError) as ei:
        osc.space_charge_step(ctx, m, e, e, e, total_charge=1e-9)
    assert ei.value.code == native.OSC_E_INVALID
    x, y, z = gendist(5000, seed=65)
    meshes = [osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=2.0) for _ in range(2)]
    with pytest.raises(osc.OscError) as ei:  # a bunch with no particles
        osc.batch_space_charge_step(ctx, meshes, x, y, z, [5000, 0], total_charges=[1e-9, 1e-9])
    assert ei.value.code == native.OSC_E_INVALID
    # the context stays usable after the errors
    E, _ = osc.space_charge_step(ctx, osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=2.0), x, y, z, total_charge=1e-9)
    assert np.isfinite(E).all() and np.abs(E).max() > 0
