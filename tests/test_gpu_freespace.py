"""GPU parity of the free-space IGF solves against the FP64 oracle.

Tolerances (normwise, per component: max|E-E_ref|/max|E_ref|):
  OSC_PREC_FP64_PLAIN and OSC_PREC_FP64: 1e-10 (FP64 roundoff amplified by the IGF
    corner-difference cancellation and by different FFT factorisations);
  OSC_PREC_FP32: 1e-5, the accuracy bar of the FP32 path.
"""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu

TOL = {osc.PREC_FP64_PLAIN: 1e-10, osc.PREC_FP64: 1e-10, osc.PREC_FP32: 1e-5}
PRECS = [osc.PREC_FP64_PLAIN, osc.PREC_FP64, osc.PREC_FP32]


def make_rho(oracle, n, npart=100000, sigma=(1e-3, 1e-3, 0.4e-3), seed=21, centroid=(0, 0, 0), isetzmin=0):
    x, y, z = gendist(npart, sigma=sigma, seed=seed, centroid=centroid)
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, isetzmin)
    rho, ifail = oracle.depose_rho_scalar(x, y, z, 1e-9 / npart, (1, 1, 1), n, delta, umin)
    umax = umin + (np.array(n) - 1) * delta
    return rho, delta, umin, umax


@pytest.mark.parametrize("n", [(16, 12, 20), (12, 24, 18), (10, 10, 10), (8, 8, 40)])
@pytest.mark.parametrize("prec", PRECS)
def test_solver2_matches_oracle(ctx, oracle, n, prec):
    rho, delta, _, _ = make_rho(oracle, n)
    gamma = 9.784756683727565
    e_ref, p_ref = oracle.freespace_solver2(rho, gamma, delta, want_phi=True)
    e, p = osc.osc_freespace_solver2(ctx, rho, gamma, delta, efield=True, phi=True, precision=prec)
    mx, rm = field_err(e, e_ref)
    pm = np.abs(p - p_ref).max() / np.abs(p_ref).max()
    assert mx <= TOL[prec] and pm <= TOL[prec], (mx, rm, pm)


@pytest.mark.parametrize("prec", PRECS)
def test_solver2_with_offset_matches_oracle(ctx, oracle, prec):
    n = (12, 10, 16)
    rho, delta, _, _ = make_rho(oracle, n)
    off = (3.0e-4, -2.0e-4, 1.0e-3)
    e_ref, _ = oracle.freespace_solver2(rho, 2.0, delta, offset=off)
    e, _ = osc.osc_freespace_solver2(ctx, rho, 2.0, delta, offset=off, precision=prec)
    mx, rm = field_err(e, e_ref)
    assert mx <= TOL[prec], (mx, rm)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("at_cathode", [False, True])
def test_space_charge_3d_matches_oracle(ctx, oracle, prec, at_cathode):
    n = (16, 16, 24)
    rho, delta, umin, umax = make_rho(oracle, n, centroid=(0, 0, 3e-3), isetzmin=1 if at_cathode else 0)
    gamma = 9.784756683727565
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umax, delta, gamma)
    e_ref, b_ref = oracle.space_charge_3d(om, rho, at_cathode=at_cathode, calc_bfield=True)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin.copy(), max=umax.copy(), delta=delta.copy(), gamma=gamma)
    m.rho = rho
    osc.space_charge_3d(ctx, m, at_cathode=at_cathode, calc_bfield=True, precision=prec)
    mx, rm = field_err(m.efield, e_ref)
    assert mx <= TOL[prec], (mx, rm)
    for c in range(2):
        bm = np.abs(m.bfield[..., c] - b_ref[..., c]).max() / np.abs(b_ref[..., c]).max()
        assert bm <= TOL[prec], (c, bm)
    assert np.all(m.bfield[..., 2] == 0)


def test_fp32_vs_fp64_at_64cubed(ctx, oracle):
    """Config-1 sized grid: the FP32 path against the GPU FP64 path (both vs the oracle too)."""
    n = (64, 64, 64)
    rho, delta, umin, umax = make_rho(oracle, n, npart=1_000_000, sigma=(1e-3, 1e-3, 0.3e-3))
    gamma = 9.784756683727565
    e_ref, _ = oracle.freespace_solver2(rho, gamma, delta)
    e32, _ = osc.osc_freespace_solver2(ctx, rho, gamma, delta, precision=osc.PREC_FP32)
    e64, _ = osc.osc_freespace_solver2(ctx, rho, gamma, delta, precision=osc.PREC_FP64)
    mx32, rm32 = field_err(e32, e_ref)
    mx64, _ = field_err(e64, e_ref)
    assert mx64 <= 1e-10
    assert mx32 <= 1e-5 and rm32 <= 1e-5, (mx32, rm32)


def test_unsupported_fft_length_is_an_error(ctx):
    rho = np.zeros((7, 8, 8), order="F")  # doubled length 14 = 2*7 has a factor 7
    with pytest.raises(osc.OscError) as ei:
        osc.osc_freespace_solver2(ctx, rho, 1.0, (1e-4, 1e-4, 1e-4), precision=osc.PREC_FP32)
    assert ei.value.code == osc.native.OSC_E_FFT_SIZE


def test_green_cache_reuse_is_exact(ctx, oracle):
    n = (16, 16, 16)
    rho, delta, _, _ = make_rho(oracle, n)
    a, _ = osc.osc_freespace_solver2(ctx, rho, 3.0, delta, precision=osc.PREC_FP32)
    b, _ = osc.osc_freespace_solver2(ctx, rho, 3.0, delta, precision=osc.PREC_FP32)
    assert np.array_equal(a, b)
    ctx.clear_green_cache()
    c, _ = osc.osc_freespace_solver2(ctx, rho, 3.0, delta, precision=osc.PREC_FP32)
    assert np.array_equal(a, c)


@pytest.mark.parametrize("n", [(16, 12, 256), (24, 20, 256)])
def test_z_pass_engines_at_length_512_agree_with_oracle(oracle, n):
    """Doubled z length 512 with staged Green spectra has three FP32 engines: the radix-8 warp
    engine (the default), one exchange per transform (16 x 32 split with a radix-2 lane-pair
    shuffle) and the warp engine with rows ky and Ny - ky paired on one CTA; all must match
    the oracle, and each other to FP32 round-off."""
    rho, delta, _, _ = make_rho(oracle, n, sigma=(1e-3, 1e-3, 3e-3))
    gamma = 9.784756683727565
    e_ref, _ = oracle.freespace_solver2(rho, gamma, delta)
    out = []
    with osc.Context(0) as c:
        for engine in (0, 1, 2):
            c.set_tuning("zconv_engine:f32:L512", engine)
            e, _ = osc.osc_freespace_solver2(c, rho, gamma, delta, precision=osc.PREC_FP32)
            mx, rm = field_err(e, e_ref)
            assert mx <= 1e-5 and rm <= 1e-5, (engine, mx, rm)
            out.append(e)
    assert field_err(out[0], out[1])[0] <= 2e-6
    assert field_err(out[0], out[2])[0] <= 2e-6


@pytest.mark.parametrize("nz", [48, 64, 96, 128, 192])
@pytest.mark.parametrize("prec", [osc.PREC_FP64, osc.PREC_FP32])
def test_paired_z_engine_matches_oracle(oracle, nz, prec):
    """Engine 2 of the z pass (one CTA per pair of rows ky, Ny - ky sharing their Green
    columns) at the warp lengths it covers (doubled z 96, 128, 256, 384; at 192 the pass
    keeps engine 0), against the oracle and against engine 0."""
    n = (12, 10, nz)
    rho, delta, _, _ = make_rho(oracle, n, sigma=(1e-3, 1e-3, 2e-3))
    gamma = 9.784756683727565
    e_ref, _ = oracle.freespace_solver2(rho, gamma, delta)
    tag = "f32" if prec == osc.PREC_FP32 else "f64"
    out = []
    with osc.Context(0) as c:
        for engine in (0, 2):
            c.set_tuning(f"zconv_engine:{tag}:L{2 * nz}", engine)
            e, _ = osc.osc_freespace_solver2(c, rho, gamma, delta, precision=prec)
            mx, rm = field_err(e, e_ref)
            assert mx <= TOL[prec], (engine, mx, rm)
            out.append(e)
    assert field_err(out[0], out[1])[0] <= (2e-6 if prec == osc.PREC_FP32 else 1e-13)


@pytest.mark.parametrize("nz", [48, 64, 96, 128, 192])
@pytest.mark.parametrize("prec", [osc.PREC_FP64, osc.PREC_FP32])
def test_cathode_image_z_pass_lengths_match_oracle(ctx, oracle, nz, prec):
    """The image z pass (both Green columns staged, image spectra stored for kz <= nz with
    the z-flip phase applied, the mirrored spectrum taken by warp shuffles) at every warp
    length it covers -- doubled z 96, 128, 256, 384 -- and the general image path at 192;
    with B, whose two extra outputs add the image with the opposite sign."""
    n = (12, 10, nz)
    rho, delta, umin, umax = make_rho(oracle, n, sigma=(1e-3, 1e-3, 2e-3), centroid=(0, 0, 6e-3), isetzmin=1)
    gamma = 9.784756683727565
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umax, delta, gamma)
    e_ref, b_ref = oracle.space_charge_3d(om, rho, at_cathode=True, calc_bfield=True)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin.copy(), max=umax.copy(), delta=delta.copy(), gamma=gamma)
    m.rho = rho
    osc.space_charge_3d(ctx, m, at_cathode=True, calc_bfield=True, precision=prec)
    mx, rm = field_err(m.efield, e_ref)
    assert mx <= TOL[prec], (mx, rm)
    for c in range(2):
        bm = np.abs(m.bfield[..., c] - b_ref[..., c]).max() / np.abs(b_ref[..., c]).max()
        assert bm <= TOL[prec], (c, bm)
