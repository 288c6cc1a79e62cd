"""GPU parity of the legacy free-space solver, the legacy cathode-image methods and the
rectangular pipe against the FP64 oracle (tolerances as in test_gpu_freespace)."""
import os

import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200 import native
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu

TOL = {osc.PREC_FP64_PLAIN: 1e-10, osc.PREC_FP64: 1e-10, osc.PREC_FP32: 1e-5}
# E of the pipe is the central difference of phi (core:588-605), which amplifies phi's
# normwise error by about max|phi| / (max|E| * delta); FP64 keeps 10x the phi bar, FP32 the
# accuracy bar of the FP32 path
E_TOL = {osc.PREC_FP64_PLAIN: 1e-9, osc.PREC_FP64: 1e-9, osc.PREC_FP32: 1e-5}


def bunch_mesh(oracle, n, npart=60000, sigma=(1e-3, 1e-3, 0.5e-3), seed=5, centroid=(0, 0, 0), isetzmin=0):
    x, y, z = gendist(npart, sigma=sigma, seed=seed, centroid=centroid)
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, isetzmin)
    rho, _ = oracle.depose_rho_scalar(x, y, z, 1e-9 / npart, (1, 1, 1), n, delta, umin)
    umax = umin + (np.array(n) - 1) * delta
    return rho, delta, umin, umax


@pytest.mark.parametrize("direct", [True, False])
def test_legacy_freespace_matches_oracle(ctx, oracle, direct):
    n = (12, 16, 10)
    rho, delta, umin, umax = bunch_mesh(oracle, n)
    gam = 3.0
    phi0, e0, b0 = oracle.freespace_solver(rho, gam, delta, (1, 1, 1), n, direct=direct)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umax, delta=delta, gamma=gam)
    m.rho = rho
    osc.space_charge_freespace(ctx, m, direct_field_calc=direct)
    mx, _ = field_err(m.efield, e0)
    assert mx <= 1e-10, mx
    for c in range(2):
        assert np.abs(m.bfield[..., c] - b0[..., c]).max() <= 1e-10 * np.abs(b0[..., c]).max()
    if not direct:
        assert np.abs(m.phi - phi0).max() <= 1e-10 * np.abs(phi0).max()


def test_legacy_freespace_rejects_direct_without_igf(ctx, oracle):
    n = (8, 8, 8)
    rho, delta, umin, umax = bunch_mesh(oracle, n, npart=5000)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umax, delta=delta, gamma=2.0)
    m.rho = rho
    with pytest.raises(osc.OscError) as ei:
        osc.space_charge_freespace(ctx, m, direct_field_calc=True, integrated_green_function=False)
    assert ei.value.code == native.OSC_E_UNSUPPORTED


@pytest.mark.parametrize("imethod", [1, 2])
@pytest.mark.parametrize("direct", [True, False])
def test_legacy_cathode_matches_oracle(ctx, oracle, imethod, direct):
    n = (12, 12, 16)
    rho, delta, umin, umax = bunch_mesh(oracle, n, centroid=(0, 0, 2e-3), isetzmin=1)
    gam = 1e6 / 0.510998910e6
    phi0, e0, b0, rho_after = oracle.cathodeimages_solver(rho, gam, umin, delta, (1, 1, 1), n, direct=direct,
                                                          imethod=imethod)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umax, delta=delta, gamma=gam)
    m.rho = rho.copy(order="F")
    osc.space_charge_cathodeimages(ctx, m, direct_field_calc=direct, image_method=imethod)
    mx, _ = field_err(m.efield, e0)
    assert mx <= 1e-10, mx
    for c in range(2):
        assert np.abs(m.bfield[..., c] - b0[..., c]).max() <= 1e-10 * np.abs(b0[..., c]).max()
    assert np.array_equal(m.rho, rho_after)


@pytest.fixture(scope="module")
def pipe_case(oracle):
    a, b = 20e-3, 10e-3
    n = (16, 16, 24)
    x, y, z = gendist(60000, sigma=(2e-3, 1e-3, 1e-3), seed=9, pipe=(a, b), centroid=(3e-3, -1e-3, 0))
    umin = np.array([-a / 2, -b / 2, -6e-3])
    delta = np.array([a / (n[0] - 1), b / (n[1] - 1), 12e-3 / (n[2] - 1)])
    umax = umin + (np.array(n) - 1) * delta
    rho, _ = oracle.depose_rho_scalar(x, y, z, 1e-9 / len(x), (1, 1, 1), n, delta, umin)
    gam = 5e6 / 0.510998910e6
    grn = oracle.getgrnpipe(gam, a, b, delta, umin, (1, 1, 1), n)
    phi0, e0, b0 = oracle.rectpipe_solver(rho, grn, gam, delta, (1, 1, 1), n)
    return dict(a=a, b=b, n=n, umin=umin, umax=umax, delta=delta, rho=rho, gam=gam, phi=phi0, e=e0, bf=b0,
                x=x, y=y, z=z)


@pytest.mark.parametrize("prec", [osc.PREC_FP64_PLAIN, osc.PREC_FP64, osc.PREC_FP32])
def test_rectpipe_matches_oracle(ctx, pipe_case, prec):
    c = pipe_case
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=c["n"], min=c["umin"], max=c["umax"], delta=c["delta"], gamma=c["gam"])
    m.rho = c["rho"]
    osc.osc_rectpipe_green(ctx, m, c["a"], c["b"], precision=prec)
    osc.space_charge_rectpipe(ctx, m, c["a"], c["b"], direct_field_calc=False, precision=prec)
    pm = np.abs(m.phi - c["phi"]).max() / np.abs(c["phi"]).max()
    mx, _ = field_err(m.efield, c["e"])
    print(f"pipe prec={prec}: phi {pm:.3e} E {mx:.3e}")
    assert pm <= TOL[prec] and mx <= E_TOL[prec], (pm, mx)


def test_rectpipe_reference_errors(ctx, pipe_case):
    c = pipe_case
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=c["n"], min=c["umin"], max=c["umax"], delta=c["delta"], gamma=c["gam"])
    m.rho = c["rho"]
    with pytest.raises(osc.OscError) as ei:
        osc.space_charge_rectpipe(ctx, m, c["a"], c["b"])  # default direct_field_calc, as the reference
    assert ei.value.code == native.OSC_E_UNSUPPORTED
    m2 = osc.Mesh3D(nlo=(1, 1, 1), nhi=(10, 10, 10), min=c["umin"], max=c["umax"], delta=c["delta"], gamma=c["gam"])
    m2.rho = np.zeros((10, 10, 10), order="F")
    with pytest.raises(osc.OscError) as ei:
        osc.space_charge_rectpipe(ctx, m2, c["a"], c["b"], direct_field_calc=False)
    assert ei.value.code == native.OSC_E_STATE


def test_rectpipe_green_file_roundtrip(ctx, pipe_case, tmp_path):
    c = pipe_case
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=c["n"], min=c["umin"], max=c["umax"], delta=c["delta"], gamma=c["gam"])
    m.rho = c["rho"]
    osc.osc_rectpipe_green(ctx, m, c["a"], c["b"], precision=osc.PREC_FP64_PLAIN)
    path = tmp_path / "rectpipegrn.dat"
    osc.osc_write_rectpipe_grn(ctx, path, c["a"], c["b"], m)
    raw = path.read_bytes()
    # record 1: 4-byte marker, 11 doubles, 9 int32, 1 double, marker
    assert int.from_bytes(raw[:4], "little") == 132 and int.from_bytes(raw[136:140], "little") == 132
    hdr = np.frombuffer(raw[4:92], dtype=np.float64)
    assert hdr[0] == c["a"] and hdr[1] == c["b"] and np.array_equal(hdr[2:5], c["delta"])
    ints = np.frombuffer(raw[92:128], dtype=np.int32)
    assert list(ints[3:6]) == list(c["n"]) and list(ints[6:9]) == [2 * v for v in c["n"]]
    osc.space_charge_rectpipe(ctx, m, c["a"], c["b"], direct_field_calc=False, precision=osc.PREC_FP64_PLAIN)
    phi_a = m.phi.copy()
    ctx2 = osc.Context(0)
    a, b = osc.osc_read_rectpipe_grn(ctx2, path, m)
    assert (a, b) == (c["a"], c["b"])
    osc.space_charge_rectpipe(ctx2, m, c["a"], c["b"], direct_field_calc=False, precision=osc.PREC_FP64_PLAIN)
    assert np.array_equal(m.phi, phi_a)
    ctx2.close()


@pytest.mark.parametrize("prec", [osc.PREC_FP64_PLAIN, osc.PREC_FP64, osc.PREC_FP32])
def test_fused_pipe_step_matches_oracle(ctx, oracle, pipe_case, prec):
    """deposit + space_charge_rectpipe + interpolate_field in one device call against the
    oracle's chain (depose_rho_scalar, osc_rectpipe_solver, interpolate_field)."""
    torch = pytest.importorskip("torch")
    c = pipe_case
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=c["n"], min=c["umin"], max=c["umax"], delta=c["delta"], gamma=c["gam"])
    osc.osc_rectpipe_green(ctx, m, c["a"], c["b"], precision=prec)
    dev = torch.device("cuda", 0)
    tx, ty, tz = (torch.from_numpy(v).to(dev) for v in (c["x"], c["y"], c["z"]))
    E = torch.empty((len(c["x"]), 3), dtype=torch.float64, device=dev)
    B = torch.empty_like(E)
    osc.space_charge_step_rectpipe_dev(ctx, m, tx, ty, tz, E, c["a"], c["b"], total_charge=1e-9, precision=prec,
                                       B=B)
    ctx.synchronize()
    om = oracle.make_mesh((1, 1, 1), c["n"], (1, 1, 1), c["umin"], c["umax"], c["delta"], c["gam"])
    E0, B0, _ = oracle.interpolate_field(om, c["e"], c["x"], c["y"], c["z"], bfield=c["bf"])
    mx, _ = field_err(E.cpu().numpy(), E0)
    bm = np.abs(B.cpu().numpy()[:, :2] - B0[:, :2]).max() / np.abs(B0[:, :2]).max()
    print(f"fused pipe prec={prec}: E {mx:.3e} B {bm:.3e}")
    assert mx <= E_TOL[prec], mx
    assert bm <= E_TOL[prec], bm


def test_fused_pipe_step_without_b(ctx, oracle, pipe_case):
    """FP32 fused pipe step with no B requested: E goes from phi straight to the x-pair grid.
    Same fields as the call that also computes B (float atomics reorder: 2e-6) and as the
    oracle's chain."""
    torch = pytest.importorskip("torch")
    c = pipe_case
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=c["n"], min=c["umin"], max=c["umax"], delta=c["delta"], gamma=c["gam"])
    osc.osc_rectpipe_green(ctx, m, c["a"], c["b"], precision=osc.PREC_FP32)
    dev = torch.device("cuda", 0)
    tx, ty, tz = (torch.from_numpy(v).to(dev) for v in (c["x"], c["y"], c["z"]))
    E1 = torch.empty((len(c["x"]), 3), dtype=torch.float64, device=dev)
    E2, B2 = torch.empty_like(E1), torch.empty_like(E1)
    osc.space_charge_step_rectpipe_dev(ctx, m, tx, ty, tz, E1, c["a"], c["b"], total_charge=1e-9,
                                       precision=osc.PREC_FP32)
    osc.space_charge_step_rectpipe_dev(ctx, m, tx, ty, tz, E2, c["a"], c["b"], total_charge=1e-9,
                                       precision=osc.PREC_FP32, B=B2)
    ctx.synchronize()
    E1, E2 = E1.cpu().numpy(), E2.cpu().numpy()
    mx, _ = field_err(E1, E2)
    assert mx <= 2e-6, mx
    om = oracle.make_mesh((1, 1, 1), c["n"], (1, 1, 1), c["umin"], c["umax"], c["delta"], c["gam"])
    E0, _, _ = oracle.interpolate_field(om, c["e"], c["x"], c["y"], c["z"])
    mx, _ = field_err(E1, E0)
    assert mx <= E_TOL[osc.PREC_FP32], mx
