"""GPU parity of the fused step (deposit -> field -> interpolation at every particle)
against the oracle's deposit_particles + space_charge_3d + interpolate_field chain.
Tolerances as in test_gpu_freespace (normwise per component at the particles)."""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu

TOL = {osc.PREC_FP64_PLAIN: 1e-10, osc.PREC_FP64: 1e-10, osc.PREC_FP32: 1e-5}


def oracle_step(oracle, x, y, z, n, gamma, total_charge, at_cathode=False, want_b=False):
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), (0, 0, 0), (0, 0, 0), (0, 0, 0), gamma)
    rho, nout = oracle.deposit_particles(x, y, z, om, total_charge=total_charge, resize_mesh=True)
    ef, bf = oracle.space_charge_3d(om, rho, at_cathode=at_cathode, calc_bfield=want_b)
    E, B, ncl = oracle.interpolate_field(om, ef, x, y, z, bfield=bf)
    return E, B, om


@pytest.mark.parametrize("prec", [osc.PREC_FP64_PLAIN, osc.PREC_FP64, osc.PREC_FP32])
@pytest.mark.parametrize("at_cathode", [False, True])
def test_step_matches_oracle(ctx, oracle, prec, at_cathode):
    n = (24, 24, 32)
    x, y, z = gendist(200000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=31, centroid=(0, 0, 3e-3 if at_cathode else 0))
    gamma = 9.784756683727565
    E0, B0, om = oracle_step(oracle, x, y, z, n, gamma, 1e-9, at_cathode, want_b=True)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=gamma)
    E1, B1 = osc.space_charge_step(ctx, m, x, y, z, total_charge=1e-9, resize_mesh=True, at_cathode=at_cathode,
                                   precision=prec, want_b=True)
    assert np.array_equal(m.delta, np.array(om.delta[:]))
    mx, rm = field_err(E1, E0)
    assert mx <= TOL[prec], (mx, rm)
    for c in range(2):
        bm = np.abs(B1[:, c] - B0[:, c]).max() / np.abs(B0[:, c]).max()
        assert bm <= TOL[prec], (c, bm)


def test_step_dev_matches_host_step(ctx):
    torch = pytest.importorskip("torch")
    n = (32, 32, 32)
    x, y, z = gendist(300000, sigma=(1e-3, 1e-3, 1e-3), seed=41)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=2.0)
    E1, _ = osc.space_charge_step(ctx, m, x, y, z, total_charge=1e-9, resize_mesh=True, precision=osc.PREC_FP32)
    dev = torch.device("cuda", 0)
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    E = torch.empty((len(x), 3), dtype=torch.float64, device=dev)
    m2 = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=2.0, min=m.min.copy(), max=m.max.copy(), delta=m.delta.copy())
    osc.space_charge_step_dev(ctx, m2, tx, ty, tz, E, total_charge=1e-9, resize_mesh=False, precision=osc.PREC_FP32)
    ctx.synchronize()
    E2 = E.cpu().numpy()
    mx, _ = field_err(E2, E1)
    assert mx < 1e-6  # float atomics reorder; same pipeline otherwise
