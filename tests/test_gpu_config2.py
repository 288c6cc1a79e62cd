"""The headline configuration pinned to the FP64 oracle at its full size.

128x128x256 grid, 10^7 particles from a seeded Gaussian (sigma 0.5, 0.5, 2 mm, cut at
4 sigma), 1 nC, gamma = 5 MeV / m_e c^2, test-path mesh (get_mesh_quantities).  Both the
free-space case and the cathode-image case (centroid at z = 3 mm, cathode at z = 0,
samples at z <= 0 dropped and counted, mesh with zmin pinned to 1e-9 as the reference's
test driver does for cathodes, code/test_opensc.f90:141-142) run the fused step on the GPU
(deposit_particles + space_charge_3d + interpolate_field, code/open_spacecharge_mod.f90:
156-288, 431-489, 311-390) and the same three routines in the oracle, on the same arrays.

Error: per component, max|E - E_oracle| / max|E_oracle| and the RMS ratio, over all
particles.  Tolerances: FP32 1e-5 (the accuracy bar of the FP32 path); FP64 1e-9: at this
size both FP64 paths differ from the oracle by 1e-10 to 3e-10 (FP64 round-off of 33.5-million-
point transforms, amplified by the IGF corner-difference cancellation, and, with the cathode,
of the image kernel's full doubled-grid transform), against 1e-11 at 64^3.
"""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist

pytestmark = pytest.mark.gpu

GRID = (128, 128, 256)
NPART = 10_000_000
SIGMA = (0.5e-3, 0.5e-3, 2e-3)
QTOT = 1e-9
GAMMA = 5e6 / 0.510998910e6
TOL = {osc.PREC_FP32: 1e-5, osc.PREC_FP64: 1e-9}


def _errors(E, ref):
    mx = [float(np.abs(E[:, c] - ref[:, c]).max() / np.abs(ref[:, c]).max()) for c in range(3)]
    rms = [float(np.sqrt(np.mean((E[:, c] - ref[:, c]) ** 2)) / np.sqrt(np.mean(ref[:, c] ** 2))) for c in range(3)]
    return mx, rms


@pytest.fixture(scope="module", params=["free", "cathode"])
def case(request, oracle):
    cathode = request.param == "cathode"
    x, y, z = gendist(NPART, sigma=SIGMA, cutoff=4.0, disttype=1, seed=1,
                      centroid=(0.0, 0.0, 3e-3 if cathode else 0.0))
    dropped = 0
    if cathode:
        keep = z > 0.0
        dropped = int((~keep).sum())
        x, y, z = (np.ascontiguousarray(v[keep]) for v in (x, y, z))
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), GRID, 1 if cathode else 0)
    umax = umin + (np.array(GRID) - 1) * delta
    om = oracle.make_mesh((1, 1, 1), GRID, (1, 1, 1), umin, umax, delta, GAMMA)
    rho, nout = oracle.deposit_particles(x, y, z, om, total_charge=QTOT, resize_mesh=False)
    ef, _ = oracle.space_charge_3d(om, rho, at_cathode=cathode)
    E_ref, _, _ = oracle.interpolate_field(om, ef, x, y, z)
    return dict(cathode=cathode, x=x, y=y, z=z, umin=umin, umax=umax, delta=delta, E_ref=E_ref,
                dropped=dropped, n_outside=nout)


@pytest.mark.parametrize("prec", [osc.PREC_FP32, osc.PREC_FP64])
def test_headline_config_matches_oracle(ctx, case, prec):
    if case["cathode"]:
        # the image case drops the samples behind the cathode and counts them
        assert 0 < case["dropped"] < NPART // 2
        assert case["umin"][2] == 1e-9
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=GRID, min=case["umin"].copy(), max=case["umax"].copy(),
                   delta=case["delta"].copy(), gamma=GAMMA)
    E, _ = osc.space_charge_step(ctx, m, case["x"], case["y"], case["z"], total_charge=QTOT, resize_mesh=False,
                                 at_cathode=case["cathode"], precision=prec)
    assert m.charge == QTOT
    mx, rms = _errors(E, case["E_ref"])
    print(f"{'cathode' if case['cathode'] else 'free'} prec={prec}: max {mx} rms {rms} dropped {case['dropped']} "
          f"outside {case['n_outside']}")
    assert max(mx) <= TOL[prec], (mx, rms)
    assert max(rms) <= TOL[prec], (mx, rms)
