"""CPU tests of the FP64 oracle: golden values printed by the reference, the reference's
published cross-method differences, and analytic known-answer tests."""
import json
import os

import numpy as np
import pytest

from conftest import field_err

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "notebook_runs.json")))


@pytest.mark.parametrize("shape", [(8, 6, 10), (16, 12, 20), (24, 10, 14), (14, 7, 5)])
@pytest.mark.parametrize("idir", [(1, 1, 1), (-1, -1, -1), (1, -1, 1), (-1, 1, -1)])
def test_fft_matches_numpy(oracle, shape, idir):
    rng = np.random.default_rng(0)
    a = np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    b = oracle.ccfft3d(a, idir)
    ref = a.copy()
    for ax, s in enumerate(idir):
        n = shape[ax]
        ref = np.fft.ifft(ref, axis=ax) * n if s > 0 else np.fft.fft(ref, axis=ax)
    assert np.abs(b - ref).max() / np.abs(ref).max() < 1e-14


def test_fft_unsupported_length(oracle):
    with pytest.raises(ValueError):
        oracle.ccfft3d(np.zeros((29 * 2, 4, 4), dtype=complex), (1, 1, 1))


@pytest.mark.parametrize("run", range(len(GOLD["runs"])))
def test_mesh_quantities_bit_exact_vs_reference_output(oracle, run):
    """get_mesh_quantities reproduces the mesh the reference printed for its own bunch."""
    r = GOLD["runs"][run]
    g = r["grid"]
    nlo = (g["nxlo"], g["nylo"], g["nzlo"])
    nhi = (g["nxhi"], g["nyhi"], g["nzhi"])
    x = np.array(r["particle xmin,xmax"])
    y = np.array(r["particle ymin,ymax"])
    z = np.array(r["particle zmin,zmax"])
    delta, umin = oracle.get_mesh_quantities(x, y, z, nlo, nhi, 0)
    umax = umin + (np.array(nhi) - np.array(nlo)) * delta
    assert list(delta) == r["delta(1:3)"]
    assert [umin[0], umax[0]] == r["mesh xmin,xmax"]
    assert [umin[1], umax[1]] == r["mesh ymin,ymax"]
    assert [umin[2], umax[2]] == r["mesh zmin,zmax"]


def _uniform_ball_cathode(oracle, n, npart, seed):
    from openspacecharge_b200.bunch import gendist
    x, y, z = gendist(npart, sigma=(1e-3, 1e-3, 1e-3), disttype=0, seed=seed, centroid=(0, 0, 1.2e-4))
    nlo, nhi = (1, 1, 1), (n, n, n)
    gamma = 1e6 / 0.510998910e6
    delta, umin = oracle.get_mesh_quantities(x, y, z, nlo, nhi, 1)
    umax = umin + (np.array(nhi) - 1) * delta
    rho, ifail = oracle.depose_rho_scalar(x, y, z, 1e-9 / npart, nlo, nhi, delta, umin)
    mesh = oracle.make_mesh(nlo, nhi, (1, 1, 1), umin, umax, delta, gamma)
    return mesh, rho, gamma, delta, umin, nlo, nhi


def test_cathode_cross_method_matches_published(oracle):
    """The three image methods agree to the orders the reference notebook publishes
    (examples/benchmark.ipynb cells 25-26: 1.75e-6 for 3 vs 1, 8.49e-11 for 2 vs 1) on a
    uniform 1 mm ball at 64^3, E=1 MeV, with Ez read on the y=0 plane through interpolate_field."""
    mesh, rho, gamma, delta, umin, nlo, nhi = _uniform_ball_cathode(oracle, 64, 1_000_000, 7)
    e3, _ = oracle.space_charge_3d(mesh, rho, at_cathode=True)
    _, e1, _, _ = oracle.cathodeimages_solver(rho, gamma, umin, delta, nlo, nhi, imethod=1)
    _, e2, _, _ = oracle.cathodeimages_solver(rho, gamma, umin, delta, nlo, nhi, imethod=2)
    xs = umin[0] + np.arange(nhi[0] - 1) * delta[0]
    zs = umin[2] + np.arange(nhi[2] - 1) * delta[2]
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    X, Z = X.ravel(), Z.ravel()
    Y = np.zeros_like(X)
    ez = [oracle.interpolate_field(mesh, e, X, Y, Z)[0][:, 2] for e in (e1, e2, e3)]
    d31 = np.abs(ez[2] / ez[0] - 1).max()
    d21 = np.abs(ez[1] / ez[0] - 1).max()
    pub = GOLD["cathode_cross_method"]
    assert 0.1 * pub["3v1"]["max_rel_Ez_diff"] < d31 < 10 * pub["3v1"]["max_rel_Ez_diff"]
    assert d21 < 30 * pub["2v1"]["max_rel_Ez_diff"]


def test_method2_flips_rho_in_place(oracle):
    mesh, rho, gamma, delta, umin, nlo, nhi = _uniform_ball_cathode(oracle, 16, 20000, 3)
    _, _, _, rho_after = oracle.cathodeimages_solver(rho, gamma, umin, delta, nlo, nhi, imethod=2)
    assert np.array_equal(rho_after, rho[:, :, ::-1])


def _gauss_rho(oracle, n, npart=200000, sigma=(1e-3, 1e-3, 0.5e-3), seed=11):
    from openspacecharge_b200.bunch import gendist
    x, y, z = gendist(npart, sigma=sigma, seed=seed)
    nlo, nhi = (1, 1, 1), n
    delta, umin = oracle.get_mesh_quantities(x, y, z, nlo, nhi, 0)
    rho, ifail = oracle.depose_rho_scalar(x, y, z, 1e-9 / npart, nlo, nhi, delta, umin)
    assert ifail == 0
    return rho, delta, umin, (x, y, z)


def test_legacy_solver_matches_solver2(oracle):
    """osc_freespace_solver (legacy, point IGFs, low-corner window) and
    osc_freespace_solver2 (corner differences, shifted window) compute the same field; they
    differ by the ratio of their 1/(4 pi eps0) constants and cancellation roundoff."""
    n = (16, 12, 20)
    rho, delta, umin, _ = _gauss_rho(oracle, n)
    gamma = 3.0
    e2, _ = oracle.freespace_solver2(rho, gamma, delta)
    _, el, bl = oracle.freespace_solver(rho, gamma, delta, (1, 1, 1), n)
    c = np.float32(299792458.0)
    ratio = (float(np.float32(c * c)) * 1.00000000055e-7) / (299792458.0 ** 2 * 1e-7)
    mx, rm = field_err(el * ratio, e2)
    assert mx < 1e-9 and rm < 1e-10
    beta = np.sqrt(1 - 1 / gamma ** 2)
    assert np.allclose(bl[..., 0], -el[..., 1] * beta / 299792458.0, rtol=0, atol=1e-30)
    assert np.all(bl[..., 2] == 0)


def _numpy_solver2(rho, gamma, delta, offset=(0, 0, 0)):
    """Independent numpy restatement of osc_get_cgrn_freespace + osc_freespace_solver2."""
    nx, ny, nz = rho.shape
    N = (2 * nx, 2 * ny, 2 * nz)
    dx, dy, dz = delta[0], delta[1], delta[2] * gamma
    u = (np.arange(N[0]) + 0.5 - N[0] // 2) * dx + offset[0]
    v = (np.arange(N[1]) + 0.5 - N[1] // 2) * dy + offset[1]
    w = (np.arange(N[2]) + 0.5 - N[2] // 2) * dz + offset[2] * gamma
    U, V, W = np.meshgrid(u, v, w, indexing="ij")

    def xla(x, y, z):
        r = np.sqrt(x * x + y * y + z * z)
        return x * np.arctan((y * z) / (r * x)) - z * np.log(r + y) + y * np.log((r - z) / (r + z)) / 2

    crho = np.zeros(N, dtype=complex)
    crho[:nx, :ny, :nz] = rho
    rh = np.fft.ifftn(crho) * np.prod(N)  # sign +1
    out = np.zeros(rho.shape + (3,))
    fpei = float(np.float32(np.float32(299792458.0) ** 2)) * 1.00000000055e-7
    for c in range(3):
        fac = gamma / (dx * dy * dz) if c < 2 else 1.0 / (dx * dy * dz)
        F = [xla(U, V, W), xla(V, W, U), xla(W, U, V)][c] * fac
        G = F.copy()
        G[:-1, :-1, :-1] = (F[1:, 1:, 1:] - F[:-1, 1:, 1:] - F[1:, :-1, 1:] - F[1:, 1:, :-1] - F[:-1, :-1, :-1]
                            + F[:-1, :-1, 1:] + F[:-1, 1:, :-1] + F[1:, :-1, :-1])
        gh = np.fft.ifftn(G) * np.prod(N)
        conv = np.fft.fftn(rh * gh)  # sign -1
        out[..., c] = fpei / np.prod(N) * conv[nx - 1:2 * nx - 1, ny - 1:2 * ny - 1, nz - 1:2 * nz - 1].real
    return out


@pytest.mark.parametrize("offset", [(0, 0, 0), (1e-4, -2e-4, 3e-3)])
def test_solver2_matches_numpy_restatement(oracle, offset):
    n = (8, 10, 12)
    rho, delta, umin, _ = _gauss_rho(oracle, n, npart=50000)
    gamma = 2.5
    e, _ = oracle.freespace_solver2(rho, gamma, delta, offset=offset)
    ref = _numpy_solver2(rho, gamma, delta, offset)
    mx, rm = field_err(e, ref)
    assert mx < 1e-10, mx


def test_point_charge_is_coulomb(oracle):
    """KAT: one macro-charge on a node gives the Coulomb field 1/(4 pi eps0) q r/|r|^3 far away."""
    n = (24, 24, 24)
    rho = np.zeros(n, order="F")
    q = 1e-12
    rho[4, 5, 6] = q
    delta = np.array([1e-4, 1e-4, 1e-4])
    e, _ = oracle.freespace_solver2(rho, 1.0, delta)
    fpei = float(np.float32(np.float32(299792458.0) ** 2)) * 1.00000000055e-7
    for node in [(20, 5, 6), (4, 21, 6), (4, 5, 22), (18, 17, 16)]:
        r = (np.array(node) - np.array([4, 5, 6])) * delta
        ref = fpei * q * r / np.linalg.norm(r) ** 3
        got = e[node]
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-3


def test_symmetric_bunch_field_parity(oracle):
    """KAT: a bunch symmetric under x -> -x gives Ex odd and Ey, Ez even in x."""
    n = (16, 12, 14)
    rho, delta, umin, _ = _gauss_rho(oracle, n, npart=40000)
    rho = 0.5 * (rho + rho[::-1, :, :])
    e, _ = oracle.freespace_solver2(rho, 1.5, delta)
    s = np.abs(e).max(axis=(0, 1, 2))
    assert np.abs(e[..., 0] + e[::-1, :, :, 0]).max() < 1e-12 * s[0]
    assert np.abs(e[..., 1] - e[::-1, :, :, 1]).max() < 1e-12 * s[1]
    assert np.abs(e[..., 2] - e[::-1, :, :, 2]).max() < 1e-12 * s[2]


def test_gauss_law_flux(oracle):
    """KAT: the E flux through a box enclosing the bunch is Q/eps0 (at gamma=1)."""
    n = (32, 32, 32)
    rho, delta, umin, _ = _gauss_rho(oracle, n, npart=100000, sigma=(0.5e-3, 0.5e-3, 0.5e-3))
    Q = rho.sum()
    e, _ = oracle.freespace_solver2(rho, 1.0, delta)
    a, b = 2, 29  # box faces at nodes a and b
    dx, dy, dz = delta
    flux = (e[b, a:b, a:b, 0].sum() - e[a, a:b, a:b, 0].sum()) * dy * dz
    flux += (e[a:b, b, a:b, 1].sum() - e[a:b, a, a:b, 1].sum()) * dx * dz
    flux += (e[a:b, a:b, b, 2].sum() - e[a:b, a:b, a, 2].sum()) * dx * dy
    fpei = float(np.float32(np.float32(299792458.0) ** 2)) * 1.00000000055e-7
    assert abs(flux / (4 * np.pi * fpei * Q) - 1) < 0.02


def test_deposit_conserves_charge_and_matches_depose_rho_scalar(oracle):
    from openspacecharge_b200.bunch import gendist
    x, y, z = gendist(20000, seed=5)
    n = (20, 18, 22)
    delta, umin = oracle.get_mesh_quantities(x, y, z, (1, 1, 1), n, 0)
    umax = umin + (np.array(n) - 1) * delta
    mesh = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umax, delta, 1.0)
    rho, nout = oracle.deposit_particles(x, y, z, mesh, total_charge=2e-9, resize_mesh=False)
    assert nout == 0
    assert abs(rho.sum() / 2e-9 - 1) < 1e-12
    rho2, ifail = oracle.depose_rho_scalar(x, y, z, 2e-9 / len(x), (1, 1, 1), n, delta, umin)
    assert ifail == 0
    assert np.abs(rho - rho2).max() < 1e-12 * np.abs(rho).max()
    # resize_mesh refits to the bunch with the 1e-6*delta pad
    mesh2 = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), (0, 0, 0), (0, 0, 0), (0, 0, 0), 1.0)
    rho3, nout3 = oracle.deposit_particles(x, y, z, mesh2, qa=np.full(len(x), 1e-13), resize_mesh=True)
    assert nout3 == 0 and abs(mesh2.charge / (1e-13 * len(x)) - 1) < 1e-11
    assert mesh2.min[0] < x.min() and mesh2.max[2] > z.max()


def test_interpolate_at_nodes_and_clamp(oracle):
    n = (6, 5, 7)
    rng = np.random.default_rng(3)
    ef = np.asfortranarray(rng.standard_normal(n + (3,)))
    delta = np.array([0.1, 0.2, 0.3])
    umin = np.array([-1.0, 0.5, 2.0])
    mesh = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), umin, umin + (np.array(n) - 1) * delta, delta, 1.0)
    i, j, k = 2, 3, 4
    pt = umin + np.array([i, j, k]) * delta
    E, _, ncl = oracle.interpolate_field(mesh, ef, [pt[0]], [pt[1]], [pt[2]])
    assert ncl == 0 and np.allclose(E[0], ef[i, j, k], rtol=1e-12)
    E, _, ncl = oracle.interpolate_field(mesh, ef, [umin[0] - 1.0], [pt[1]], [pt[2]])
    assert ncl == 1


def test_pipe_phi_vanishes_on_walls(oracle):
    """KAT: the rectangular-pipe potential is ~0 on the conducting walls."""
    from openspacecharge_b200.bunch import gendist
    a, b = 20e-3, 10e-3
    n = (16, 16, 16)
    x, y, z = gendist(30000, sigma=(2e-3, 1e-3, 1e-3), seed=9, pipe=(a, b), centroid=(3e-3, -1e-3, 0))
    umin = np.array([-a / 2, -b / 2, -6e-3])
    delta = np.array([a / (n[0] - 1), b / (n[1] - 1), 12e-3 / (n[2] - 1)])
    rho, ifail = oracle.depose_rho_scalar(x, y, z, 1e-9 / len(x), (1, 1, 1), n, delta, umin)
    gam = 5e6 / 0.510998910e6
    grn = oracle.getgrnpipe(gam, a, b, delta, umin, (1, 1, 1), n)
    phi, ef, bf = oracle.rectpipe_solver(rho, grn, gam, delta, (1, 1, 1), n)
    pmax = np.abs(phi).max()
    assert np.abs(phi[0]).max() < 1e-6 * pmax and np.abs(phi[-1]).max() < 1e-6 * pmax
    assert np.abs(phi[:, 0]).max() < 1e-6 * pmax and np.abs(phi[:, -1]).max() < 1e-6 * pmax
