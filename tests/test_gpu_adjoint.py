"""Adjoint of the fused step (osc_space_charge_step_vjp_dev) and its torch.autograd wrapper.

The loss is L = sum_m q_m |E(x_m)|^2 on a fixed mesh.  Within one cell the deposit and the
gather are trilinear in a particle's position, so central differences of L are exact up
to round-off; components whose +-h step would cross a cell face are skipped.  The FP64
gradients match central differences of the FP64 oracle's forward chain (deposit_particles,
space_charge_3d, interpolate_field: the reference algorithm, with no GPU code) and of the
GPU's own FP64 forward to 1e-6 (relative to the largest gradient); the FP32 path matches
FP64 to 1e-4, also at the differentiable-step configuration (128^3, 4e6 particles)."""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N = (32, 32, 32)
GAMMA = 9.784756683727565


@pytest.fixture(scope="module")
def det():
    c = osc.Context(0)
    c.set_option(osc.OPT_DEPOSIT_MODE, osc.DEPOSIT_DETERMINISTIC)
    yield c
    c.close()


# z length 2*32 = 64 has no warp z engine: the FP32 adjoint potential takes three one-
# component solves; 2*48 = 96 has one: the three are summed in one solve
N_SUMMED = (32, 32, 48)


def setup(ctx, npart=20000, seed=51, n=N):
    x, y, z = gendist(npart, sigma=(1e-3, 1e-3, 1e-3), seed=seed)
    q = np.random.default_rng(seed).uniform(0.5, 1.5, npart) * 1e-15
    delta, umin = osc.get_mesh_quantities(ctx, x, y, z, (1, 1, 1), n, 0)
    umax = umin + (np.array(n) - 1) * delta
    mesh = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umax, delta=delta, gamma=GAMMA)
    return x, y, z, q, mesh


def loss(ctx, mesh, x, y, z, q, prec):
    m = osc.Mesh3D(nlo=mesh.nlo, nhi=mesh.nhi, min=mesh.min.copy(), max=mesh.max.copy(), delta=mesh.delta.copy(),
                   gamma=mesh.gamma)
    E, _ = osc.space_charge_step(ctx, m, x, y, z, qa=q, resize_mesh=False, precision=prec)
    return float((q[:, None] * E * E).sum()), E


def vjp(ctx, mesh, x, y, z, q, gE, prec):
    import ctypes
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (x, y, z, q, gE)]
    g = [torch.empty_like(t[0]) for _ in range(4)]
    m = mesh.to_c()
    ctx.call("osc_space_charge_step_vjp_dev", ctypes.byref(m), ctypes.c_int64(len(x)),
             *[ctypes.c_void_p(a.data_ptr()) for a in t[:4]], ctypes.c_double(0.0), int(prec),
             ctypes.c_void_p(t[4].data_ptr()), *[ctypes.c_void_p(a.data_ptr()) for a in g])
    ctx.synchronize()
    return [a.cpu().numpy() for a in g]


def test_vjp_matches_central_differences(det):
    x, y, z, q, mesh = setup(det)
    L0, E = loss(det, mesh, x, y, z, q, osc.PREC_FP64)
    gx, gy, gz, gq = vjp(det, mesh, x, y, z, q, 2 * q[:, None] * E, osc.PREC_FP64)
    # the VJP's own part of dL/dq excludes the explicit q in the loss: add |E|^2
    grads = [gx, gy, gz]
    scale = max(np.abs(g).max() for g in grads)
    rng = np.random.default_rng(7)
    picks = rng.choice(len(x), 64, replace=False)
    pos = [x, y, z]
    checked = 0
    for m in picks:
        for d in range(3):
            h = 1e-4 * 1e-3
            u = (pos[d][m] - mesh.min[d]) / mesh.delta[d]
            if min(u - np.floor(u), np.ceil(u) - u) * mesh.delta[d] < 3 * h:
                continue  # the step would cross a cell face
            p = [a.copy() for a in pos]
            p[d][m] += h
            Lp, _ = loss(det, mesh, *p, q, osc.PREC_FP64)
            p[d][m] -= 2 * h
            Lm, _ = loss(det, mesh, *p, q, osc.PREC_FP64)
            fd = (Lp - Lm) / (2 * h)
            assert abs(fd - grads[d][m]) <= 1e-6 * scale, (m, d, fd, grads[d][m])
            checked += 1
    assert checked >= 150
    # charges: L is quadratic in q_m, so central differences are exact too
    for m in picks[:16]:
        hq = 1e-3 * q[m]
        qp = q.copy()
        qp[m] += hq
        Lp, _ = loss(det, mesh, x, y, z, qp, osc.PREC_FP64)
        qp[m] -= 2 * hq
        Lm, _ = loss(det, mesh, x, y, z, qp, osc.PREC_FP64)
        fd = (Lp - Lm) / (2 * hq)
        full = (E[m] ** 2).sum() + gq[m]
        assert abs(fd - full) <= 1e-6 * abs(full), (m, fd, full)


def oracle_loss(oracle, mesh, x, y, z, q):
    om = oracle.make_mesh((1, 1, 1), mesh.nhi, (1, 1, 1), mesh.min, mesh.max, mesh.delta, mesh.gamma)
    rho, _ = oracle.deposit_particles(x, y, z, om, qa=q, resize_mesh=False)
    ef, _ = oracle.space_charge_3d(om, rho)
    E, _, _ = oracle.interpolate_field(om, ef, x, y, z)
    return float((q[:, None] * E * E).sum()), E


def fd_check(lossf, mesh, x, y, z, q, grads, gq, E, picks, tol, h=1e-7, hq_rel=1e-3):
    """Central differences of lossf on the picked particles (position steps h, charge steps
    hq_rel * q) against the gradients."""
    scale = max(np.abs(g).max() for g in grads)
    pos = [x, y, z]
    checked = 0
    for m in picks:
        for d in range(3):
            u = (pos[d][m] - mesh.min[d]) / mesh.delta[d]
            if min(u - np.floor(u), np.ceil(u) - u) * mesh.delta[d] < 3 * h:
                continue  # the step would cross a cell face
            p = [a.copy() for a in pos]
            p[d][m] += h
            Lp = lossf(*p, q)
            p[d][m] -= 2 * h
            Lm = lossf(*p, q)
            fd = (Lp - Lm) / (2 * h)
            assert abs(fd - grads[d][m]) <= tol * scale, (m, d, fd, grads[d][m])
            checked += 1
    for m in picks[:16]:
        hq = hq_rel * q[m]
        qp = q.copy()
        qp[m] += hq
        Lp = lossf(x, y, z, qp)
        qp[m] -= 2 * hq
        Lm = lossf(x, y, z, qp)
        fd = (Lp - Lm) / (2 * hq)
        full = (E[m] ** 2).sum() + gq[m]
        assert abs(fd - full) <= tol * abs(full), (m, fd, full)
    return checked


@pytest.mark.parametrize("n", [(16, 16, 16), (16, 16, 24)])
def test_vjp_matches_oracle_central_differences(ctx, oracle, n):
    """FP64 reference gradients: central differences of the oracle's forward chain."""
    x, y, z, q, mesh = setup(ctx, npart=20000, seed=56, n=n)
    L0, E_orc = oracle_loss(oracle, mesh, x, y, z, q)
    _, E = loss(ctx, mesh, x, y, z, q, osc.PREC_FP64)
    assert np.abs(E - E_orc).max() <= 1e-10 * np.abs(E_orc).max()
    gE = 2 * q[:, None] * E_orc
    g64 = vjp(ctx, mesh, x, y, z, q, gE, osc.PREC_FP64)
    picks = np.random.default_rng(8).choice(len(x), 64, replace=False)
    # the oracle's full complex doubled-grid transforms leave ~1e-13 of L as round-off that
    # changes with the input, so its differences take steps of 1e-6 m (0.2% of a cell) and 1% of q
    checked = fd_check(lambda a, b, c, qq: oracle_loss(oracle, mesh, a, b, c, qq)[0], mesh, x, y, z, q,
                       g64[:3], g64[3], E_orc, picks, 1e-6, h=1e-6, hq_rel=1e-2)
    assert checked >= 150
    g32 = vjp(ctx, mesh, x, y, z, q, gE, osc.PREC_FP32)
    for a, b in zip(g32, g64):
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()


def test_differentiable_step_configuration(det, oracle):
    """128^3 grid, 4e6 particles (sigma 1 mm, 1 nC): the forward E against the oracle, FP32
    gradients against FP64 at every particle, FP64 gradients against central differences of
    the GPU's FP64 forward on 64 particles.  With 4e6 particles one particle's share of L is
    ~1e-10 of it, so the differences take larger steps (1e-6 m, 1% of q) and a 1e-4
    tolerance, and the deposits are fixed point (no atomic-order noise in L)."""
    ctx = det
    npart = 4_000_000
    x, y, z = gendist(npart, sigma=(1e-3, 1e-3, 1e-3), seed=1)
    q = np.full(npart, 1e-9 / npart)
    n = (128, 128, 128)
    delta, umin = osc.get_mesh_quantities(ctx, x, y, z, (1, 1, 1), n, 0)
    mesh = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umin + (np.array(n) - 1) * delta, delta=delta,
                      gamma=GAMMA)
    _, E_orc = oracle_loss(oracle, mesh, x, y, z, q)
    _, E = loss(ctx, mesh, x, y, z, q, osc.PREC_FP64)
    assert np.abs(E - E_orc).max() <= 1e-10 * np.abs(E_orc).max()
    _, E32 = loss(ctx, mesh, x, y, z, q, osc.PREC_FP32)
    assert np.abs(E32 - E_orc).max() <= 1e-5 * np.abs(E_orc).max()
    gE = 2 * q[:, None] * E
    g64 = vjp(ctx, mesh, x, y, z, q, gE, osc.PREC_FP64)
    g32 = vjp(ctx, mesh, x, y, z, q, 2 * q[:, None] * E32, osc.PREC_FP32)
    for a, b in zip(g32, g64):
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()
    picks = np.random.default_rng(9).choice(npart, 64, replace=False)
    checked = fd_check(lambda a, b, c, qq: loss(ctx, mesh, a, b, c, qq, osc.PREC_FP64)[0], mesh, x, y, z, q,
                       g64[:3], g64[3], E, picks, 1e-4, h=1e-6, hq_rel=1e-2)
    assert checked >= 120


@pytest.mark.parametrize("n", [N, N_SUMMED])
def test_fp32_vjp_matches_fp64(ctx, n):
    x, y, z, q, mesh = setup(ctx, npart=100000, seed=52, n=n)
    _, E = loss(ctx, mesh, x, y, z, q, osc.PREC_FP64)
    gE = 2 * q[:, None] * E
    g64 = vjp(ctx, mesh, x, y, z, q, gE, osc.PREC_FP64)
    g32 = vjp(ctx, mesh, x, y, z, q, gE, osc.PREC_FP32)
    for a, b in zip(g32, g64):
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()


@pytest.mark.parametrize("n", [N, N_SUMMED])
def test_fp32_vjp_outside_particles_and_total_charge(ctx, n):
    """FP32 path (quad deposits, x-pair gather) against FP64 with the mesh shifted by three
    cells, so some particles lie outside it (clamped gather cell, no adjoint-potential term),
    and with the charge given as a total (q null)."""
    import ctypes
    x, y, z, q, mesh = setup(ctx, npart=60000, seed=54, n=n)
    mesh.min = mesh.min + 3 * mesh.delta
    mesh.max = mesh.max + 3 * mesh.delta
    rng = np.random.default_rng(7)
    gE = rng.normal(size=(len(x), 3)) * 1e-3
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (x, y, z, gE)]
    m = mesh.to_c()
    out = {}
    for prec in (osc.PREC_FP64, osc.PREC_FP32):
        g = [torch.empty_like(t[0]) for _ in range(4)]
        ctx.call("osc_space_charge_step_vjp_dev", ctypes.byref(m), ctypes.c_int64(len(x)),
                 *[ctypes.c_void_p(a.data_ptr()) for a in t[:3]], None, ctypes.c_double(1e-9), int(prec),
                 ctypes.c_void_p(t[3].data_ptr()), *[ctypes.c_void_p(a.data_ptr()) for a in g])
        ctx.synchronize()
        out[prec] = [a.cpu().numpy() for a in g]
    lam64 = out[osc.PREC_FP64][3]
    assert (lam64 == 0).sum() > 0 and (lam64 != 0).sum() > 0  # some particles outside, some inside
    for a, b in zip(out[osc.PREC_FP32], out[osc.PREC_FP64]):
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()
    assert np.array_equal(out[osc.PREC_FP32][3] == 0, lam64 == 0)


def test_autograd_function(ctx):
    from openspacecharge_b200.autograd import space_charge_field
    x, y, z, q, mesh = setup(ctx, npart=50000, seed=53)
    dev = torch.device("cuda", 0)
    tx, ty, tz, tq = (torch.from_numpy(a).to(dev).requires_grad_() for a in (x, y, z, q))
    E = space_charge_field(tx, ty, tz, tq, mesh, ctx, precision=osc.PREC_FP64)
    L = (tq[:, None] * E * E).sum()
    L.backward()
    Ed = E.detach().cpu().numpy()
    gx, gy, gz, gq = vjp(ctx, mesh, x, y, z, q, 2 * q[:, None] * Ed, osc.PREC_FP64)
    for t, ref in ((tx, gx), (ty, gy), (tz, gz)):
        assert np.allclose(t.grad.cpu().numpy(), ref, rtol=0, atol=1e-9 * np.abs(ref).max())
    assert np.allclose(tq.grad.cpu().numpy(), (Ed ** 2).sum(1) + gq, rtol=1e-9, atol=0)


@pytest.mark.parametrize("n", [N, N_SUMMED])
def test_fp32_vjp_reuses_the_forward_grid(ctx, n):
    """OPT_VJP_REUSE_FORWARD: the FP32 VJP right after the FP32 step on the same arrays takes
    E on the grid from that step (fewer kernels) and gives the gradients of the recomputing
    VJP to FP32 round-off; a step in between (other particles) makes it recompute."""
    import ctypes
    x, y, z, q, mesh = setup(ctx, npart=60000, seed=55, n=n)
    dev = torch.device("cuda", 0)
    tx, ty, tz, tq = (torch.from_numpy(a).to(dev) for a in (x, y, z, q))
    E = torch.empty((len(x), 3), dtype=torch.float64, device=dev)
    m = mesh.to_c()

    def step(ax=tx):
        ms = osc.Mesh3D(nlo=mesh.nlo, nhi=mesh.nhi, min=mesh.min.copy(), max=mesh.max.copy(),
                        delta=mesh.delta.copy(), gamma=mesh.gamma)
        osc.space_charge_step_dev(ctx, ms, ax, ty, tz, E, qa=tq, precision=osc.PREC_FP32)

    def vjp32():
        gE = 2 * tq[:, None] * E
        g = [torch.empty_like(tx) for _ in range(4)]
        l0 = ctx.launch_count()
        ctx.call("osc_space_charge_step_vjp_dev", ctypes.byref(m), ctypes.c_int64(len(x)),
                 *[ctypes.c_void_p(a.data_ptr()) for a in (tx, ty, tz, tq)], ctypes.c_double(0.0),
                 int(osc.PREC_FP32), ctypes.c_void_p(gE.data_ptr()), *[ctypes.c_void_p(a.data_ptr()) for a in g])
        ctx.synchronize()
        return [a.cpu().numpy() for a in g], ctx.launch_count() - l0

    step()
    ref, n_ref = vjp32()  # the option is off: recomputed
    ctx.set_option(osc.OPT_VJP_REUSE_FORWARD, 1)
    try:
        step()
        got, n_got = vjp32()
        assert n_got < n_ref
        for a, b in zip(got, ref):
            assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()
        # the last step ran on another x array: its grid is not the one of (tx, ty, tz)
        step(tx + 0.25 * float(mesh.delta[0]))
        _, n_other = vjp32()
        assert n_other == n_ref
    finally:
        ctx.set_option(osc.OPT_VJP_REUSE_FORWARD, 0)
