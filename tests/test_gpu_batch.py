"""Batched steps (osc_batch_space_charge_step): many bunches with their own meshes in one call.
Every bunch must get the fields that a single step of that bunch gives (same mesh refit,
same Green spectra, same pipeline; FP32 atomics reorder, hence 2e-6), and one bunch is
checked against the oracle's deposit_particles + space_charge_3d + interpolate_field chain
(code/open_spacecharge_mod.f90:156-489) at the FP32 tolerance."""
import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist
from conftest import field_err

pytestmark = pytest.mark.gpu

GAMMA = 9.784756683727565


def make_bunches(nb, edges, seed, np_range=(2000, 30000)):
    rng = np.random.default_rng(seed)
    meshes, xs, ys, zs, counts, charges = [], [], [], [], [], []
    for b in range(nb):
        n = tuple(int(rng.choice(edges)) for _ in range(3))
        npart = int(np.exp(rng.uniform(np.log(np_range[0]), np.log(np_range[1]))))
        sig = tuple(rng.uniform(0.2e-3, 2e-3, 3))
        x, y, z = gendist(npart, sigma=sig, seed=seed * 1000 + b)
        meshes.append(osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=GAMMA))
        xs.append(x), ys.append(y), zs.append(z)
        counts.append(npart)
        charges.append(rng.uniform(0.1e-9, 2e-9))
    return meshes, np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), counts, charges


@pytest.mark.parametrize("prec", [osc.PREC_FP32, osc.PREC_FP64])
def test_batch_matches_single_steps(ctx, prec):
    meshes, x, y, z, counts, charges = make_bunches(9, (16, 24, 32), seed=5)
    E, nout = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges, precision=prec)
    assert nout == [0] * len(meshes)
    off = 0
    for b, m in enumerate(meshes):
        sl = slice(off, off + counts[b])
        ms = osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA)
        Es, _ = osc.space_charge_step(ctx, ms, x[sl], y[sl], z[sl], total_charge=charges[b], resize_mesh=True,
                                      precision=prec)
        assert np.array_equal(ms.min, m.min) and np.array_equal(ms.delta, m.delta)
        assert ms.charge == m.charge
        mx, _ = field_err(E[sl], Es)
        assert mx <= (2e-6 if prec == osc.PREC_FP32 else 1e-12), (b, m.nhi, mx)
        off += counts[b]


def test_batch_with_charges_and_fixed_meshes(ctx):
    meshes, x, y, z, counts, _ = make_bunches(5, (16, 32), seed=6)
    q = np.random.default_rng(9).uniform(0.5, 1.5, len(x)) * 1e-15
    osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, qa=q, resize_mesh=True)
    # shift every mesh by 3 cells: some particles fall outside and are counted per bunch
    for m in meshes:
        m.min = m.min + 3 * m.delta
        m.max = m.max + 3 * m.delta
    E, nout = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, qa=q, resize_mesh=False)
    off = 0
    for b, m in enumerate(meshes):
        sl = slice(off, off + counts[b])
        ms = osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA, min=m.min.copy(), max=m.max.copy(),
                        delta=m.delta.copy())
        Es, _ = osc.space_charge_step(ctx, ms, x[sl], y[sl], z[sl], qa=q[sl], resize_mesh=False)
        assert abs(ms.charge / m.charge - 1) < 1e-12
        nref = osc.deposit_particles(ctx, x[sl], y[sl], z[sl],
                                     osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, min=m.min.copy(), max=m.max.copy(),
                                                delta=m.delta.copy()), qa=q[sl], resize_mesh=False)
        assert nout[b] == nref > 0
        mx, _ = field_err(E[sl], Es)
        assert mx <= 2e-6, (b, mx)
        off += counts[b]


def test_batch_bunch_matches_oracle(ctx, oracle):
    meshes, x, y, z, counts, charges = make_bunches(4, (24,), seed=7, np_range=(40000, 60000))
    E, _ = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges)
    b = 2
    off = sum(counts[:b])
    sl = slice(off, off + counts[b])
    n = tuple(meshes[b].nhi)
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), (0, 0, 0), (0, 0, 0), (0, 0, 0), GAMMA)
    rho, _ = oracle.deposit_particles(x[sl], y[sl], z[sl], om, total_charge=charges[b], resize_mesh=True)
    ef, _ = oracle.space_charge_3d(om, rho)
    E0, _, _ = oracle.interpolate_field(om, ef, x[sl], y[sl], z[sl])
    assert np.array_equal(meshes[b].delta, np.array(om.delta[:]))
    mx, rm = field_err(E[sl], E0)
    assert mx <= 1e-5, (mx, rm)


def test_batch_dev_matches_host(ctx):
    torch = pytest.importorskip("torch")
    meshes, x, y, z, counts, charges = make_bunches(6, (16, 24, 32, 48), seed=8)
    E1, _ = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges)
    dev = torch.device("cuda", 0)
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    E = torch.empty((len(x), 3), dtype=torch.float64, device=dev)
    meshes2 = [osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA) for m in meshes]
    osc.batch_space_charge_step_dev(ctx, meshes2, tx, ty, tz, counts, E, total_charges=charges)
    ctx.synchronize()
    for m1, m2 in zip(meshes, meshes2):
        assert np.array_equal(m1.delta, m2.delta)
    mx, _ = field_err(E.cpu().numpy(), E1)
    assert mx < 2e-6


@pytest.mark.parametrize("stream", ["own", "legacy_default"])
def test_batch_graph_replay(ctx, stream):
    """A repeated call signature runs the FP32 batched step as one captured CUDA graph (the
    first call runs directly, the second captures): the replays refit the meshes from the
    particles' current positions and give the fields of single steps, and equal the direct
    launches of the same step (OPT_BATCH_GRAPH = 0) to FP32 round-off.  Also with the
    context on CUDA's legacy default stream (torch's default), which cannot be captured
    itself: the capture runs on a private stream and the graph launches on the caller's."""
    torch = pytest.importorskip("torch")
    ctx.set_stream(0 if stream == "legacy_default" else None)
    meshes, x, y, z, counts, charges = make_bunches(9, (16, 24, 32), seed=11)
    dev = torch.device("cuda", 0)
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    E = torch.empty((len(x), 3), dtype=torch.float64, device=dev)

    def run(scale):
        tx.copy_(torch.from_numpy(x * scale).to(dev))
        tz.copy_(torch.from_numpy(z + 1e-3 * scale).to(dev))
        ms = [osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA) for m in meshes]
        osc.batch_space_charge_step_dev(ctx, ms, tx, ty, tz, counts, E, total_charges=charges)
        ctx.synchronize()
        return ms, E.cpu().numpy()

    g0 = ctx.graph_launch_count()
    results = [run(s) for s in (1.0, 1.0, 1.3, 0.7)]
    # 3 replays after the direct first call, 4 when torch handed out the arrays of an
    # earlier call of this test again (the same signature, its graph reused)
    assert ctx.graph_launch_count() - g0 >= 3
    for (ms, Eb), scale in zip(results, (1.0, 1.0, 1.3, 0.7)):
        off = 0
        for b, m in enumerate(ms):
            sl = slice(off, off + counts[b])
            m1 = osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA)
            Es, _ = osc.space_charge_step(ctx, m1, x[sl] * scale, y[sl], z[sl] + 1e-3 * scale,
                                          total_charge=charges[b], resize_mesh=True)
            assert np.array_equal(m1.min, m.min) and np.array_equal(m1.delta, m.delta) and m1.charge == m.charge
            mx, _ = field_err(Eb[sl], Es)
            assert mx <= 2e-6, (scale, b, mx)
            off += counts[b]
    ctx.set_option(osc.OPT_BATCH_GRAPH, 0)
    try:
        g1 = ctx.graph_launch_count()
        _, Ed = run(0.7)
        assert ctx.graph_launch_count() == g1
    finally:
        ctx.set_option(osc.OPT_BATCH_GRAPH, 1)
        ctx.set_stream(None)
    assert field_err(results[-1][1], Ed)[0] <= 2e-6


def test_batch_graph_recaptures_after_tuning_and_new_signature(ctx):
    """A tuning change or a different bunch set is a new signature: the step is planned and
    captured again and still matches single steps."""
    meshes, x, y, z, counts, charges = make_bunches(5, (16, 32), seed=12)
    for _ in range(3):
        E1, _ = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges)
    ctx.set_tuning("zconv_engine:f32:L64", 2)
    try:
        # the host-array call solves its bunches in chunks, one plan (and graph) each: the
        # first call after the change runs them directly, the second replays them
        g0 = ctx.graph_launch_count()
        E2, _ = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges)
        assert ctx.graph_launch_count() == g0
        E2, _ = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges)
        assert ctx.graph_launch_count() > g0
    finally:
        ctx.set_tuning("zconv_engine:f32:L64", 0)
    assert field_err(E1, E2)[0] <= 2e-6
    n2 = counts[:3]
    m2 = [osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA) for m in meshes[:3]]
    k = sum(n2)
    for _ in range(3):
        E3, _ = osc.batch_space_charge_step(ctx, m2, x[:k], y[:k], z[:k], n2, total_charges=charges[:3])
    assert field_err(E3, E1[:k])[0] <= 2e-6


def test_batch_from_host_arrays_any_bunch_order(ctx):
    """The host-array batch copies chunks of bunches in and out while others are solved
    (chunks follow the bunches' offsets, not their order in the call): bunches listed in
    reverse order give the same fields and meshes as the listed order and as the device
    entry point on the same arrays."""
    import ctypes
    from openspacecharge_b200 import native
    from openspacecharge_b200.mesh import _bunches
    meshes, x, y, z, counts, charges = make_bunches(13, (16, 24, 32), seed=14)
    E1, n1 = osc.batch_space_charge_step(ctx, meshes, x, y, z, counts, total_charges=charges)
    m2 = [osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA) for m in meshes]
    arr, total = _bunches(m2, counts, charges)
    rev = (native.OscBunch * len(m2))(*[arr[b] for b in reversed(range(len(m2)))])
    E2 = np.zeros((total, 3))
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    ctx.call("osc_batch_space_charge_step", len(m2), rev, p(x), p(y), p(z), None, 1, int(osc.PREC_FP32), p(E2))
    for i, b in enumerate(reversed(range(len(m2)))):
        m2[b].from_c(rev[i].mesh)
        assert rev[i].n_outside == n1[b]
    for a, b in zip(meshes, m2):
        assert np.array_equal(a.delta, b.delta) and np.array_equal(a.min, b.min) and a.charge == b.charge
    assert field_err(E2, E1)[0] <= 2e-6
    dev = torch_dev = pytest.importorskip("torch")
    d = dev.device("cuda", 0)
    tx, ty, tz = (torch_dev.from_numpy(a).to(d) for a in (x, y, z))
    E3 = torch_dev.empty((total, 3), dtype=torch_dev.float64, device=d)
    m3 = [osc.Mesh3D(nlo=(1, 1, 1), nhi=m.nhi, gamma=GAMMA) for m in meshes]
    osc.batch_space_charge_step_dev(ctx, m3, tx, ty, tz, counts, E3, total_charges=charges)
    ctx.synchronize()
    assert field_err(E3.cpu().numpy(), E1)[0] <= 2e-6
