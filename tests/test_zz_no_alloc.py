"""The deposit entry point that allocates nothing (osc_deposit_particles_dev_noalloc).

It serves callers that may not allocate device memory when they deposit charge: code
running inside another framework's memory pool, loops that cannot take the device
synchronisation of cudaMalloc/cudaFree, and programs that do not create a library context.
Its FP32 accumulation grid is a fixed array inside the library, shared by every call, so
each call must clear the part it uses: two calls in a row, a smaller mesh after a larger
one and a call without particles must all reproduce the ordinary entry point, including
its count of particles outside the mesh or with non-finite coordinates.
This file is collected last and also runs on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200 import native
from openspacecharge_b200.bunch import gendist

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5  # normwise tolerance of the FP32 paths in this test suite


def _noalloc(mesh_c, x, y, z, q, total_charge, rho):
    err = ctypes.create_string_buffer(256)
    nout = ctypes.c_int64(-1)
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    rc = native.lib().osc_deposit_particles_dev_noalloc(
        ctypes.c_void_p(stream), ctypes.byref(mesh_c), ctypes.c_int64(x.numel()),
        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(z.data_ptr()),
        ctypes.c_void_p(q.data_ptr()) if q is not None else None, ctypes.c_double(total_charge),
        ctypes.c_void_p(rho.data_ptr()), ctypes.byref(nout), err, ctypes.sizeof(err))
    return rc, int(nout.value), err.value.decode()


@pytest.mark.parametrize("use_q", [False, True])
def test_noalloc_deposit_matches_entry_point_twice(ctx, use_q):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    x, y, z = gendist(400_000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=77)
    n = (48, 40, 64)
    delta, umin = osc.get_mesh_quantities(ctx, x, y, z, (1, 1, 1), n, 0)
    umax = umin + (np.array(n) - 1) * delta
    q = np.random.default_rng(3).uniform(0.5, 1.5, len(x)) * 2.5e-15 if use_q else None
    mesh = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umax, delta=delta)
    mc = mesh.to_c()
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    tq = torch.from_numpy(q).to(dev) if use_q else None
    # the ordinary entry point (FP64 atomics, context workspaces)
    ref = torch.zeros(n[::-1], dtype=torch.float64, device=dev)
    tc = ctypes.c_double(1e-9)
    nref = ctypes.c_int64()
    torch.cuda.synchronize()
    ctx.call("osc_deposit_particles_dev", ctypes.c_int64(len(x)), ctypes.c_void_p(tx.data_ptr()),
             ctypes.c_void_p(ty.data_ptr()), ctypes.c_void_p(tz.data_ptr()),
             ctypes.c_void_p(tq.data_ptr()) if use_q else None, None if use_q else ctypes.byref(tc), 0,
             ctypes.byref(mc), ctypes.c_void_p(ref.data_ptr()), ctypes.byref(nref))
    ctx.synchronize()
    r = ref.cpu().numpy()
    for call in range(2):
        out = torch.full(n[::-1], -1.0, dtype=torch.float64, device=dev)
        rc, nout, msg = _noalloc(mesh.to_c(), tx, ty, tz, tq, 1e-9, out)
        torch.cuda.synchronize()
        assert rc == native.OSC_OK, msg
        assert nout == nref.value == 0
        o = out.cpu().numpy()
        err = np.abs(o - r).max() / np.abs(r).max()
        assert err <= FP32_TOL, (call, err)
        assert abs(o.sum() / r.sum() - 1) <= FP32_TOL


def test_noalloc_rejects_meshes_above_its_limit(ctx):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    n = (256, 256, 128)  # 8.4 M nodes > OSC_NOALLOC_MAX_NODES
    mesh = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=np.zeros(3), max=np.ones(3), delta=np.full(3, 1e-3))
    t = torch.zeros(4, dtype=torch.float64, device=dev)
    rho = torch.zeros(1, dtype=torch.float64, device=dev)
    rc, _, msg = _noalloc(mesh.to_c(), t, t, t, None, 1e-9, rho)
    assert rc == native.OSC_E_INVALID
    assert "OSC_NOALLOC_MAX_NODES" in msg


def _ordinary(ctx, mesh_c, tx, ty, tz, total_charge, n):
    """rho and the outside count from the ordinary entry point (context workspaces)."""
    import torch
    ref = torch.zeros(n[::-1], dtype=torch.float64, device=tx.device)
    tc = ctypes.c_double(total_charge)
    nref = ctypes.c_int64()
    torch.cuda.synchronize()
    ctx.call("osc_deposit_particles_dev", ctypes.c_int64(tx.numel()), ctypes.c_void_p(tx.data_ptr()),
             ctypes.c_void_p(ty.data_ptr()), ctypes.c_void_p(tz.data_ptr()), None, ctypes.byref(tc), 0,
             ctypes.byref(mesh_c), ctypes.c_void_p(ref.data_ptr()), ctypes.byref(nref))
    ctx.synchronize()
    return ref.cpu().numpy(), int(nref.value)


def test_noalloc_counts_outside_and_non_finite_like_the_entry_point(ctx):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    x, y, z = gendist(200_000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=78)
    n = (32, 32, 48)
    delta, umin = osc.get_mesh_quantities(ctx, x, y, z, (1, 1, 1), n, 0)
    # shrink the mesh so the tails fall outside, and plant non-finite coordinates
    delta = delta * 0.8
    x[:50] = np.nan
    y[50:60] = np.inf
    z[60:70] = -np.inf
    mesh = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umin + (np.array(n) - 1) * delta, delta=delta)
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    r, nref = _ordinary(ctx, mesh.to_c(), tx, ty, tz, 1e-9, n)
    assert nref > 70
    out = torch.full(n[::-1], -1.0, dtype=torch.float64, device=dev)
    rc, nout, msg = _noalloc(mesh.to_c(), tx, ty, tz, None, 1e-9, out)
    torch.cuda.synchronize()
    assert rc == native.OSC_OK, msg
    assert nout == nref
    o = out.cpu().numpy()
    assert np.abs(o - r).max() / np.abs(r).max() <= FP32_TOL


def test_noalloc_smaller_mesh_after_larger_and_empty_call(ctx):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    x, y, z = gendist(300_000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=79)
    tx, ty, tz = (torch.from_numpy(a).to(dev) for a in (x, y, z))
    for n in [(64, 64, 96), (20, 24, 28)]:  # the second call uses a prefix of what the first filled
        delta, umin = osc.get_mesh_quantities(ctx, x, y, z, (1, 1, 1), n, 0)
        mesh = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, min=umin, max=umin + (np.array(n) - 1) * delta, delta=delta)
        r, nref = _ordinary(ctx, mesh.to_c(), tx, ty, tz, 1e-9, n)
        out = torch.full(n[::-1], -1.0, dtype=torch.float64, device=dev)
        rc, nout, msg = _noalloc(mesh.to_c(), tx, ty, tz, None, 1e-9, out)
        torch.cuda.synchronize()
        assert rc == native.OSC_OK, msg
        assert nout == nref == 0
        o = out.cpu().numpy()
        assert np.abs(o - r).max() / np.abs(r).max() <= FP32_TOL
    # no particles: rho comes back all zero although the array holds the last call's sums
    empty = torch.zeros(0, dtype=torch.float64, device=dev)
    out = torch.full(n[::-1], -1.0, dtype=torch.float64, device=dev)
    rc, nout, msg = _noalloc(mesh.to_c(), empty, empty, empty, None, 1e-9, out)
    torch.cuda.synchronize()
    assert rc == native.OSC_OK, msg
    assert nout == 0
    assert not out.any().item()
