"""CPU checks of the drop-in boundary: the native library loads, exports every symbol the
public header declares, and rejects bad calls with status codes (no GPU needed)."""
import ctypes
import os

import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200 import native


def test_header_declares_entry_points():
    syms = native.header_symbols()
    for name in ("osc_deposit_particles", "osc_space_charge_3d", "osc_interpolate_field",
                 "osc_space_charge_rectpipe", "osc_space_charge_step_dev", "osc_last_error"):
        assert name in syms
    # every declared function has a ctypes signature in the binding
    assert set(syms) <= set(native.SIGNATURES)


def test_library_exports_every_header_symbol():
    L = native.lib()
    missing = [s for s in native.header_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_version_string():
    assert "sm_100a" in native.version()


def test_null_context_is_rejected_not_crashed():
    L = native.lib()
    assert L.osc_deposit_particles(None, 0, None, None, None, None, None, 0, None, None, None) == native.OSC_E_INVALID
    assert L.osc_space_charge_3d(None, None, None, None, 0, 0, 0, None, None) == native.OSC_E_INVALID
    assert L.osc_ctx_destroy(None) == native.OSC_OK
    out = ctypes.c_void_p()
    assert L.osc_ctx_create(0, None) == native.OSC_E_INVALID


def test_mesh_struct_layout_matches_header():
    # int32[9] then double[11]: 36 bytes of ints, padded to 40, then 88 bytes of doubles
    assert ctypes.sizeof(native.OscMesh3D) == 128
    assert native.OscMesh3D.min.offset == 40


def test_mesh3d_roundtrip():
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=(8, 9, 10), gamma=2.0)
    m.min[:] = [1, 2, 3]
    m.delta[:] = [0.1, 0.2, 0.3]
    c = m.to_c()
    assert list(c.nhi) == [8, 9, 10] and c.gamma == 2.0
    m2 = osc.Mesh3D()
    m2.from_c(c)
    assert list(m2.delta) == [0.1, 0.2, 0.3]
    assert m.shape == (8, 9, 10)


def test_bunch_generator_shapes():
    from openspacecharge_b200.bunch import gendist
    import numpy as np
    x, y, z = gendist(5000, sigma=(1e-3, 2e-3, 3e-3), cutoff=4.0, seed=2)
    r2 = (x / 1e-3) ** 2 + (y / 2e-3) ** 2 + (z / 3e-3) ** 2
    assert r2.max() <= 4.0 ** 2 * 1.01 and x[0] == 0 and y[0] == 0
    x2, _, _ = gendist(5000, sigma=(1e-3, 2e-3, 3e-3), seed=2)
    assert np.array_equal(x, x2)
    xp, yp, _ = gendist(5000, sigma=(2e-3, 1e-3, 1e-3), seed=3, pipe=(20e-3, 10e-3), centroid=(3e-3, -1e-3, 0))
    assert (((xp - 3e-3) / 10e-3) ** 2 + ((yp + 1e-3) / 5e-3) ** 2).max() <= 0.81 * 1.05


def _noalloc_status(nlo, nhi, total_charge=1e-9):
    """Status of the no-allocation deposit for a mesh whose checks fail before any CUDA
    call; the particle and rho pointers are dummies that are never dereferenced."""
    m = native.OscMesh3D()
    for d in range(3):
        m.nlo[d], m.nhi[d], m.delta[d] = nlo[d], nhi[d], 1e-3
    dummy = ctypes.c_void_p(16)
    err = ctypes.create_string_buffer(256)
    rc = native.lib().osc_deposit_particles_dev_noalloc(None, ctypes.byref(m), 4, dummy, dummy, dummy, None,
                                                        ctypes.c_double(total_charge), dummy, None, err,
                                                        ctypes.sizeof(err))
    return rc, err.value.decode()


@pytest.mark.parametrize("nhi", [(2 ** 21, 2 ** 21, 2 ** 22),      # product 2^64 wraps to 0 in int64
                                 (2 ** 31 - 1, 2 ** 31 - 1, 8),    # each factor overflows int32 products
                                 (256, 256, 128)])                 # plainly above the limit
def test_noalloc_rejects_oversized_and_wrapping_meshes_before_any_launch(nhi):
    rc, msg = _noalloc_status((1, 1, 1), nhi)
    assert rc == native.OSC_E_INVALID
    assert "OSC_NOALLOC_MAX_NODES" in msg


def test_noalloc_rejects_a_negative_extent_and_a_non_finite_charge():
    rc, msg = _noalloc_status((1, 1, 1), (-(2 ** 31) + 1, 8, 8))
    assert rc == native.OSC_E_INVALID and "fewer than 2 nodes" in msg
    rc, msg = _noalloc_status((1, 1, 1), (8, 8, 8), total_charge=float("nan"))
    assert rc == native.OSC_E_INVALID and "total_charge" in msg


def test_noalloc_without_charges_is_the_missing_charge_error():
    """d_q NULL and total_charge 0: the reference's "must specify qa or total_charge"."""
    rc, msg = _noalloc_status((1, 1, 1), (8, 8, 8), total_charge=0.0)
    assert rc == native.OSC_E_NOCHARGE and "total_charge" in msg
