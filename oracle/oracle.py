"""ctypes wrapper of the FP64 CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``opensc_oracle.cpp``) restates OpenSpaceCharge's Fortran space-charge path
(RobertRyne/OpenSpaceCharge ``code/*.f90``) in C++.  It is the checker for the CUDA
product and the timed CPU baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU legs of ``bench.py`` may import this module.

Parity status: get_mesh_quantities is pinned bit-exactly against values the reference
printed in its own run (examples/benchmark.ipynb); the field solve is pinned only by the
notebook's cathode cross-method differences and analytic known-answer tests ("parity
unpinned" by reference golden data, which the reference does not ship).

Array conventions follow the reference: 3D grids are numpy arrays in Fortran order
``(nx, ny, nz)``; fields are ``(nx, ny, nz, 3)`` Fortran order (component slowest);
particle fields are ``(np, 3)``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libopensc_oracle.so")
_lib = None
_lock = threading.Lock()

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_i64 = ctypes.c_int64


class OrcMesh(ctypes.Structure):
    """Scalar members of mesh3d_struct (code/open_spacecharge_mod.f90:14-27)."""

    _fields_ = [
        ("nlo", ctypes.c_int * 3),
        ("nhi", ctypes.c_int * 3),
        ("npad", ctypes.c_int * 3),
        ("min", ctypes.c_double * 3),
        ("max", ctypes.c_double * 3),
        ("delta", ctypes.c_double * 3),
        ("gamma", ctypes.c_double),
        ("charge", ctypes.c_double),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    src = os.path.join(_HERE, "opensc_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        env = dict(os.environ)
        env.pop("CXX", None)
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "all"], check=True, env=env)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(_LIB_PATH)
            L.orc_lafun2.restype = ctypes.c_double
            L.orc_xlafun2.restype = ctypes.c_double
            L.orc_igf_point.restype = ctypes.c_double
            L.orc_rfun.restype = ctypes.c_double
            L.orc_interpolate_field.restype = ctypes.c_int64
            L.orc_depose_rho_scalar.restype = ctypes.c_int64
            for name in ("orc_lafun2", "orc_xlafun2"):
                getattr(L, name).argtypes = [ctypes.c_double] * 3
            L.orc_igf_point.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 7
            L.orc_rfun.argtypes = [ctypes.c_double] * 7 + [ctypes.c_int, ctypes.c_int]
            _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _ivec(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


def _dvec(v):
    return None if v is None else (ctypes.c_double * 3)(*[float(x) for x in v])


def _f64(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def make_mesh(nlo=(1, 1, 1), nhi=(64, 64, 64), npad=(1, 1, 1), mn=(0, 0, 0), mx=(0, 0, 0),
              delta=(0, 0, 0), gamma=1.0, charge=0.0) -> OrcMesh:
    m = OrcMesh()
    m.nlo[:] = list(nlo)
    m.nhi[:] = list(nhi)
    m.npad[:] = list(npad)
    m.min[:] = list(mn)
    m.max[:] = list(mx)
    m.delta[:] = list(delta)
    m.gamma = gamma
    m.charge = charge
    return m


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ---------------------------------------------------------------------------------------
def ccfft3d(a: np.ndarray, idir) -> np.ndarray:
    """Unnormalised 3D DFT with per-axis sign (code/fft_interface_mod.f90:96)."""
    b = np.asfortranarray(np.array(a, dtype=np.complex128))
    n1, n2, n3 = b.shape
    rc = lib().orc_ccfft3d(b.ctypes.data_as(_dp), _ivec(idir), n1, n2, n3)
    if rc:
        raise ValueError("unsupported FFT length")
    return b


def lafun2(x, y, z):
    return lib().orc_lafun2(x, y, z)


def xlafun2(x, y, z):
    return lib().orc_xlafun2(x, y, z)


def get_cgrn_freespace(shape, delta, gamma, icomp, offset=None) -> np.ndarray:
    """osc_get_cgrn_freespace (code/open_spacecharge_mod.f90:633) -> complex (2nx,2ny,2nz)."""
    c = np.zeros(shape, dtype=np.complex128, order="F")
    lib().orc_get_cgrn_freespace(c.ctypes.data_as(_dp), shape[0], shape[1], shape[2],
                                 _dvec(delta), ctypes.c_double(gamma), int(icomp), _dvec(offset))
    return c


def freespace_solver2(rho, gamma, delta, offset=None, want_phi=False, want_e=True):
    """osc_freespace_solver2 (code/open_spacecharge_mod.f90:535)."""
    rho = _f64(rho)
    n = rho.shape
    ef = np.zeros(n + (3,), order="F") if want_e else None
    ph = np.zeros(n, order="F") if want_phi else None
    rc = lib().orc_freespace_solver2(_p(rho), _ivec(n), ctypes.c_double(gamma), _dvec(delta),
                                     _dvec(offset), _p(ef), _p(ph))
    if rc:
        raise ValueError(f"orc_freespace_solver2 rc={rc}")
    return ef, ph


def space_charge_3d(mesh: OrcMesh, rho, offset=None, at_cathode=False, calc_bfield=False):
    """space_charge_3d (code/open_spacecharge_mod.f90:431) -> (efield, bfield|None)."""
    rho = _f64(rho)
    n = rho.shape
    ef = np.zeros(n + (3,), order="F")
    bf = np.zeros(n + (3,), order="F") if calc_bfield else None
    rc = lib().orc_space_charge_3d(ctypes.byref(mesh), _p(rho), _dvec(offset), int(bool(at_cathode)),
                                   int(bool(calc_bfield)), _p(ef), _p(bf))
    if rc:
        raise ValueError(f"orc_space_charge_3d rc={rc}")
    return ef, bf


def deposit_particles(x, y, z, mesh: OrcMesh, qa=None, total_charge=None, resize_mesh=True):
    """deposit_particles (code/open_spacecharge_mod.f90:156) -> (rho, n_outside)."""
    x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
    qa = None if qa is None else np.ascontiguousarray(qa, dtype=np.float64)
    n = tuple(mesh.nhi[d] - mesh.nlo[d] + 1 for d in range(3))
    rho = np.zeros(n, order="F")
    nout = ctypes.c_int64(0)
    tc = None if total_charge is None else ctypes.byref(ctypes.c_double(total_charge))
    rc = lib().orc_deposit_particles(_i64(len(x)), _p(x), _p(y), _p(z), _p(qa), tc,
                                     int(bool(resize_mesh)), ctypes.byref(mesh), _p(rho),
                                     ctypes.byref(nout))
    if rc:
        raise ValueError(f"orc_deposit_particles rc={rc}")
    return rho, int(nout.value)


def interpolate_field(mesh: OrcMesh, efield, x, y, z, bfield=None):
    """Batched interpolate_field (code/open_spacecharge_mod.f90:311) -> (E, B, n_clamped)."""
    x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
    ef = _f64(efield) if efield is not None else None
    bf = _f64(bfield) if bfield is not None else None
    E = np.zeros((len(x), 3)) if ef is not None else None
    B = np.zeros((len(x), 3)) if bf is not None else None
    ncl = lib().orc_interpolate_field(ctypes.byref(mesh), _p(ef), _p(bf), _i64(len(x)), _p(x),
                                      _p(y), _p(z), _p(E), _p(B))
    return E, B, int(ncl)


def get_mesh_quantities(x, y, z, nlo, nhi, isetzmin=0):
    """get_mesh_quantities (code/test_mod.f90:288) -> (delta, umin)."""
    x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
    d = (ctypes.c_double * 3)()
    u = (ctypes.c_double * 3)()
    lib().orc_get_mesh_quantities(_i64(len(x)), _p(x), _p(y), _p(z), _ivec(nlo), _ivec(nhi),
                                  int(isetzmin), d, u)
    return np.array(d[:]), np.array(u[:])


def depose_rho_scalar(x, y, z, chrgpermacro, nlo, nhi, delta, umin, lostflag=None, nlogbl=None):
    """depose_rho_scalar (code/test_mod.f90:410) -> (rho, ifail)."""
    x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
    lf = None if lostflag is None else np.ascontiguousarray(lostflag, dtype=np.float64)
    n = tuple(nhi[d] - nlo[d] + 1 for d in range(3))
    rho = np.zeros(n, order="F")
    ifail = lib().orc_depose_rho_scalar(_i64(len(x)), _p(x), _p(y), _p(z), _p(lf), _p(rho),
                                        ctypes.c_double(chrgpermacro), _ivec(nlo), _ivec(nhi),
                                        _dvec(delta), _dvec(umin), _ivec(nlogbl or nlo))
    return rho, int(ifail)


def freespace_solver(rho, gam0, delta, nlo, nhi, npad=(1, 1, 1), direct=True, igf=True):
    """Legacy osc_freespace_solver (code/open_spacecharge_core_mod.f90:30)."""
    rho = _f64(rho)
    n = rho.shape
    phi = np.zeros(n, order="F")
    ef = np.zeros(n + (3,), order="F")
    bf = np.zeros(n + (3,), order="F")
    rc = lib().orc_freespace_solver(_p(rho), ctypes.c_double(gam0), _dvec(delta), _p(phi), _p(ef),
                                    _p(bf), _ivec(nlo), _ivec(nhi), _ivec(npad), int(bool(direct)),
                                    int(bool(igf)))
    if rc:
        raise ValueError(f"orc_freespace_solver rc={rc}")
    return phi, ef, bf


def cathodeimages_solver(rho, gam0, umin, delta, nlo, nhi, npad=(1, 1, 1), direct=True, igf=True,
                         imethod=1):
    """Legacy osc_cathodeimages_solver (core:905).  Returns (phi, efield, bfield, rho_after)."""
    rho = np.array(_f64(rho), order="F")
    n = rho.shape
    phi = np.zeros(n, order="F")
    ef = np.zeros(n + (3,), order="F")
    bf = np.zeros(n + (3,), order="F")
    rc = lib().orc_cathodeimages_solver(_p(rho), ctypes.c_double(gam0), _dvec(umin), _dvec(delta),
                                        _p(phi), _p(ef), _p(bf), _ivec(nlo), _ivec(nhi), _ivec(npad),
                                        int(bool(direct)), int(bool(igf)), int(imethod))
    if rc:
        raise ValueError(f"orc_cathodeimages_solver rc={rc}")
    return phi, ef, bf, rho


def igf_point(icomp, igfflag, u, v, w, gam, dx, dy, dz):
    return lib().orc_igf_point(icomp, igfflag, u, v, w, gam, dx, dy, dz)


def rfun(u, v, w, gam, a, b, hz, i, j):
    return lib().orc_rfun(u, v, w, gam, a, b, hz, i, j)


def getgrnpipe(gam, a, b, delta, umin, nlo, nhi, npad=(1, 1, 1)):
    """osc_alloc_rectpipe_arrays + osc_getgrnpipe (core:876, :632) -> 4 complex arrays."""
    per = tuple(2 * (nhi[d] - nlo[d]) + 1 + npad[d] for d in range(3))
    g = [np.zeros(per, dtype=np.complex128, order="F") for _ in range(4)]
    rc = lib().orc_getgrnpipe(ctypes.c_double(gam), ctypes.c_double(a), ctypes.c_double(b),
                              _dvec(delta), _dvec(umin), _ivec(nlo), _ivec(nhi), _ivec(npad),
                              *[x.ctypes.data_as(_dp) for x in g])
    if rc:
        raise ValueError(f"orc_getgrnpipe rc={rc}")
    return g


def rectpipe_solver(rho, grn, gam0, delta, nlo, nhi, npad=(1, 1, 1), direct=False):
    """osc_rectpipe_solver (core:536) -> (phi, efield, bfield)."""
    rho = _f64(rho)
    n = rho.shape
    phi = np.zeros(n, order="F")
    ef = np.zeros(n + (3,), order="F")
    bf = np.zeros(n + (3,), order="F")
    rc = lib().orc_rectpipe_solver(_p(rho), *[x.ctypes.data_as(_dp) for x in grn],
                                   ctypes.c_double(gam0), _dvec(delta), _p(phi), _p(ef), _p(bf),
                                   _ivec(nlo), _ivec(nhi), _ivec(npad), int(bool(direct)))
    if rc:
        raise ValueError(f"orc_rectpipe_solver rc={rc}")
    return phi, ef, bf
