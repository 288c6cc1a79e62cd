"""Host-side mirror of OpenSpaceCharge's Fortran module API over the C ABI.

Names, argument meaning and error behaviour follow ``open_spacecharge_mod``
(code/open_spacecharge_mod.f90) and the test helpers of ``test_mod`` (code/test_mod.f90);
the work runs in ``libopensc_b200.so`` on the GPU.  Grids are numpy arrays in Fortran
order: ``rho``/``phi`` are ``(nx, ny, nz)``, ``efield``/``bfield`` are ``(nx, ny, nz, 3)``
(component slowest, as ``efield(:,:,:,1:3)``).  Per-particle fields are ``(np, 3)``.

Device-resident variants (``*_dev``) take torch CUDA tensors and do no host copies.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import native
from .native import (PREC_FP32, PREC_FP64, PREC_FP64_PLAIN, Context, OscError, OscMesh3D)

__all__ = [
    "Mesh3D", "Context", "OscError", "PREC_FP32", "PREC_FP64", "PREC_FP64_PLAIN",
    "deposit_particles", "space_charge_3d", "osc_freespace_solver2", "space_charge_freespace",
    "space_charge_cathodeimages", "osc_rectpipe_green", "space_charge_rectpipe",
    "osc_write_rectpipe_grn", "osc_read_rectpipe_grn", "interpolate_field",
    "get_mesh_quantities", "depose_rho_scalar", "space_charge_step", "space_charge_step_dev",
    "sort_particles_dev", "cell_keys",
]


@dataclass
class Mesh3D:
    """mesh3d_struct (code/open_spacecharge_mod.f90:14-27)."""

    nlo: tuple = (1, 1, 1)
    nhi: tuple = (64, 64, 64)
    npad: tuple = (1, 1, 1)
    min: np.ndarray = field(default_factory=lambda: np.zeros(3))
    max: np.ndarray = field(default_factory=lambda: np.zeros(3))
    delta: np.ndarray = field(default_factory=lambda: np.zeros(3))
    gamma: float = 1.0
    charge: float = 0.0
    rho: np.ndarray | None = None
    phi: np.ndarray | None = None
    efield: np.ndarray | None = None
    bfield: np.ndarray | None = None

    @property
    def shape(self) -> tuple:
        return tuple(int(self.nhi[d]) - int(self.nlo[d]) + 1 for d in range(3))

    def to_c(self) -> OscMesh3D:
        m = OscMesh3D()
        m.nlo[:] = [int(v) for v in self.nlo]
        m.nhi[:] = [int(v) for v in self.nhi]
        m.npad[:] = [int(v) for v in self.npad]
        m.min[:] = [float(v) for v in self.min]
        m.max[:] = [float(v) for v in self.max]
        m.delta[:] = [float(v) for v in self.delta]
        m.gamma = float(self.gamma)
        m.charge = float(self.charge)
        return m

    def from_c(self, m: OscMesh3D) -> None:
        self.min = np.array(m.min[:])
        self.max = np.array(m.max[:])
        self.delta = np.array(m.delta[:])
        self.charge = float(m.charge)

    def allocate(self) -> None:
        """(Re)allocate the grids when their bounds changed (code/open_spacecharge_mod.f90:193-219)."""
        n = self.shape
        if self.rho is None or self.rho.shape != n:
            self.rho = np.zeros(n, order="F")
            self.phi = np.zeros(n, order="F")
            self.efield = np.zeros(n + (3,), order="F")
            self.bfield = np.zeros(n + (3,), order="F")


def _p(a) -> ctypes.c_void_p | None:
    if a is None:
        return None
    return ctypes.c_void_p(a.ctypes.data)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="K"))


def _grid(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _dvec(v):
    return None if v is None else (ctypes.c_double * 3)(*[float(x) for x in v])


def _ivec(v):
    return (ctypes.c_int32 * 3)(*[int(x) for x in v])


def _ctx(ctx) -> Context:
    if not isinstance(ctx, Context):
        raise TypeError("ctx must be an openspacecharge_b200.Context")
    return ctx


# ---------------------------------------------------------------------------------------
def deposit_particles(ctx, xa, ya, za, mesh3d: Mesh3D, qa=None, total_charge=None, resize_mesh=True) -> int:
    """deposit_particles (code/open_spacecharge_mod.f90:156).  Fills mesh3d.rho, sets
    mesh3d.charge (and min/max/delta when resize_mesh).  Returns the number of particles
    skipped because their stencil leaves the mesh."""
    ctx = _ctx(ctx)
    x, y, z = _f64(xa), _f64(ya), _f64(za)
    q = None if qa is None else _f64(qa)
    mesh3d.allocate()
    m = mesh3d.to_c()
    tc = None if total_charge is None else ctypes.byref(ctypes.c_double(float(total_charge)))
    nout = ctypes.c_int64(0)
    rho = np.zeros(mesh3d.shape, order="F")
    try:
        ctx.call("osc_deposit_particles", ctypes.c_int64(len(x)), _p(x), _p(y), _p(z), _p(q), tc,
                 int(bool(resize_mesh)), ctypes.byref(m), _p(rho), ctypes.byref(nout))
    except OscError as e:
        if e.code == native.OSC_E_NOCHARGE:
            print("Error, must specify qa or total_charge")  # the reference prints and returns
            return 0
        raise
    mesh3d.from_c(m)
    mesh3d.rho = rho
    return int(nout.value)


def space_charge_3d(ctx, mesh3d: Mesh3D, offset=None, at_cathode=False, calc_bfield=False,
                    precision=PREC_FP32) -> None:
    """space_charge_3d (code/open_spacecharge_mod.f90:431): fills mesh3d.efield (and bfield)."""
    ctx = _ctx(ctx)
    rho = _grid(mesh3d.rho)
    n = rho.shape
    ef = np.zeros(n + (3,), order="F")
    bf = np.zeros(n + (3,), order="F") if calc_bfield else None
    m = mesh3d.to_c()
    ctx.call("osc_space_charge_3d", ctypes.byref(m), _p(rho), _dvec(offset), int(bool(at_cathode)),
             int(bool(calc_bfield)), int(precision), _p(ef), _p(bf))
    mesh3d.efield = ef
    if calc_bfield:
        mesh3d.bfield = bf


def osc_freespace_solver2(ctx, rho, gamma, delta, efield=True, phi=False, offset=None, precision=PREC_FP32):
    """osc_freespace_solver2 (code/open_spacecharge_mod.f90:535) -> (efield|None, phi|None)."""
    ctx = _ctx(ctx)
    rho = _grid(rho)
    n = rho.shape
    ef = np.zeros(n + (3,), order="F") if efield else None
    ph = np.zeros(n, order="F") if phi else None
    ctx.call("osc_freespace_solver2", _ivec(n), _p(rho), ctypes.c_double(gamma), _dvec(delta),
             _dvec(offset), int(precision), _p(ef), _p(ph))
    return ef, ph


def space_charge_freespace(ctx, mesh3d: Mesh3D, direct_field_calc=True, integrated_green_function=True,
                           precision=PREC_FP64_PLAIN) -> None:
    """space_charge_freespace (code/open_spacecharge_mod.f90:60) -> legacy solver."""
    ctx = _ctx(ctx)
    rho = _grid(mesh3d.rho)
    n = rho.shape
    phi = np.zeros(n, order="F")
    ef = np.zeros(n + (3,), order="F")
    bf = np.zeros(n + (3,), order="F")
    m = mesh3d.to_c()
    ctx.call("osc_space_charge_freespace", ctypes.byref(m), _p(rho), int(bool(direct_field_calc)),
             int(bool(integrated_green_function)), int(precision), _p(phi), _p(ef), _p(bf))
    mesh3d.phi, mesh3d.efield, mesh3d.bfield = phi, ef, bf


def space_charge_cathodeimages(ctx, mesh3d: Mesh3D, direct_field_calc=True, integrated_green_function=True,
                               image_method=1, precision=PREC_FP64_PLAIN) -> None:
    """space_charge_cathodeimages (code/open_spacecharge_mod.f90:83).  Method 2 leaves
    mesh3d.rho flipped in z, as the reference does."""
    ctx = _ctx(ctx)
    rho = np.array(_grid(mesh3d.rho), order="F")
    n = rho.shape
    phi = np.zeros(n, order="F")
    ef = np.zeros(n + (3,), order="F")
    bf = np.zeros(n + (3,), order="F")
    m = mesh3d.to_c()
    ctx.call("osc_space_charge_cathodeimages", ctypes.byref(m), _p(rho), int(bool(direct_field_calc)),
             int(bool(integrated_green_function)), int(image_method), int(precision), _p(phi), _p(ef), _p(bf))
    mesh3d.rho, mesh3d.phi, mesh3d.efield, mesh3d.bfield = rho, phi, ef, bf


def osc_rectpipe_green(ctx, mesh3d: Mesh3D, apipe, bpipe, precision=PREC_FP32) -> None:
    """osc_alloc_rectpipe_arrays + osc_getgrnpipe (code/open_spacecharge_core_mod.f90:876, :632)."""
    ctx = _ctx(ctx)
    m = mesh3d.to_c()
    ctx.call("osc_rectpipe_green", ctypes.byref(m), ctypes.c_double(apipe), ctypes.c_double(bpipe),
             int(precision))


def space_charge_rectpipe(ctx, mesh3d: Mesh3D, apipe, bpipe, direct_field_calc=True,
                          integrated_green_function=True, precision=PREC_FP32) -> None:
    """space_charge_rectpipe (code/open_spacecharge_mod.f90:110).  As in the reference, the
    default direct_field_calc=True is rejected (the pipe solves for phi and differences it):
    pass direct_field_calc=False."""
    ctx = _ctx(ctx)
    rho = _grid(mesh3d.rho)
    n = rho.shape
    phi = np.zeros(n, order="F")
    ef = np.zeros(n + (3,), order="F")
    bf = np.zeros(n + (3,), order="F")
    m = mesh3d.to_c()
    ctx.call("osc_space_charge_rectpipe", ctypes.byref(m), _p(rho), ctypes.c_double(apipe),
             ctypes.c_double(bpipe), int(bool(direct_field_calc)), int(bool(integrated_green_function)),
             int(precision), _p(phi), _p(ef), _p(bf))
    mesh3d.phi, mesh3d.efield, mesh3d.bfield = phi, ef, bf


def osc_write_rectpipe_grn(ctx, path, apipe, bpipe, mesh3d: Mesh3D) -> None:
    """osc_write_rectpipe_grn (code/open_spacecharge_core_mod.f90:851)."""
    m = mesh3d.to_c()
    _ctx(ctx).call("osc_write_rectpipe_grn", str(path).encode(), ctypes.c_double(apipe),
                   ctypes.c_double(bpipe), ctypes.byref(m))


def osc_read_rectpipe_grn(ctx, path, mesh3d: Mesh3D):
    """osc_read_rectpipe_grn (code/open_spacecharge_core_mod.f90:825) -> (apipe, bpipe)."""
    m = mesh3d.to_c()
    a = ctypes.c_double()
    b = ctypes.c_double()
    _ctx(ctx).call("osc_read_rectpipe_grn", str(path).encode(), ctypes.byref(m), ctypes.byref(a),
                   ctypes.byref(b))
    return a.value, b.value


def interpolate_field(ctx, x, y, z, mesh3d: Mesh3D, E=True, B=False):
    """Batched interpolate_field (code/open_spacecharge_mod.f90:311).
    Returns (E (np,3)|None, B (np,3)|None, n_clamped)."""
    ctx = _ctx(ctx)
    x, y, z = _f64(x), _f64(y), _f64(z)
    npart = len(x)
    ef = _grid(mesh3d.efield) if E else None
    bf = _grid(mesh3d.bfield) if B else None
    Eo = np.zeros((npart, 3)) if E else None
    Bo = np.zeros((npart, 3)) if B else None
    ncl = ctypes.c_int64(0)
    m = mesh3d.to_c()
    ctx.call("osc_interpolate_field", ctypes.byref(m), _p(ef), _p(bf), ctypes.c_int64(npart), _p(x), _p(y),
             _p(z), _p(Eo), _p(Bo), ctypes.byref(ncl))
    return Eo, Bo, int(ncl.value)


def get_mesh_quantities(ctx, xa, ya, za, nlo, nhi, isetzmin=0):
    """get_mesh_quantities (code/test_mod.f90:288) -> (delta, umin)."""
    x, y, z = _f64(xa), _f64(ya), _f64(za)
    d = (ctypes.c_double * 3)()
    u = (ctypes.c_double * 3)()
    _ctx(ctx).call("osc_get_mesh_quantities", ctypes.c_int64(len(x)), _p(x), _p(y), _p(z), _ivec(nlo),
                   _ivec(nhi), int(isetzmin), d, u)
    return np.array(d[:]), np.array(u[:])


def depose_rho_scalar(ctx, xa, ya, za, chrgpermacro, nlo, nhi, delta, umin, lostflag=None):
    """depose_rho_scalar (code/test_mod.f90:410) -> (rho, ifail)."""
    x, y, z = _f64(xa), _f64(ya), _f64(za)
    lf = None if lostflag is None else _f64(lostflag)
    n = tuple(int(nhi[d]) - int(nlo[d]) + 1 for d in range(3))
    rho = np.zeros(n, order="F")
    ifail = ctypes.c_int64(0)
    _ctx(ctx).call("osc_depose_rho_scalar", ctypes.c_int64(len(x)), _p(x), _p(y), _p(z), _p(lf),
                   ctypes.c_double(chrgpermacro), _ivec(nlo), _ivec(nhi), _dvec(delta), _dvec(umin), _p(rho),
                   ctypes.byref(ifail))
    return rho, int(ifail.value)


def space_charge_step(ctx, mesh3d: Mesh3D, x, y, z, qa=None, total_charge=None, resize_mesh=True,
                      at_cathode=False, precision=PREC_FP32, want_b=False):
    """deposit_particles + space_charge_3d + interpolate_field at every particle, host arrays.
    Returns (E (np,3), B (np,3)|None)."""
    ctx = _ctx(ctx)
    x, y, z = _f64(x), _f64(y), _f64(z)
    q = None if qa is None else _f64(qa)
    npart = len(x)
    E = np.zeros((npart, 3))
    B = np.zeros((npart, 3)) if want_b else None
    m = mesh3d.to_c()
    tc = None if total_charge is None else ctypes.byref(ctypes.c_double(float(total_charge)))
    ctx.call("osc_space_charge_step", ctypes.byref(m), ctypes.c_int64(npart), _p(x), _p(y), _p(z), _p(q), tc,
             int(bool(resize_mesh)), int(bool(at_cathode)), int(precision), _p(E), _p(B))
    mesh3d.from_c(m)
    return E, B


def _tp(t) -> ctypes.c_void_p | None:
    """Device pointer of a torch CUDA tensor (contiguous float64 required)."""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("device entry points need contiguous CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def space_charge_step_dev(ctx, mesh3d: Mesh3D, x, y, z, E, qa=None, total_charge=None, resize_mesh=False,
                          at_cathode=False, precision=PREC_FP32, B=None) -> None:
    """Device-resident step on torch CUDA float64 tensors x, y, z (np) -> E (np,3) in place."""
    ctx = _ctx(ctx)
    m = mesh3d.to_c()
    tc = None if total_charge is None else ctypes.byref(ctypes.c_double(float(total_charge)))
    ctx.call("osc_space_charge_step_dev", ctypes.byref(m), ctypes.c_int64(x.numel()), _tp(x), _tp(y), _tp(z),
             _tp(qa), tc, int(bool(resize_mesh)), int(bool(at_cathode)), int(precision), _tp(E), _tp(B))
    mesh3d.from_c(m)


def _bunches(meshes, counts, total_charges):
    counts = [int(c) for c in counts]
    if len(meshes) != len(counts):
        raise ValueError("one mesh per bunch")
    arr = (native.OscBunch * len(meshes))()
    off = 0
    for b, (m, n) in enumerate(zip(meshes, counts)):
        arr[b].mesh = m.to_c()
        arr[b].offset = off
        arr[b].np = n
        arr[b].total_charge = 0.0 if total_charges is None else float(total_charges[b])
        off += n
    return arr, off


def batch_space_charge_step(ctx, meshes, x, y, z, counts, qa=None, total_charges=None, resize_mesh=True,
                            precision=PREC_FP32):
    """The fused step for many independent bunches in one call (osc_batch_space_charge_step).

    x, y, z (and qa) hold the particles of all bunches back to back, bunch b owning the next
    counts[b] entries; each mesh in `meshes` is refit (resize_mesh) and updated in place.
    Returns (E (total, 3), n_outside per bunch)."""
    ctx = _ctx(ctx)
    if qa is None and total_charges is None:
        raise ValueError("need qa or total_charges")
    arr, total = _bunches(meshes, counts, total_charges)
    x, y, z = _f64(x), _f64(y), _f64(z)
    q = None if qa is None else _f64(qa)
    if len(x) < total:
        raise ValueError("particle arrays shorter than the sum of counts")
    E = np.zeros((total, 3))
    ctx.call("osc_batch_space_charge_step", len(meshes), arr, _p(x), _p(y), _p(z), _p(q),
             int(bool(resize_mesh)), int(precision), _p(E))
    for b, m in enumerate(meshes):
        m.from_c(arr[b].mesh)
    return E, [int(arr[b].n_outside) for b in range(len(meshes))]


def batch_space_charge_step_dev(ctx, meshes, x, y, z, counts, E, qa=None, total_charges=None, resize_mesh=True,
                                precision=PREC_FP32):
    """Device-resident batched step on torch CUDA float64 tensors; E (total, 3) in place."""
    ctx = _ctx(ctx)
    if qa is None and total_charges is None:
        raise ValueError("need qa or total_charges")
    arr, total = _bunches(meshes, counts, total_charges)
    ctx.call("osc_batch_space_charge_step_dev", len(meshes), arr, _tp(x), _tp(y), _tp(z), _tp(qa),
             int(bool(resize_mesh)), int(precision), _tp(E))
    for b, m in enumerate(meshes):
        m.from_c(arr[b].mesh)
    return [int(arr[b].n_outside) for b in range(len(meshes))]


def write_lines(ctx, mesh3d: Mesh3D, xcent, ycent, zcent, directory=None) -> None:
    """write_lines of the reference's test program (code/test_opensc.f90:237-274): x/y/z
    line-outs of E through (xcent, ycent, zcent) into x_lineout.dat, y_lineout.dat and
    z_lineout.dat in `directory` (default: the working directory)."""
    ef = _grid(mesh3d.efield)
    m = mesh3d.to_c()
    d = None if directory is None else str(directory).encode()
    _ctx(ctx).call("osc_write_lines", ctypes.byref(m), _p(ef), float(xcent), float(ycent), float(zcent), d)


def write_plane(ctx, mesh3d: Mesh3D, directory=None) -> None:
    """write_plane of the reference's test program (code/test_opensc.f90:278-295): x, z, Ex,
    Ez, By on the plane y = 0 into x_z_Ex_Ez_By.dat."""
    ef = _grid(mesh3d.efield)
    bf = _grid(mesh3d.bfield)
    m = mesh3d.to_c()
    d = None if directory is None else str(directory).encode()
    _ctx(ctx).call("osc_write_plane", ctypes.byref(m), _p(ef), _p(bf), d)


def format_1pe14_7(v: float) -> str:
    """One value in Fortran's 1PE14.7 edit descriptor (the line-out files' format)."""
    buf = ctypes.create_string_buffer(16)
    rc = native.lib().osc_format_1pe14_7(ctypes.c_double(float(v)), buf)
    if rc:
        raise ValueError("format")
    return buf.value.decode()


def space_charge_step_rectpipe_dev(ctx, mesh3d: Mesh3D, x, y, z, E, apipe, bpipe, qa=None, total_charge=None,
                                   precision=PREC_FP32, B=None) -> None:
    """Fused step in the rectangular pipe on torch CUDA float64 tensors (mesh as given; its
    pipe Green spectra must exist, osc_rectpipe_green): E (np, 3) (and B) in place."""
    ctx = _ctx(ctx)
    m = mesh3d.to_c()
    tc = None if total_charge is None else ctypes.byref(ctypes.c_double(float(total_charge)))
    ctx.call("osc_space_charge_step_rectpipe_dev", ctypes.byref(m), ctypes.c_int64(x.numel()), _tp(x), _tp(y),
             _tp(z), _tp(qa), tc, ctypes.c_double(apipe), ctypes.c_double(bpipe), int(precision), _tp(E), _tp(B))


def cell_keys(mesh3d: Mesh3D, x, y, z) -> np.ndarray:
    """Host restatement of the cell key osc_sort_particles_dev sorts by: the linear index
    i + nx*(j + ny*k) of the lowest corner of the particle's deposit cell
    (deposit_particles' ip = floor((x-xmin)/dx + 1), code/open_spacecharge_mod.f90:259-261),
    or nx*ny*nz when the particle's 2x2x2 stencil leaves the mesh or a coordinate is not
    finite.  Used to check and to prepare cell order."""
    n = mesh3d.shape
    idx = []
    inside = np.ones(len(x), dtype=bool)
    for d, v in enumerate((x, y, z)):
        with np.errstate(invalid="ignore"):
            f = np.floor((np.asarray(v, dtype=np.float64) - mesh3d.min[d]) * (1.0 / mesh3d.delta[d]) + 1.0)
            inside &= (f >= mesh3d.nlo[d]) & (f + 1 <= mesh3d.nhi[d])
        idx.append(np.where(inside, f, mesh3d.nlo[d]).astype(np.int64) - mesh3d.nlo[d])
    key = idx[0] + n[0] * (idx[1] + n[1] * idx[2])
    return np.where(inside, key, n[0] * n[1] * n[2])


def sort_particles_dev(ctx, mesh3d: Mesh3D, x, y, z, q=None, want_perm=True):
    """osc_sort_particles_dev on torch CUDA float64 tensors: returns (xs, ys, zs, qs|None,
    perm|None, n_outside), the particles in cell order and perm[s] = original index."""
    import torch
    ctx = _ctx(ctx)
    xs, ys, zs = torch.empty_like(x), torch.empty_like(y), torch.empty_like(z)
    qs = torch.empty_like(q) if q is not None else None
    perm = torch.empty(x.numel(), dtype=torch.int64, device=x.device) if want_perm else None
    nout = ctypes.c_int64(0)
    m = mesh3d.to_c()
    ctx.call("osc_sort_particles_dev", ctypes.byref(m), ctypes.c_int64(x.numel()), _tp(x), _tp(y), _tp(z), _tp(q),
             _tp(xs), _tp(ys), _tp(zs), _tp(qs), _tp(perm), ctypes.byref(nout))
    return xs, ys, zs, qs, perm, int(nout.value)

