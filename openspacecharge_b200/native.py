"""ctypes binding of ``libopensc_b200.so`` (the C ABI in ``include/opensc_gpu.h``).

This module only loads the library and declares signatures; :mod:`openspacecharge_b200.mesh`
holds the Fortran-shaped API.  There is no CPU fallback: loading fails loudly when the
library is missing, and any non-zero status raises :class:`OscError`.
"""
from __future__ import annotations

import ctypes
import os
import re
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libopensc_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "opensc_gpu.h")

OSC_OK = 0
OSC_E_INVALID = 1
OSC_E_BOUNDS = 2
OSC_E_FFT_SIZE = 3
OSC_E_ALLOC = 4
OSC_E_CUDA = 5
OSC_E_TIMEOUT = 6
OSC_E_NAN = 7
OSC_E_NOCHARGE = 8
OSC_E_UNSUPPORTED = 9
OSC_E_STATE = 10

PREC_FP32 = 0
PREC_FP64 = 1
PREC_FP64_PLAIN = 2

DEPOSIT_ATOMIC = 0
DEPOSIT_DETERMINISTIC = 1
DEPOSIT_SORTED_SEGMENT = 2

ORDER_ANY = 0
ORDER_CELL_SORTED = 1
ORDER_SORT = 2

OPT_PRECISION = 1
OPT_DEPOSIT_MODE = 2
OPT_STRICT_BOUNDS = 3
OPT_GREEN_CACHE_MB = 4
OPT_PROFILE = 5
OPT_CHECK_FINITE = 6
OPT_TEST_WAIT_TIMEOUT = 7
OPT_PARTICLE_ORDER = 8
OPT_BATCH_GRAPH = 9
OPT_VJP_REUSE_FORWARD = 10

_ERRNAMES = {v: k for k, v in globals().items() if k.startswith("OSC_E_") or k == "OSC_OK"}


class OscError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, code: int, message: str, func: str = ""):
        self.code = code
        self.func = func
        super().__init__(f"{func}: {_ERRNAMES.get(code, code)}: {message}")


class OscMesh3D(ctypes.Structure):
    """``osc_mesh3d``: scalar members of mesh3d_struct (code/open_spacecharge_mod.f90:14-27)."""

    _fields_ = [
        ("nlo", ctypes.c_int32 * 3),
        ("nhi", ctypes.c_int32 * 3),
        ("npad", ctypes.c_int32 * 3),
        ("min", ctypes.c_double * 3),
        ("max", ctypes.c_double * 3),
        ("delta", ctypes.c_double * 3),
        ("gamma", ctypes.c_double),
        ("charge", ctypes.c_double),
    ]


class OscBunch(ctypes.Structure):
    """``osc_bunch``: one bunch of a batched step (its mesh, particle range and charge)."""

    _fields_ = [
        ("mesh", OscMesh3D),
        ("offset", ctypes.c_int64),
        ("np", ctypes.c_int64),
        ("total_charge", ctypes.c_double),
        ("n_outside", ctypes.c_int64),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
_PM = ctypes.POINTER(OscMesh3D)
_PI64 = ctypes.POINTER(ctypes.c_int64)
_PD = ctypes.POINTER(ctypes.c_double)

# name -> argtypes (all return int unless listed in _RESTYPES)
SIGNATURES = {
    "osc_ctx_create": [_I, ctypes.POINTER(_P)],
    "osc_ctx_destroy": [_P],
    "osc_last_error": [_P],
    "osc_ctx_set_stream": [_P, _P],
    "osc_ctx_set_option": [_P, _I, _I64],
    "osc_ctx_get_option": [_P, _I, _PI64],
    "osc_ctx_synchronize": [_P],
    "osc_ctx_set_tuning": [_P, ctypes.c_char_p, _I],
    "osc_ctx_get_tuning": [_P, ctypes.c_char_p, ctypes.POINTER(_I)],
    "osc_clear_green_cache": [_P],
    "osc_version": [],
    "osc_profile_reset": [_P],
    "osc_profile_count": [_P, ctypes.POINTER(_I)],
    "osc_profile_entry": [_P, _I, ctypes.POINTER(ctypes.c_char_p), _PI64, _PD],
    "osc_launch_count": [_P, _PI64],
    "osc_graph_launch_count": [_P, _PI64],
    "osc_deposit_particles": [_P, _I64, _P, _P, _P, _P, _P, _I, _PM, _P, _PI64],
    "osc_deposit_particles_dev": [_P, _I64, _P, _P, _P, _P, _P, _I, _PM, _P, _PI64],
    "osc_sort_particles_dev": [_P, _PM, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _PI64],
    "osc_deposit_particles_dev_noalloc": [_P, _PM, _I64, _P, _P, _P, _P, _D, _P, _PI64, ctypes.c_char_p,
                                          ctypes.c_size_t],
    "osc_get_mesh_quantities": [_P, _I64, _P, _P, _P, _P, _P, _I, _P, _P],
    "osc_depose_rho_scalar": [_P, _I64, _P, _P, _P, _P, _D, _P, _P, _P, _P, _P, _PI64],
    "osc_space_charge_3d": [_P, _PM, _P, _P, _I, _I, _I, _P, _P],
    "osc_space_charge_3d_dev": [_P, _PM, _P, _P, _I, _I, _I, _P, _P],
    "osc_freespace_solver2": [_P, _P, _P, _D, _P, _P, _I, _P, _P],
    "osc_space_charge_freespace": [_P, _PM, _P, _I, _I, _I, _P, _P, _P],
    "osc_space_charge_cathodeimages": [_P, _PM, _P, _I, _I, _I, _I, _P, _P, _P],
    "osc_rectpipe_green": [_P, _PM, _D, _D, _I],
    "osc_space_charge_rectpipe": [_P, _PM, _P, _D, _D, _I, _I, _I, _P, _P, _P],
    "osc_space_charge_rectpipe_dev": [_P, _PM, _P, _D, _D, _I, _I, _I, _P, _P, _P],
    "osc_space_charge_step_rectpipe_dev": [_P, _PM, _I64, _P, _P, _P, _P, _P, _D, _D, _I, _P, _P],
    "osc_write_rectpipe_grn": [_P, ctypes.c_char_p, _D, _D, _PM],
    "osc_read_rectpipe_grn": [_P, ctypes.c_char_p, _PM, _PD, _PD],
    "osc_interpolate_field": [_P, _PM, _P, _P, _I64, _P, _P, _P, _P, _P, _PI64],
    "osc_interpolate_field_dev": [_P, _PM, _P, _P, _I64, _P, _P, _P, _P, _P, _PI64],
    "osc_space_charge_step": [_P, _PM, _I64, _P, _P, _P, _P, _P, _I, _I, _I, _P, _P],
    "osc_space_charge_step_dev": [_P, _PM, _I64, _P, _P, _P, _P, _P, _I, _I, _I, _P, _P],
    "osc_write_lines": [_P, _PM, _P, _D, _D, _D, ctypes.c_char_p],
    "osc_write_plane": [_P, _PM, _P, _P, ctypes.c_char_p],
    "osc_format_1pe14_7": [_D, ctypes.c_char_p],
    "osc_space_charge_step_vjp_dev": [_P, _PM, _I64, _P, _P, _P, _P, _D, _I, _P, _P, _P, _P, _P],
    "osc_batch_space_charge_step": [_P, _I, ctypes.POINTER(OscBunch), _P, _P, _P, _P, _I, _I, _P],
    "osc_batch_space_charge_step_dev": [_P, _I, ctypes.POINTER(OscBunch), _P, _P, _P, _P, _I, _I, _P],
    "osc_slab_deposit_dev": [_P, _PM, _I, _I, _I64, _P, _P, _P, _P, _D, _P, _PI64],
    "osc_slab_forward_dev": [_P, _PM, _I, _I, _P, _P],
    "osc_slab_zpass_dev": [_P, _PM, _I, _I, _P, _P],
    "osc_slab_inverse_dev": [_P, _PM, _I, _I, _P, _P],
    "osc_slab_interp_dev": [_P, _PM, _I, _I, _I64, _P, _P, _P, _P, _P],
}
_RESTYPES = {"osc_last_error": ctypes.c_char_p, "osc_version": ctypes.c_char_p}

_lib = None
_lock = threading.Lock()


def header_symbols(path: str = HEADER) -> list[str]:
    """Function names declared in the public header."""
    txt = open(path).read()
    return sorted(set(re.findall(r"^OSC_API\s+(?:const\s+char\s*\*|int)\s*(osc_\w+)\s*\(", txt, flags=re.M)))


def lib() -> ctypes.CDLL:
    """Load the native library (raises if it is missing; there is no fallback)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing; build it with `python -m openspacecharge_b200.build`")
            L = ctypes.CDLL(LIB_PATH)
            for name, args in SIGNATURES.items():
                f = getattr(L, name)
                f.argtypes = args
                f.restype = _RESTYPES.get(name, ctypes.c_int)
            _lib = L
    return _lib


def call(ctx, name: str, *args) -> None:
    """Call an entry point taking ``ctx`` first and raise OscError on a non-zero status."""
    rc = getattr(lib(), name)(ctx, *args)
    if rc != OSC_OK:
        msg = lib().osc_last_error(ctx)
        raise OscError(rc, msg.decode() if msg else "", name)


class Context:
    """An ``osc_ctx``: one CUDA stream, workspaces and the Green-spectrum cache."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        rc = lib().osc_ctx_create(int(device), ctypes.byref(self._h))
        if rc != OSC_OK:
            raise OscError(rc, "could not create a context (no usable CUDA device?)", "osc_ctx_create")
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if self._h:
            lib().osc_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def call(self, name: str, *args) -> None:
        call(self._h, name, *args)

    def set_option(self, opt: int, value: int) -> None:
        self.call("osc_ctx_set_option", int(opt), int(value))

    def get_option(self, opt: int) -> int:
        v = ctypes.c_int64()
        self.call("osc_ctx_get_option", int(opt), ctypes.byref(v))
        return int(v.value)

    def set_tuning(self, key: str, value: int) -> None:
        """Launch shape `key` (see osc_ctx_set_tuning); 0 restores the default."""
        self.call("osc_ctx_set_tuning", key.encode(), int(value))

    def get_tuning(self, key: str) -> int:
        v = ctypes.c_int()
        self.call("osc_ctx_get_tuning", key.encode(), ctypes.byref(v))
        return int(v.value)

    def set_stream(self, stream_ptr: int | None) -> None:
        """Run on the CUDA stream `stream_ptr` (0 = the default stream, e.g. torch's
        ``cuda_stream`` of it); None returns to the context's own stream."""
        self.call("osc_ctx_set_stream", ctypes.c_void_p(-1 if stream_ptr is None else int(stream_ptr)))

    def synchronize(self) -> None:
        self.call("osc_ctx_synchronize")

    def clear_green_cache(self) -> None:
        self.call("osc_clear_green_cache")

    def launch_count(self) -> int:
        v = ctypes.c_int64()
        self.call("osc_launch_count", ctypes.byref(v))
        return int(v.value)

    def graph_launch_count(self) -> int:
        """Batched steps that ran as one CUDA graph launch (OPT_BATCH_GRAPH)."""
        v = ctypes.c_int64()
        self.call("osc_graph_launch_count", ctypes.byref(v))
        return int(v.value)

    def profile(self) -> dict[str, tuple[int, float]]:
        """Per kernel name: (launches, summed ms) since the last reset (OPT_PROFILE=1)."""
        n = ctypes.c_int()
        self.call("osc_profile_count", ctypes.byref(n))
        out = {}
        for i in range(n.value):
            name = ctypes.c_char_p()
            cnt = ctypes.c_int64()
            ms = ctypes.c_double()
            self.call("osc_profile_entry", i, ctypes.byref(name), ctypes.byref(cnt), ctypes.byref(ms))
            out[name.value.decode()] = (int(cnt.value), float(ms.value))
        return out

    def profile_reset(self) -> None:
        self.call("osc_profile_reset")


def version() -> str:
    return lib().osc_version().decode()
