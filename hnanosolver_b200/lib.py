"""ctypes binding of libhns.so (include/hns.h).

The binding is thin: a Grid owns an hns_ctx; operator methods take torch CUDA tensors
(plumbing only: device memory and streams) and pass their raw pointers through the C ABI.
There is no CPU fallback: if libhns.so is missing or fails to load, import fails loudly.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libhns.so")

HNS_OK = 0
STATUS_NAMES = {
    0: "HNS_OK", 1: "HNS_ERR_INVALID_ARG", 2: "HNS_ERR_CUDA", 3: "HNS_ERR_OUT_OF_MEMORY", 4: "HNS_ERR_NOT_FOUND",
    5: "HNS_ERR_LAYOUT", 6: "HNS_ERR_NOT_CONVERGED", 7: "HNS_ERR_UNSUPPORTED", 8: "HNS_ERR_TIMEOUT",
}
SOLVE_ZERO_INIT = 1
SOLVE_NEUMANN = 2

_p = ctypes.c_void_p
_i64 = ctypes.c_int64
_f = ctypes.c_float
_i = ctypes.c_int
_u = ctypes.c_uint


class HnsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", _i), ("residual", ctypes.c_double), ("initial_residual", ctypes.c_double)]


def _sig(lib, name, res, *args):
    fn = getattr(lib, name)
    fn.restype = res
    fn.argtypes = list(args)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built: run `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ctypes.CDLL(LIB_PATH)
    _sig(lib, "hns_abi_version", _i)
    _sig(lib, "hns_status_string", ctypes.c_char_p, _i)
    _sig(lib, "hns_last_error", ctypes.c_char_p)
    _sig(lib, "hns_create", _i, ctypes.POINTER(_p), _p, _i64, _f, _i)
    _sig(lib, "hns_create_from_coords", _i, ctypes.POINTER(_p), _p, _i64, _f, _i)
    _sig(lib, "hns_destroy", _i, _p)
    _sig(lib, "hns_set_stream", _i, _p, _p)
    _sig(lib, "hns_get_stream", _p, _p)
    _sig(lib, "hns_synchronize", _i, _p)
    _sig(lib, "hns_num_voxels", _i64, _p)
    _sig(lib, "hns_num_leaves", _i64, _p)
    _sig(lib, "hns_voxel_size", _f, _p)
    _sig(lib, "hns_leaf_origins", _i, _p, _p)
    _sig(lib, "hns_index_offsets", _i, _p, _p, _i64, _p)
    _sig(lib, "hns_sort_leaves_nanovdb", _i, _p, _i64)
    _sig(lib, "hns_is_nanovdb_order", _i, _p, ctypes.POINTER(_i))
    _sig(lib, "hns_advect_vec3", _i, _p, _p, _p, _f)
    _sig(lib, "hns_advect_scalar", _i, _p, _p, _p, _p, _f)
    _sig(lib, "hns_advect_scalars", _i, _p, _p, _p, _p, _i, _f)
    _sig(lib, "hns_divergence", _i, _p, _p, _p)
    _sig(lib, "hns_rbgs", _i, _p, _p, _p, _i, _f, _u)
    _sig(lib, "hns_subtract_gradient", _i, _p, _p, _p, _p)
    _sig(lib, "hns_vorticity_confinement", _i, _p, _p, _p, _f, _f, _f)
    _sig(lib, "hns_project", _i, _p, _p, _i, _f, _u, ctypes.POINTER(SolveInfo))
    return lib


lib = _load()


def check(status: int) -> None:
    if status != HNS_OK:
        raise HnsError(status, lib.hns_last_error().decode(errors="replace"))


def sort_leaves_nanovdb(origins) -> np.ndarray:
    o = np.ascontiguousarray(np.asarray(origins, dtype=np.int32).reshape(-1, 3)).copy()
    check(lib.hns_sort_leaves_nanovdb(o.ctypes.data, len(o)))
    return o


def _dptr(t) -> int:
    """Raw device pointer of a contiguous torch CUDA tensor."""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return t.data_ptr()


class Grid:
    """A leaf-dense sparse domain on one GPU (an hns_ctx)."""

    def __init__(self, leaf_origins=None, voxel_size: float = 1.0, device: int = 0, coords=None):
        self._h = _p()
        if coords is not None:
            c = np.ascontiguousarray(np.asarray(coords, dtype=np.int32).reshape(-1, 3))
            check(lib.hns_create_from_coords(ctypes.byref(self._h), c.ctypes.data, len(c), voxel_size, device))
        else:
            o = np.ascontiguousarray(np.asarray(leaf_origins, dtype=np.int32).reshape(-1, 3))
            check(lib.hns_create(ctypes.byref(self._h), o.ctypes.data, len(o), voxel_size, device))
        self.device = device
        self.num_voxels = int(lib.hns_num_voxels(self._h))
        self.num_leaves = int(lib.hns_num_leaves(self._h))
        self.voxel_size = float(lib.hns_voxel_size(self._h))

    def close(self):
        if self._h:
            check(lib.hns_destroy(self._h))
            self._h = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        check(lib.hns_synchronize(self._h))

    def set_stream(self, stream_ptr):
        check(lib.hns_set_stream(self._h, stream_ptr))

    def leaf_origins(self) -> np.ndarray:
        out = np.zeros((self.num_leaves, 3), np.int32)
        check(lib.hns_leaf_origins(self._h, out.ctypes.data))
        return out

    def index_offsets(self, ijk) -> np.ndarray:
        ijk = np.ascontiguousarray(np.asarray(ijk, dtype=np.int32).reshape(-1, 3))
        out = np.zeros(len(ijk), np.uint64)
        check(lib.hns_index_offsets(self._h, ijk.ctypes.data, len(ijk), out.ctypes.data))
        return out

    def is_nanovdb_order(self) -> bool:
        v = _i()
        check(lib.hns_is_nanovdb_order(self._h, ctypes.byref(v)))
        return bool(v.value)

    # ---- operators (torch CUDA tensors in slot order; vec3 as (N, 3)) ----
    def advect_vec3(self, vel, out, dt):
        check(lib.hns_advect_vec3(self._h, _dptr(vel), _dptr(out), dt))

    def advect_scalar(self, vel, src, out, dt):
        check(lib.hns_advect_scalar(self._h, _dptr(vel), _dptr(src), _dptr(out), dt))

    def advect_scalars(self, vel, srcs, outs, dt):
        n = len(srcs)
        pin = (_p * max(1, n))(*[_dptr(t) for t in srcs])
        pout = (_p * max(1, n))(*[_dptr(t) for t in outs])
        check(lib.hns_advect_scalars(self._h, _dptr(vel), pin, pout, n, dt))

    def divergence(self, vel, div):
        check(lib.hns_divergence(self._h, _dptr(vel), _dptr(div)))

    def rbgs(self, div, p, iterations, omega, flags=0):
        check(lib.hns_rbgs(self._h, _dptr(div), _dptr(p), iterations, omega, flags))

    def subtract_gradient(self, vel, p, out):
        check(lib.hns_subtract_gradient(self._h, _dptr(vel), _dptr(p), _dptr(out)))

    def vorticity_confinement(self, vel, out, dt, scale, factor_scale):
        check(lib.hns_vorticity_confinement(self._h, _dptr(vel), _dptr(out), dt, scale, factor_scale))

    def project(self, vel, iterations, omega=-1.0, flags=0, info=True):
        si = SolveInfo()
        check(lib.hns_project(self._h, _dptr(vel), iterations, omega, flags, ctypes.byref(si) if info else None))
        return si if info else None
