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
OPT_RBGS_KERNEL = 1
RBGS_PLAIN, RBGS_BULK, RBGS_SPLIT = 0, 1, 2
OPT_INNER_LAYOUT = 2
INNER_ROWS, INNER_PACKED, INNER_SPLIT = 0, 1, 2
OPT_WAIT_POLLS = 3
OPT_SPLIT_SOLVE = 4
SPLIT_PER_COLOUR, SPLIT_PERSISTENT = 0, 1
OPT_COARSE_SOLVE = 5
COARSE_LAUNCHES, COARSE_CLUSTER = 0, 1
OPT_L2_PERSIST = 6
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


class StepDesc(ctypes.Structure):
    _fields_ = [("dt", _f), ("max_iterations", _i), ("omega", _f), ("tolerance", ctypes.c_double),
                ("check_every", _i), ("flags", _u), ("max_outer", _i), ("inner_iterations", _i)]


class MixedDesc(ctypes.Structure):
    _fields_ = [("dt", _f), ("omega", _f), ("tolerance", ctypes.c_double), ("max_outer", _i),
                ("inner_iterations", _i), ("flags", _u)]


DTYPE_F32, DTYPE_F16, DTYPE_BF16, DTYPE_F64 = 0, 1, 2, 3
SOLVE_REFINE = 4
SOLVE_MULTIGRID = 8


COMBUSTION_OXYGEN, COMBUSTION_RATE, COMBUSTION_NONE = 0, 1, 2


class ForceModel(ctypes.Structure):
    """hns_force_model: the burn (COMBUSTION_*) and the buoyancy's density term; the zero value
    is the reference's HNS_Advance."""

    _fields_ = [("combustion", _i), ("burn_rate", _f), ("heat_release", _f), ("ignition_temp", _f),
                ("density_buoyancy", _f)]


FIRE_FIELDS = ("velocity", "density", "temperature", "fuel", "waste", "flame")
FIRE_SOURCES = ("velocity", "temperature", "density", "fuel")


class FireFields(ctypes.Structure):
    """hns_fire_fields: BF16 velocity and FP16 scalars (device pointers, None: absent)."""

    _fields_ = [(k, _p) for k in FIRE_FIELDS]


class FireSources(ctypes.Structure):
    _fields_ = [(k, _p) for k in FIRE_SOURCES]


class FireF32(ctypes.Structure):
    """hns_fire_f32: FP32 arrays (host or device pointers by use; None: absent)."""

    _fields_ = [(k, _p) for k in FIRE_FIELDS]


class FireSourcesF32(ctypes.Structure):
    _fields_ = [(k, _p) for k in FIRE_SOURCES]


class CombustionParams(ctypes.Structure):
    """hns_combustion_params: the layout of the reference's CombustionParams."""

    _fields_ = [
        ("expansionRate", _f), ("temperatureRelease", _f), ("buoyancyStrength", _f), ("ambientTemp", _f),
        ("vorticityScale", _f), ("factorScale", _f), ("disturbanceEnable", _f), ("disturbanceStrength", _f),
        ("disturbanceSwirl", _f), ("disturbanceThreshold", _f), ("disturbanceGain", _f),
        ("disturbanceFrequency", _f), ("substeps", _i), ("gravity", _f), ("maskDensityMin", _f),
        ("maskDensityMax", _f), ("downloadVel", _i), ("simReset", _i),
    ]


NUM_PHASES = 8
PHASES = {"advect": 0, "divergence": 1, "solve": 2, "gradient": 3, "forces": 4, "inner": 5}


class ProfileData(ctypes.Structure):
    _fields_ = [("phase_ms", ctypes.c_double * NUM_PHASES), ("phase_count", _i * NUM_PHASES),
                ("solver_launches", ctypes.c_ulonglong), ("kernel_launches", ctypes.c_ulonglong)]


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
    _sig(lib, "hns_create_from_voxels", _i, ctypes.POINTER(_p), _p, _i64, _i, _i, _f, _i)
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
    _sig(lib, "hns_project_static", _i, _p, _p, _i, _f, _u, ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_step_plain", _i, _p, _p, _p, _p, _p, _i, ctypes.POINTER(StepDesc), ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_step_plain_host", _i, _p, _p, _p, _i, ctypes.POINTER(StepDesc), ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_last_solve", _i, _p, ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_solve_log", _i, _p, ctypes.POINTER(SolveInfo), _i, ctypes.POINTER(_i), _i)
    _sig(lib, "hns_field_set", _i, _p, ctypes.c_char_p, _i, _p, _i)
    _sig(lib, "hns_field_get", _i, _p, ctypes.c_char_p, _p, _i)
    _sig(lib, "hns_field_ptr", _i, _p, ctypes.c_char_p, ctypes.POINTER(_p), ctypes.POINTER(_i))
    _sig(lib, "hns_field_remove", _i, _p, ctypes.c_char_p)
    _sig(lib, "hns_field_count", _i, _p)
    _sig(lib, "hns_field_info", _i, _p, _i, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(_i))
    _sig(lib, "hns_advance", _i, _p, _i, _f, ctypes.POINTER(CombustionParams))
    _sig(lib, "hns_advance_model", _i, _p, _i, _f, ctypes.POINTER(CombustionParams), ctypes.POINTER(ForceModel))
    _sig(lib, "hns_active_mask", _i, _p, _p)
    _sig(lib, "hns_adjoint_advance", _i, _p, ctypes.POINTER(FireF32), ctypes.POINTER(FireSourcesF32),
         ctypes.POINTER(FireF32), ctypes.POINTER(FireF32), _f, _i, ctypes.POINTER(CombustionParams),
         ctypes.POINTER(ForceModel))
    _sig(lib, "hns_adjoint_advance_mixed", _i, _p, ctypes.POINTER(FireFields), ctypes.POINTER(FireSources),
         ctypes.POINTER(FireF32), ctypes.POINTER(FireF32), _f, ctypes.POINTER(CombustionParams),
         ctypes.POINTER(ForceModel), ctypes.POINTER(MixedDesc))
    _sig(lib, "hns_advance_solve", _i, _p, _f, ctypes.POINTER(CombustionParams), ctypes.POINTER(ForceModel),
         ctypes.POINTER(StepDesc), ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_advance_mixed_host", _i, _p, ctypes.POINTER(FireF32), ctypes.POINTER(FireSourcesF32), _f,
         ctypes.POINTER(CombustionParams), ctypes.POINTER(ForceModel), ctypes.POINTER(MixedDesc),
         ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_advance_mixed", _i, _p, ctypes.POINTER(FireFields), ctypes.POINTER(FireFields),
         ctypes.POINTER(FireSources), _f, ctypes.POINTER(CombustionParams), ctypes.POINTER(ForceModel),
         ctypes.POINTER(MixedDesc), ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_convert", _i, _p, _p, _i, _p, _i, _i64)
    _sig(lib, "hns_step_mixed", _i, _p, _p, _p, _p, _p, _i, ctypes.POINTER(MixedDesc), ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_step_mixed_host", _i, _p, _p, _p, _i, ctypes.POINTER(MixedDesc), ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_last_refine", _i, _p, ctypes.POINTER(SolveInfo))
    _sig(lib, "hns_refine_pressure", _i, _p, _p, ctypes.POINTER(_i), ctypes.POINTER(ctypes.c_double))
    _sig(lib, "hns_adjoint_advect_scalar", _i, _p, _p, _p, _p, _p, _p, _f)
    _sig(lib, "hns_adjoint_advect_vec3", _i, _p, _p, _p, _p, _f)
    _sig(lib, "hns_adjoint_divergence", _i, _p, _p, _p)
    _sig(lib, "hns_adjoint_subtract_gradient", _i, _p, _p, _p, _p)
    _sig(lib, "hns_adjoint_rbgs", _i, _p, _p, _p, _i, _f)
    _sig(lib, "hns_adjoint_project", _i, _p, _p, _i, _f)
    _sig(lib, "hns_adjoint_vorticity_confinement", _i, _p, _p, _p, _p, _f, _f, _f)
    _sig(lib, "hns_adjoint_step_plain", _i, _p, _p, _p, _i, _p, _p, _p, _p, _f, _i, _f)
    _sig(lib, "hns_set_option", _i, _p, _i, _i)
    _sig(lib, "hns_device_status", _i, _p)
    _sig(lib, "hns_profile_enable", _i, _p, _i)
    _sig(lib, "hns_profile_read", _i, _p, ctypes.POINTER(ProfileData))
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

    def __init__(self, leaf_origins=None, voxel_size: float = 1.0, device: int = 0, coords=None, voxels=None,
                 padding: int = 0):
        """leaf_origins (hns_create), coords of a leaf-dense layout (hns_create_from_coords), or
        voxels: active voxel coordinates (N, 3), a numpy array or a CUDA tensor on `device`,
        whose touched leaves after a `padding`-voxel dilation form the grid
        (hns_create_from_voxels)."""
        self._h = _p()
        if voxels is not None:
            if hasattr(voxels, "is_cuda") and voxels.is_cuda:
                if voxels.dtype != __import__("torch").int32 or not voxels.is_contiguous():
                    raise ValueError("voxels on the device must be a contiguous int32 tensor")
                check(lib.hns_create_from_voxels(ctypes.byref(self._h), voxels.data_ptr(), voxels.numel() // 3, padding, 1,
                                                 voxel_size, device))
            else:
                v = np.ascontiguousarray(np.asarray(voxels, dtype=np.int32).reshape(-1, 3))
                check(lib.hns_create_from_voxels(ctypes.byref(self._h), v.ctypes.data, len(v), padding, 0, voxel_size,
                                                 device))
        elif coords is not None:
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

    # ---- steps ----
    def step_plain(self, vel_in, vel_out, scalars_in, scalars_out, desc: StepDesc, info=False):
        n = len(scalars_in)
        pin = (_p * max(1, n))(*[_dptr(t) for t in scalars_in])
        pout = (_p * max(1, n))(*[_dptr(t) for t in scalars_out])
        si = SolveInfo()
        check(lib.hns_step_plain(self._h, _dptr(vel_in), _dptr(vel_out), pin, pout, n, ctypes.byref(desc),
                                 ctypes.byref(si) if info else None))
        return si if info else None

    def step_plain_host(self, vel: np.ndarray, scalars, desc: StepDesc, info=False):
        """vel (N,3) float32 and scalars (N,) float32 host arrays, updated in place."""
        for a in [vel, *scalars]:
            if a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError("host fields must be contiguous float32")
        ptrs = (_p * max(1, len(scalars)))(*[a.ctypes.data for a in scalars])
        si = SolveInfo()
        check(lib.hns_step_plain_host(self._h, vel.ctypes.data, ptrs, len(scalars), ctypes.byref(desc),
                                      ctypes.byref(si) if info else None))
        return si if info else None

    def last_solve(self) -> SolveInfo:
        si = SolveInfo()
        check(lib.hns_last_solve(self._h, ctypes.byref(si)))
        return si

    def profile_enable(self, on: bool = True):
        check(lib.hns_profile_enable(self._h, 1 if on else 0))

    def profile_read(self) -> ProfileData:
        d = ProfileData()
        check(lib.hns_profile_read(self._h, ctypes.byref(d)))
        return d

    # ---- named fields and the all-in-one step ----
    def field_set(self, name: str, data: np.ndarray | None = None, components: int | None = None):
        """Host numpy data ((N,) or (N,3) float32) or None for a zero field."""
        if data is not None:
            data = np.ascontiguousarray(data, dtype=np.float32)
            components = 3 if data.ndim == 2 else 1
        check(lib.hns_field_set(self._h, name.encode(), components or 1,
                                None if data is None else data.ctypes.data, 0))

    def field_get(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """Copy of a field into a new host array, or into `out` (contiguous float32 of the
        field's size)."""
        ptr, comps = _p(), _i()
        check(lib.hns_field_ptr(self._h, name.encode(), ctypes.byref(ptr), ctypes.byref(comps)))
        size = self.num_voxels * comps.value
        if out is None:
            out = np.zeros((self.num_voxels, 3) if comps.value == 3 else self.num_voxels, np.float32)
        elif out.dtype != np.float32 or not out.flags.c_contiguous or out.size != size:
            raise ValueError(f"out must be contiguous float32 with {size} values")
        check(lib.hns_field_get(self._h, name.encode(), out.ctypes.data, 0))
        return out

    def field_names(self):
        out = []
        buf = ctypes.create_string_buffer(256)
        comps = _i()
        for q in range(lib.hns_field_count(self._h)):
            check(lib.hns_field_info(self._h, q, buf, 256, ctypes.byref(comps)))
            out.append(buf.value.decode())
        return out

    def field_remove(self, name: str):
        check(lib.hns_field_remove(self._h, name.encode()))

    def advance(self, iterations: int, dt: float, params: CombustionParams, model: ForceModel | None = None):
        if model is None:
            check(lib.hns_advance(self._h, iterations, dt, ctypes.byref(params)))
        else:
            check(lib.hns_advance_model(self._h, iterations, dt, ctypes.byref(params), ctypes.byref(model)))

    def advance_mixed(self, fields_in: dict, fields_out: dict, sources: dict | None, dt: float,
                      params: CombustionParams, model: ForceModel | None, desc: MixedDesc, info: bool = False):
        """hns_advance_mixed on torch tensors: fields_in / fields_out map names of FIRE_FIELDS to
        BF16 (velocity) or FP16 device tensors; sources maps names of FIRE_SOURCES."""
        fi = FireFields(*[_dptr(fields_in.get(k)) for k in FIRE_FIELDS])
        fo = FireFields(*[_dptr(fields_out.get(k)) for k in FIRE_FIELDS])
        src = FireSources(*[_dptr((sources or {}).get(k)) for k in FIRE_SOURCES])
        si = SolveInfo()
        check(lib.hns_advance_mixed(self._h, ctypes.byref(fi), ctypes.byref(fo), ctypes.byref(src), dt,
                                    ctypes.byref(params), ctypes.byref(model) if model is not None else None,
                                    ctypes.byref(desc), ctypes.byref(si) if info else None))
        return si if info else None

    def advance_solve(self, dt: float, params: CombustionParams, model: ForceModel | None, desc: StepDesc,
                      info: bool = False):
        """hns_advance_solve: the all-in-one step with each solve run to desc.tolerance."""
        si = SolveInfo()
        check(lib.hns_advance_solve(self._h, dt, ctypes.byref(params),
                                    ctypes.byref(model) if model is not None else None, ctypes.byref(desc),
                                    ctypes.byref(si) if info else None))
        return si if info else None

    def advance_mixed_host(self, fields: dict, sources: dict | None, dt: float, params: CombustionParams,
                           model: ForceModel | None, desc: MixedDesc, info: bool = False):
        """hns_advance_mixed_host: `fields` maps FIRE_FIELDS names to contiguous float32 host
        arrays, updated in place; `sources` maps FIRE_SOURCES names to float32 host arrays."""
        for a in list(fields.values()) + list((sources or {}).values()):
            if a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError("host fields must be contiguous float32")
        fh = FireF32(*[fields[k].ctypes.data if k in fields else None for k in FIRE_FIELDS])
        src = FireSourcesF32(*[(sources or {})[k].ctypes.data if k in (sources or {}) else None for k in FIRE_SOURCES])
        si = SolveInfo()
        check(lib.hns_advance_mixed_host(self._h, ctypes.byref(fh), ctypes.byref(src), dt, ctypes.byref(params),
                                         ctypes.byref(model) if model is not None else None, ctypes.byref(desc),
                                         ctypes.byref(si) if info else None))
        return si if info else None

    def adjoint_advance(self, fields_in: dict, sources: dict | None, out_bar: dict, in_bar: dict, dt: float,
                        iterations: int, params: CombustionParams, model: ForceModel | None):
        """hns_adjoint_advance on FP32 device tensors (dicts keyed by FIRE_FIELDS / FIRE_SOURCES)."""
        f = lambda d, cls, keys: cls(*[_dptr((d or {}).get(k)) for k in keys])  # noqa: E731
        check(lib.hns_adjoint_advance(self._h, ctypes.byref(f(fields_in, FireF32, FIRE_FIELDS)),
                                      ctypes.byref(f(sources, FireSourcesF32, FIRE_SOURCES)),
                                      ctypes.byref(f(out_bar, FireF32, FIRE_FIELDS)),
                                      ctypes.byref(f(in_bar, FireF32, FIRE_FIELDS)), dt, iterations,
                                      ctypes.byref(params), ctypes.byref(model) if model is not None else None))

    def adjoint_advance_mixed(self, fields_in: dict, sources: dict | None, out_bar: dict, in_bar: dict, dt: float,
                              params: CombustionParams, model: ForceModel | None, desc: MixedDesc):
        """hns_adjoint_advance_mixed: BF16/FP16 inputs and sources, FP32 adjoints."""
        f = lambda d, cls, keys: cls(*[_dptr((d or {}).get(k)) for k in keys])  # noqa: E731
        check(lib.hns_adjoint_advance_mixed(self._h, ctypes.byref(f(fields_in, FireFields, FIRE_FIELDS)),
                                            ctypes.byref(f(sources, FireSources, FIRE_SOURCES)),
                                            ctypes.byref(f(out_bar, FireF32, FIRE_FIELDS)),
                                            ctypes.byref(f(in_bar, FireF32, FIRE_FIELDS)), dt, ctypes.byref(params),
                                            ctypes.byref(model) if model is not None else None, ctypes.byref(desc)))

    def active_mask(self) -> np.ndarray:
        out = np.zeros(self.num_voxels, np.uint8)
        check(lib.hns_active_mask(self._h, out.ctypes.data))
        return out

    def set_option(self, option: int, value: int):
        check(lib.hns_set_option(self._h, option, value))

    def device_status(self):
        check(lib.hns_device_status(self._h))

    # ---- adjoints (each adds into the *_bar arrays) ----
    def adjoint_advect_scalar(self, vel, inp, out_bar, in_bar, vel_bar, dt):
        check(lib.hns_adjoint_advect_scalar(self._h, _dptr(vel), _dptr(inp), _dptr(out_bar), _dptr(in_bar), _dptr(vel_bar), dt))

    def adjoint_advect_vec3(self, vel, out_bar, vel_bar, dt):
        check(lib.hns_adjoint_advect_vec3(self._h, _dptr(vel), _dptr(out_bar), _dptr(vel_bar), dt))

    def adjoint_divergence(self, div_bar, vel_bar):
        check(lib.hns_adjoint_divergence(self._h, _dptr(div_bar), _dptr(vel_bar)))

    def adjoint_subtract_gradient(self, out_bar, vel_bar, p_bar):
        check(lib.hns_adjoint_subtract_gradient(self._h, _dptr(out_bar), _dptr(vel_bar), _dptr(p_bar)))

    def adjoint_rbgs(self, p_bar, div_bar, iterations, omega):
        check(lib.hns_adjoint_rbgs(self._h, _dptr(p_bar), _dptr(div_bar), iterations, omega))

    def adjoint_project(self, vel_bar, iterations, omega=-1.0):
        check(lib.hns_adjoint_project(self._h, _dptr(vel_bar), iterations, omega))

    def adjoint_vorticity_confinement(self, vel, out_bar, vel_bar, dt, scale, factor_scale):
        check(lib.hns_adjoint_vorticity_confinement(self._h, _dptr(vel), _dptr(out_bar), _dptr(vel_bar), dt, scale,
                                                    factor_scale))

    def adjoint_step_plain(self, vel_in, scalars_in, vel_out_bar, scalars_out_bar, vel_in_bar, scalars_in_bar, dt,
                           iterations, omega):
        n = len(scalars_in)
        arr = lambda ts: (_p * max(1, n))(*[_dptr(t) for t in ts])  # noqa: E731
        check(lib.hns_adjoint_step_plain(self._h, _dptr(vel_in), arr(scalars_in), n, _dptr(vel_out_bar),
                                         arr(scalars_out_bar), _dptr(vel_in_bar), arr(scalars_in_bar), dt, iterations,
                                         omega))

    # ---- mixed precision ----
    def convert(self, src, src_dtype: int, dst, dst_dtype: int, count: int):
        check(lib.hns_convert(self._h, _dptr(src), src_dtype, _dptr(dst), dst_dtype, count))

    def step_mixed(self, vel_in, vel_out, scalars_in, scalars_out, desc: MixedDesc, info=False):
        """vel as torch bfloat16 (N,3), scalars as torch float16 (N,)."""
        n = len(scalars_in)
        pin = (_p * max(1, n))(*[_dptr(t) for t in scalars_in])
        pout = (_p * max(1, n))(*[_dptr(t) for t in scalars_out])
        si = SolveInfo()
        check(lib.hns_step_mixed(self._h, _dptr(vel_in), _dptr(vel_out), pin, pout, n, ctypes.byref(desc),
                                 ctypes.byref(si) if info else None))
        return si if info else None

    def step_mixed_host(self, vel: np.ndarray, scalars, desc: MixedDesc, info=False):
        for a in [vel, *scalars]:
            if a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError("host fields must be contiguous float32")
        ptrs = (_p * max(1, len(scalars)))(*[a.ctypes.data for a in scalars])
        si = SolveInfo()
        check(lib.hns_step_mixed_host(self._h, vel.ctypes.data, ptrs, len(scalars), ctypes.byref(desc),
                                      ctypes.byref(si) if info else None))
        return si if info else None

    def solve_log(self, capacity: int = 4096, reset: bool = True):
        """(count, entries): solves logged since the last reset, and the most recent
        min(count, 4096, capacity) of them, oldest first (hns_solve_log)."""
        arr = (SolveInfo * max(1, capacity))()
        count = _i()
        check(lib.hns_solve_log(self._h, arr, capacity, ctypes.byref(count), 1 if reset else 0))
        k = min(count.value, 4096, capacity)
        return count.value, [arr[q] for q in range(k)]

    def last_refine(self) -> SolveInfo:
        si = SolveInfo()
        check(lib.hns_last_refine(self._h, ctypes.byref(si)))
        return si

    def refine_pressure(self, out):
        outer, res = _i(), ctypes.c_double()
        check(lib.hns_refine_pressure(self._h, _dptr(out), ctypes.byref(outer), ctypes.byref(res)))
        return outer.value, res.value
