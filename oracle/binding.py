"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Two libraries:
  Oracle     oracle/_build/libhns_oracle.so -- the plain-C restatement (hns_oracle.h)
  RefOracle  oracle/_ref/libhns_ref.so      -- the reference's own src/Cuda/Kernel.cu
                                               compiled as host C++ (ref_driver.cpp)
Only tests/, bench.py's CPU-baseline leg and the smoke check use them, as the checker.
"""
from __future__ import annotations

import ctypes
import os
import platform
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libhns_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhns_ref.so")
REF_SO_V3 = os.path.join(HERE, "_ref", "libhns_ref_x86v3.so")

_p = ctypes.c_void_p
_i64 = ctypes.c_int64
_f = ctypes.c_float
_d = ctypes.c_double
_i = ctypes.c_int


def build(ref: bool | None = None) -> None:
    """Compile the oracle and oracle/_ref: always with ref=True, never with ref=False, and with
    ref=None only where the reference checkout exists (oracle/Makefile's ref-if-present: the
    HNS_REFERENCE environment variable or the recipe's default path)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref is None:
        subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)
    elif ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class CombustionParams(ctypes.Structure):
    """Layout of the reference's CombustionParams (src/Cuda/Kernels.cuh:5-24)."""

    _fields_ = [
        ("expansionRate", _f), ("temperatureRelease", _f), ("buoyancyStrength", _f), ("ambientTemp", _f),
        ("vorticityScale", _f), ("factorScale", _f), ("disturbanceEnable", _f), ("disturbanceStrength", _f),
        ("disturbanceSwirl", _f), ("disturbanceThreshold", _f), ("disturbanceGain", _f),
        ("disturbanceFrequency", _f), ("substeps", _i), ("gravity", _f), ("maskDensityMin", _f),
        ("maskDensityMax", _f), ("downloadVel", _i), ("simReset", _i),
    ]

    @classmethod
    def houdini_defaults(cls) -> "CombustionParams":
        """The SOP's parameter defaults (src/SOP/HNanoSolver/SOP_HNanoSolver.cpp:23-184)."""
        return cls(expansionRate=0.1, temperatureRelease=0.5, buoyancyStrength=1.0, ambientTemp=23.0,
                   vorticityScale=1.0, factorScale=0.5, disturbanceEnable=1.0, substeps=1, gravity=1.0)


class AdvanceFields(ctypes.Structure):
    _fields_ = [
        ("n", _i64), ("velocity", _p), ("nscalars", _i), ("names", ctypes.POINTER(ctypes.c_char_p)),
        ("scalars", ctypes.POINTER(_p)), ("created", _p * 4), ("src_vel", _p), ("src_vel_x", _p),
        ("src_vel_y", _p), ("src_vel_z", _p), ("src_temperature", _p), ("src_density", _p), ("src_fuel", _p),
        ("collision_sdf", _p),
    ]


class ForceModel(ctypes.Structure):
    """hnso_force_model: combustion 0 oxygen (the reference's step), 1 rate/heat, 2 none; the
    buoyancy's density term alpha; omega > 0 replaces the solves' SOR factor."""

    _fields_ = [("combustion", _i), ("burn_rate", _d), ("heat_release", _d), ("ignition_temp", _d),
                ("density_buoyancy", _d), ("omega", _d)]


# Fields each combustion model uses, created zero-filled when absent (fuel, waste, temperature, flame).
MODEL_FIELDS = {0: ("fuel", "waste", "temperature", "flame"), 1: ("fuel", "temperature"), 2: ("temperature",)}


def make_advance_fields(n, velocity, scalars: dict, created: dict, sources: dict):
    """Keep-alive tuple (struct, refs) for an HNS_Advance call. `scalars` is the ordered
    name->array dict of persistent fields present at call start; `created` maps any of
    fuel/waste/temperature/flame absent from it to an output buffer. `sources` may also hold
    "collision_sdf", the collider's signed distance per voxel."""
    names = list(scalars)
    cnames = (ctypes.c_char_p * max(1, len(names)))(*[s.encode() for s in names])
    cptrs = (_p * max(1, len(names)))(*[scalars[s].ctypes.data for s in names])
    f = AdvanceFields()
    f.n = n
    f.velocity = velocity.ctypes.data
    f.nscalars = len(names)
    f.names = ctypes.cast(cnames, ctypes.POINTER(ctypes.c_char_p))
    f.scalars = ctypes.cast(cptrs, ctypes.POINTER(_p))
    for k, nm in enumerate(("fuel", "waste", "temperature", "flame")):
        f.created[k] = created[nm].ctypes.data if nm in created else None
    for key in ("src_vel", "src_vel_x", "src_vel_y", "src_vel_z", "src_temperature", "src_density", "src_fuel",
                "collision_sdf"):
        setattr(f, key, sources[key].ctypes.data if key in sources else None)
    return f, (cnames, cptrs, velocity, scalars, created, sources)


def _sig(lib, name, res, *args):
    fn = getattr(lib, name)
    fn.restype = res
    fn.argtypes = list(args)
    return fn


class Oracle:
    """The C restatement. Fields are numpy arrays in leaf-dense slot order."""

    def __init__(self, path: str = ORACLE_SO):
        self.lib = lib = ctypes.CDLL(path)
        _sig(lib, "hnso_topo_create", _p, _p, _i64)
        _sig(lib, "hnso_topo_destroy", None, _p)
        _sig(lib, "hnso_topo_num_voxels", _i64, _p)
        _sig(lib, "hnso_offsets", None, _p, _p, _i64, _p)
        _sig(lib, "hnso_slot_coords", None, _p, _p)
        _sig(lib, "hnso_sort_leaves_nanovdb", None, _p, _i64)
        for s, r in (("_f32", _f), ("_f64", _d)):
            _sig(lib, "hnso_sample_trilinear_scalar" + s, None, _p, _p, _p, _i64, _p)
            _sig(lib, "hnso_sample_trilinear_vec3" + s, None, _p, _p, _p, _i64, _p)
            _sig(lib, "hnso_advect_vector" + s, None, _p, _p, _p, r, r)
            _sig(lib, "hnso_advect_scalars" + s, None, _p, _p, _p, _p, _i, r, r)
            _sig(lib, "hnso_advect_scalar" + s, None, _p, _p, _p, _p, r, r)
            _sig(lib, "hnso_divergence" + s, None, _p, _p, _p, r)
            _sig(lib, "hnso_rbgs_sweep" + s, None, _p, _p, _p, r, _i, r)
            _sig(lib, "hnso_rbgs" + s, None, _p, _p, _p, r, _i, r)
            _sig(lib, "hnso_residual" + s, None, _p, _p, _p, r, _p, _p)
            _sig(lib, "hnso_subtract_gradient" + s, None, _p, _p, _p, _p, r)
            _sig(lib, "hnso_vorticity_confinement" + s, None, _p, _p, _p, r, r, r, r)
            _sig(lib, "hnso_temperature_buoyancy" + s, None, _i64, _p, _p, _p, r, r, r)
            _sig(lib, "hnso_combustion" + s, None, _i64, _p, _p, _p, _p, r, r, r, r)
            _sig(lib, "hnso_combustion_oxygen" + s, None, _i64, _p, _p, _p, _p, _p, _p, _p, _p, _p, r, r)
            _sig(lib, "hnso_add_scalar_source" + s, None, _i64, _p, _p, r)
            _sig(lib, "hnso_add_velocity_source" + s, None, _i64, _p, _p, r)
            _sig(lib, "hnso_add_velocity_source_xyz" + s, None, _i64, _p, _p, _p, _p, r)
            _sig(lib, "hnso_add_gravity" + s, None, _i64, _p, r, r)
            _sig(lib, "hnso_project" + s, None, _p, _p, _p, _p, r, _i, r)
            _sig(lib, "hnso_rbgs_neumann" + s, None, _p, _p, _p, r, _i, r)
            _sig(lib, "hnso_residual_neumann" + s, None, _p, _p, _p, r, _p, _p)
            _sig(lib, "hnso_remove_mean" + s, None, _p, _p)
            _sig(lib, "hnso_project_neumann" + s, None, _p, _p, _p, _p, r, _i, r)
        for suf, real in (("_f32", _f), ("_f64", _d)):
            _sig(lib, "hnso_hns_advance_model" + suf, None, _p, ctypes.POINTER(AdvanceFields), real, _i, real,
                 ctypes.POINTER(CombustionParams), ctypes.POINTER(ForceModel))
        _sig(lib, "hnso_hns_advance_f32", None, _p, ctypes.POINTER(AdvanceFields), _f, _i, _f,
             ctypes.POINTER(CombustionParams))

    def sort_leaves(self, origins):
        o = np.ascontiguousarray(np.asarray(origins, dtype=np.int32).reshape(-1, 3)).copy()
        self.lib.hnso_sort_leaves_nanovdb(ptr(o), len(o))
        return o

    def topo(self, origins) -> "OracleTopo":
        return OracleTopo(self, origins)


class OracleTopo:
    def __init__(self, oracle: Oracle, origins):
        self.o = oracle
        self.origins = np.ascontiguousarray(np.asarray(origins, dtype=np.int32).reshape(-1, 3))
        self.h = oracle.lib.hnso_topo_create(ptr(self.origins), len(self.origins))
        self.n = int(oracle.lib.hnso_topo_num_voxels(self.h))

    def __del__(self):
        try:
            self.o.lib.hnso_topo_destroy(self.h)
        except Exception:
            pass

    def _dt(self, a):
        return "_f64" if a.dtype == np.float64 else "_f32"

    def offsets(self, ijk):
        ijk = np.ascontiguousarray(np.asarray(ijk, dtype=np.int32).reshape(-1, 3))
        out = np.zeros(len(ijk), dtype=np.uint64)
        self.o.lib.hnso_offsets(self.h, ptr(ijk), len(ijk), ptr(out))
        return out

    def coords(self):
        out = np.zeros((self.n, 3), dtype=np.int32)
        self.o.lib.hnso_slot_coords(self.h, ptr(out))
        return out

    def sample_trilinear(self, data, xyz):
        data = np.ascontiguousarray(data)
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=data.dtype).reshape(-1, 3))
        s = self._dt(data)
        if data.ndim == 2:
            out = np.zeros((len(xyz), 3), dtype=data.dtype)
            getattr(self.o.lib, "hnso_sample_trilinear_vec3" + s)(self.h, ptr(data), ptr(xyz), len(xyz), ptr(out))
        else:
            out = np.zeros(len(xyz), dtype=data.dtype)
            getattr(self.o.lib, "hnso_sample_trilinear_scalar" + s)(self.h, ptr(data), ptr(xyz), len(xyz), ptr(out))
        return out

    def advect_vector(self, vel, dt, inv_dx):
        vel = np.ascontiguousarray(vel)
        out = np.zeros_like(vel)
        getattr(self.o.lib, "hnso_advect_vector" + self._dt(vel))(self.h, ptr(vel), ptr(out), dt, inv_dx)
        return out

    def advect_scalars(self, vel, fields, dt, inv_dx):
        vel = np.ascontiguousarray(vel)
        ins = [np.ascontiguousarray(f, dtype=vel.dtype) for f in fields]
        outs = [np.zeros_like(f) for f in ins]
        pin = (_p * len(ins))(*[f.ctypes.data for f in ins])
        pout = (_p * len(outs))(*[f.ctypes.data for f in outs])
        getattr(self.o.lib, "hnso_advect_scalars" + self._dt(vel))(self.h, ptr(vel), pin, pout, len(ins), dt, inv_dx)
        return outs

    def advect_scalar(self, vel, field, dt, inv_dx):
        vel = np.ascontiguousarray(vel)
        field = np.ascontiguousarray(field, dtype=vel.dtype)
        out = np.zeros_like(field)
        getattr(self.o.lib, "hnso_advect_scalar" + self._dt(vel))(self.h, ptr(vel), ptr(field), ptr(out), dt, inv_dx)
        return out

    def divergence(self, vel, inv_dx):
        vel = np.ascontiguousarray(vel)
        out = np.zeros(len(vel), dtype=vel.dtype)
        getattr(self.o.lib, "hnso_divergence" + self._dt(vel))(self.h, ptr(vel), ptr(out), inv_dx)
        return out

    def rbgs(self, div, p, dx, iterations, omega):
        p = np.ascontiguousarray(p).copy()
        div = np.ascontiguousarray(div, dtype=p.dtype)
        getattr(self.o.lib, "hnso_rbgs" + self._dt(p))(self.h, ptr(div), ptr(p), dx, iterations, omega)
        return p

    def residual(self, div, p, dx):
        div = np.ascontiguousarray(div)
        p = np.ascontiguousarray(p, dtype=div.dtype)
        r2, b2 = ctypes.c_double(), ctypes.c_double()
        getattr(self.o.lib, "hnso_residual" + self._dt(div))(self.h, ptr(div), ptr(p), dx, ctypes.byref(r2),
                                                             ctypes.byref(b2))
        return r2.value, b2.value

    def subtract_gradient(self, vel, p, inv_dx):
        vel = np.ascontiguousarray(vel)
        p = np.ascontiguousarray(p, dtype=vel.dtype)
        out = np.zeros_like(vel)
        getattr(self.o.lib, "hnso_subtract_gradient" + self._dt(vel))(self.h, ptr(vel), ptr(p), ptr(out), inv_dx)
        return out

    def vorticity_confinement(self, vel, dt, inv_dx, scale, factor_scale):
        vel = np.ascontiguousarray(vel)
        out = np.zeros_like(vel)
        getattr(self.o.lib, "hnso_vorticity_confinement" + self._dt(vel))(self.h, ptr(vel), ptr(out), dt, inv_dx,
                                                                          scale, factor_scale)
        return out

    def rbgs_neumann(self, div, p, dx, iterations, omega):
        """Red-black SOR with zero-gradient walls (no mean removal)."""
        p = np.ascontiguousarray(p).copy()
        div = np.ascontiguousarray(div, dtype=p.dtype)
        getattr(self.o.lib, "hnso_rbgs_neumann" + self._dt(p))(self.h, ptr(div), ptr(p), dx, iterations, omega)
        return p

    def residual_neumann(self, div, p, dx):
        div = np.ascontiguousarray(div)
        p = np.ascontiguousarray(p, dtype=div.dtype)
        r2, b2 = ctypes.c_double(), ctypes.c_double()
        getattr(self.o.lib, "hnso_residual_neumann" + self._dt(div))(self.h, ptr(div), ptr(p), dx, ctypes.byref(r2),
                                                                     ctypes.byref(b2))
        return r2.value, b2.value

    def remove_mean(self, div):
        div = np.ascontiguousarray(div).copy()
        getattr(self.o.lib, "hnso_remove_mean" + self._dt(div))(self.h, ptr(div))
        return div

    def project_neumann(self, vel, dx, iterations, omega):
        vel = np.ascontiguousarray(vel).copy()
        div = np.zeros(len(vel), dtype=vel.dtype)
        p = np.zeros(len(vel), dtype=vel.dtype)
        getattr(self.o.lib, "hnso_project_neumann" + self._dt(vel))(self.h, ptr(vel), ptr(div), ptr(p), dx, iterations,
                                                                    omega)
        return vel, div, p

    def project(self, vel, dx, iterations, omega):
        vel = np.ascontiguousarray(vel).copy()
        div = np.zeros(len(vel), dtype=vel.dtype)
        p = np.zeros(len(vel), dtype=vel.dtype)
        getattr(self.o.lib, "hnso_project" + self._dt(vel))(self.h, ptr(vel), ptr(div), ptr(p), dx, iterations, omega)
        return vel, div, p

    def hns_advance(self, velocity, scalars: dict, sources: dict, dx, iteration, dt, params: CombustionParams):
        """Returns (velocity, scalars, created) after one HNS_Advance call, copies of the inputs."""
        vel = np.ascontiguousarray(velocity, dtype=np.float32).copy()
        sc = {k: np.ascontiguousarray(v, dtype=np.float32).copy() for k, v in scalars.items()}
        created = {k: np.zeros(self.n, np.float32) for k in ("fuel", "waste", "temperature", "flame") if k not in sc}
        src = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in sources.items()}
        f, keep = make_advance_fields(self.n, vel, sc, created, src)
        self.o.lib.hnso_hns_advance_f32(self.h, ctypes.byref(f), dx, iteration, dt, ctypes.byref(params))
        del keep
        return vel, sc, created


    def hns_advance_model(self, velocity, scalars: dict, sources: dict, dx, iteration, dt, params: CombustionParams,
                          model: ForceModel | None = None, dtype=np.float32):
        """hns_advance with a force model, in float32 or float64. Returns (velocity, scalars,
        created), copies of the inputs; `created` holds the fields the model made."""
        model = model or ForceModel()
        vel = np.ascontiguousarray(velocity, dtype=dtype).copy()
        sc = {k: np.ascontiguousarray(v, dtype=dtype).copy() for k, v in scalars.items()}
        created = {k: np.zeros(self.n, dtype) for k in MODEL_FIELDS[model.combustion] if k not in sc}
        src = {k: np.ascontiguousarray(v, dtype=dtype) for k, v in sources.items()}
        f, keep = make_advance_fields(self.n, vel, sc, created, src)
        suf = "_f64" if np.dtype(dtype) == np.float64 else "_f32"
        getattr(self.o.lib, "hnso_hns_advance_model" + suf)(self.h, ctypes.byref(f), dx, iteration, dt,
                                                            ctypes.byref(params), ctypes.byref(model))
        del keep
        return vel, sc, created


class RefOracle:
    """The reference's own kernels (host-compiled). Takes the leaf-dense coordinates and
    builds the reference's NanoVDB ValueOnIndex grid from them."""

    def __init__(self, path: str | None = None):
        if path is None:
            path = REF_SO_V3 if (os.path.exists(REF_SO_V3) and _cpu_has_avx2_fma()) else REF_SO
        self.path = path
        self.lib = lib = ctypes.CDLL(path)
        _sig(lib, "ref_num_threads", _i)
        _sig(lib, "ref_set_num_threads", None, _i)
        _sig(lib, "ref_set_block_stride", None, _i)
        _sig(lib, "ref_grid_create", _p, _p, _i64)
        _sig(lib, "ref_grid_destroy", None, _p)
        _sig(lib, "ref_grid_value_count", ctypes.c_uint64, _p)
        _sig(lib, "ref_grid_leaf_count", ctypes.c_uint64, _p)
        _sig(lib, "ref_grid_leaf_origins", None, _p, _p)
        _sig(lib, "ref_grid_offsets", None, _p, _p, _i64, _p)
        _sig(lib, "ref_sample_scalar", None, _p, _p, _p, _i64, _i, _p)
        _sig(lib, "ref_sample_vec3", None, _p, _p, _p, _i64, _i, _p)
        _sig(lib, "ref_advect_vector", None, _p, _p, _i64, _p, _p, _f, _f)
        _sig(lib, "ref_advect_scalars", None, _p, _p, _i64, _p, _p, _p, _i, _f, _f)
        _sig(lib, "ref_advect_scalar", None, _p, _p, _i64, _p, _p, _p, _f, _f)
        _sig(lib, "ref_divergence", None, _p, _p, _i64, _p, _p, _f)
        _sig(lib, "ref_rbgs", None, _p, _p, _i64, _p, _p, _f, _i, _f)
        _sig(lib, "ref_subtract_gradient", None, _p, _p, _i64, _p, _p, _p, _f)
        _sig(lib, "ref_vorticity_confinement", None, _p, _p, _i64, _p, _p, _f, _f, _f, _f)
        _sig(lib, "ref_temperature_buoyancy", None, _i64, _p, _p, _p, _f, _f, _f)
        _sig(lib, "ref_combustion", None, _i64, _p, _p, _p, _p, _f, _f, _f, _f)
        _sig(lib, "ref_combustion_oxygen", None, _i64, _p, _p, _p, _p, _p, _p, _p, _p, _p, _f, _f)
        _sig(lib, "ref_add_scalar_source", None, _i64, _p, _p, _f)
        _sig(lib, "ref_add_velocity_source", None, _i64, _p, _p, _f)
        _sig(lib, "ref_add_velocity_source_xyz", None, _i64, _p, _p, _p, _p, _f)
        _sig(lib, "ref_add_gravity", None, _i64, _p, _f, _f)
        _sig(lib, "ref_project", None, _p, _p, _i64, _p, _p, _p, _f, _i, _f)
        _sig(lib, "ref_hns_advance", None, _p, _p, ctypes.POINTER(AdvanceFields), _f, _i, _f,
             ctypes.POINTER(CombustionParams))
        _sig(lib, "ref_plain_step", None, _p, _p, _i64, _p, _p, _i, _f, _f, _i, _f, _p)

        _sig(lib, "ref_hns_advance_model", None, _p, _p, ctypes.POINTER(AdvanceFields), _f, _i, _f,
             ctypes.POINTER(CombustionParams), _i, _f, _f, _f, _f)

    def grid(self, coords) -> "RefGrid":
        return RefGrid(self, coords)


class RefGrid:
    def __init__(self, ref: RefOracle, coords):
        self.r = ref
        self.coords = np.ascontiguousarray(np.asarray(coords, dtype=np.int32).reshape(-1, 3))
        self.n = len(self.coords)
        self.h = ref.lib.ref_grid_create(ptr(self.coords), self.n)

    def __del__(self):
        try:
            self.r.lib.ref_grid_destroy(self.h)
        except Exception:
            pass

    @property
    def lib(self):
        return self.r.lib

    def leaf_origins(self):
        n = int(self.lib.ref_grid_leaf_count(self.h))
        out = np.zeros((n, 3), dtype=np.int32)
        self.lib.ref_grid_leaf_origins(self.h, ptr(out))
        return out

    def value_count(self):
        return int(self.lib.ref_grid_value_count(self.h))

    def offsets(self, ijk):
        ijk = np.ascontiguousarray(np.asarray(ijk, dtype=np.int32).reshape(-1, 3))
        out = np.zeros(len(ijk), dtype=np.uint64)
        self.lib.ref_grid_offsets(self.h, ptr(ijk), len(ijk), ptr(out))
        return out

    def sample(self, data, xyz, order=1):
        data = np.ascontiguousarray(data, dtype=np.float32)
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.float32).reshape(-1, 3))
        if data.ndim == 2:
            out = np.zeros((len(xyz), 3), np.float32)
            self.lib.ref_sample_vec3(self.h, ptr(data), ptr(xyz), len(xyz), order, ptr(out))
        else:
            out = np.zeros(len(xyz), np.float32)
            self.lib.ref_sample_scalar(self.h, ptr(data), ptr(xyz), len(xyz), order, ptr(out))
        return out

    def advect_vector(self, vel, dt, inv_dx):
        vel = np.ascontiguousarray(vel, dtype=np.float32)
        out = np.zeros_like(vel)
        self.lib.ref_advect_vector(self.h, ptr(self.coords), self.n, ptr(vel), ptr(out), dt, inv_dx)
        return out

    def advect_scalars(self, vel, fields, dt, inv_dx):
        vel = np.ascontiguousarray(vel, dtype=np.float32)
        ins = [np.ascontiguousarray(f, dtype=np.float32) for f in fields]
        outs = [np.zeros_like(f) for f in ins]
        pin = (_p * len(ins))(*[f.ctypes.data for f in ins])
        pout = (_p * len(outs))(*[f.ctypes.data for f in outs])
        self.lib.ref_advect_scalars(self.h, ptr(self.coords), self.n, ptr(vel), pin, pout, len(ins), dt, inv_dx)
        return outs

    def advect_scalar(self, vel, field, dt, inv_dx):
        vel = np.ascontiguousarray(vel, dtype=np.float32)
        field = np.ascontiguousarray(field, dtype=np.float32)
        out = np.zeros_like(field)
        self.lib.ref_advect_scalar(self.h, ptr(self.coords), self.n, ptr(vel), ptr(field), ptr(out), dt, inv_dx)
        return out

    def divergence(self, vel, inv_dx):
        vel = np.ascontiguousarray(vel, dtype=np.float32)
        out = np.zeros(self.n, np.float32)
        self.lib.ref_divergence(self.h, ptr(self.coords), self.n, ptr(vel), ptr(out), inv_dx)
        return out

    def rbgs(self, div, p, dx, iterations, omega):
        p = np.ascontiguousarray(p, dtype=np.float32).copy()
        div = np.ascontiguousarray(div, dtype=np.float32)
        self.lib.ref_rbgs(self.h, ptr(self.coords), self.n, ptr(div), ptr(p), dx, iterations, omega)
        return p

    def subtract_gradient(self, vel, p, inv_dx):
        vel = np.ascontiguousarray(vel, dtype=np.float32)
        p = np.ascontiguousarray(p, dtype=np.float32)
        out = np.zeros_like(vel)
        self.lib.ref_subtract_gradient(self.h, ptr(self.coords), self.n, ptr(vel), ptr(p), ptr(out), inv_dx)
        return out

    def vorticity_confinement(self, vel, dt, inv_dx, scale, factor_scale):
        vel = np.ascontiguousarray(vel, dtype=np.float32)
        out = np.zeros_like(vel)
        self.lib.ref_vorticity_confinement(self.h, ptr(self.coords), self.n, ptr(vel), ptr(out), dt, inv_dx, scale,
                                           factor_scale)
        return out

    def project(self, vel, dx, iterations, omega):
        vel = np.ascontiguousarray(vel, dtype=np.float32).copy()
        div = np.zeros(self.n, np.float32)
        p = np.zeros(self.n, np.float32)
        self.lib.ref_project(self.h, ptr(self.coords), self.n, ptr(vel), ptr(div), ptr(p), dx, iterations, omega)
        return vel, div, p

    def plain_step(self, vel, scalars, dt, dx, iterations, omega, scratch=None):
        """In place on vel (N,3) and the scalar arrays; returns the scratch buffer for reuse."""
        if scratch is None:
            scratch = np.zeros(5 * self.n, np.float32)
        ptrs = (_p * max(1, len(scalars)))(*[a.ctypes.data for a in scalars])
        self.lib.ref_plain_step(self.h, ptr(self.coords), self.n, ptr(vel), ptrs, len(scalars), dt, dx, iterations,
                                omega, ptr(scratch))
        return scratch

    def hns_advance(self, velocity, scalars: dict, sources: dict, dx, iteration, dt, params: CombustionParams):
        vel = np.ascontiguousarray(velocity, dtype=np.float32).copy()
        sc = {k: np.ascontiguousarray(v, dtype=np.float32).copy() for k, v in scalars.items()}
        created = {k: np.zeros(self.n, np.float32) for k in ("fuel", "waste", "temperature", "flame") if k not in sc}
        src = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in sources.items()}
        f, keep = make_advance_fields(self.n, vel, sc, created, src)
        self.lib.ref_hns_advance(self.h, ptr(self.coords), ctypes.byref(f), dx, iteration, dt, ctypes.byref(params))
        del keep
        return vel, sc, created


    def hns_advance_model(self, velocity, scalars: dict, sources: dict, dx, iteration, dt, params: CombustionParams,
                          combustion: int = 0, burn_rate=0.0, heat_release=0.0, ignition_temp=0.0, omega=0.0):
        """The reference's HNS_Advance sequence with its `combustion` kernel in place of
        combustion_oxygen when combustion == 1 (the reference has no density buoyancy term);
        omega > 0 replaces the solves' 2/(1+sin(3.14159 dx))."""
        vel = np.ascontiguousarray(velocity, dtype=np.float32).copy()
        sc = {k: np.ascontiguousarray(v, dtype=np.float32).copy() for k, v in scalars.items()}
        created = {k: np.zeros(self.n, np.float32) for k in MODEL_FIELDS[combustion] if k not in sc}
        src = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in sources.items()}
        f, keep = make_advance_fields(self.n, vel, sc, created, src)
        self.lib.ref_hns_advance_model(self.h, ptr(self.coords), ctypes.byref(f), dx, iteration, dt, ctypes.byref(params),
                                       combustion, burn_rate, heat_release, ignition_temp, omega)
        del keep
        return vel, sc, created


def _cpu_has_avx2_fma() -> bool:
    if platform.machine() not in ("x86_64", "AMD64"):
        return False
    try:
        with open("/proc/cpuinfo") as fh:
            flags = fh.read()
        return " avx2" in flags and " fma" in flags
    except OSError:
        return False


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"
