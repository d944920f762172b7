"""The oracle's force models of the all-in-one step (hnso_hns_advance_model) on the CPU.

* The rate/heat burn (the reference's `combustion` kernel, src/Cuda/Kernel.cu:568-588) inside
  the HNS_Advance sequence: the oracle's restatement against the reference's own kernels,
  driven by oracle/ref_driver.cpp, over two calls with sources (<= 1e-5 relative).
* The buoyancy's density term, which the reference does not have: the oracle against a numpy
  restatement of v.y += (b_T - alpha density) dt, to the bit in float32; alpha = 0 is the
  reference's temperature_buoyancy.
* The float64 step against the float32 step (the FP64 oracle of the mixed-precision tests)."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

TOL = 1e-5


def _plume_case(seed=3):
    origins = synth.spheres_topology(64, 3, 8.0, 16.0, seed=seed)
    dens, vel = synth.smoothed_fields(origins, seed=seed, box_passes=1)
    n = len(dens)
    rng = np.random.default_rng(seed)
    centres, _ = synth.spheres(64, 3, 8.0, 16.0, seed)
    src = synth.sphere_mask(origins, centres[0], 5.0)
    fields = {"density": dens, "temperature": (rng.random(n, dtype=np.float32) * 1.5).astype(np.float32),
              "fuel": rng.random(n, dtype=np.float32) * (rng.random(n) < 0.5).astype(np.float32),
              "flame": np.zeros(n, np.float32)}
    sources = {"src_fuel": src * np.float32(1.0), "src_temperature": src * np.float32(2.0)}
    return origins, (vel * 4.0).astype(np.float32), fields, sources


def _params():
    from oracle.binding import CombustionParams

    p = CombustionParams.houdini_defaults()
    p.buoyancyStrength = 0.5
    p.ambientTemp = 0.0
    p.vorticityScale = 0.3
    p.factorScale = 1.0
    p.disturbanceEnable = 0.0
    p.gravity = 0.0
    return p


def test_rate_model_matches_reference_kernels(oracle, ref_oracle):
    from oracle.binding import ForceModel

    origins, vel, fields, sources = _plume_case()
    t = oracle.topo(origins)
    g = ref_oracle.grid(synth.leaf_dense_coords(origins))
    params = _params()
    model = ForceModel(combustion=1, burn_rate=0.5, heat_release=1.0, ignition_temp=0.0)
    v_o, s_o = vel, dict(fields)
    v_r, s_r = vel, dict(fields)
    for call in range(2):
        v_o, s_o, c_o = t.hns_advance_model(v_o, s_o, sources, 0.1, 25, 1.0 / 24.0, params, model)
        v_r, s_r, c_r = g.hns_advance_model(v_r, s_r, sources, 0.1, 25, 1.0 / 24.0, params, combustion=1,
                                            burn_rate=0.5, heat_release=1.0, ignition_temp=0.0)
        assert not c_o and not c_r  # fuel and temperature were given: nothing is created
        assert rel_err(v_o, v_r) <= TOL, call
        for k in s_o:
            assert rel_err(s_o[k], s_r[k]) <= TOL, (call, k)
    # The burn ran: fuel went down where it was positive and hot enough.
    burned = fields["fuel"] > 0
    assert burned.any()


def test_rate_model_creates_only_its_fields(oracle):
    from oracle.binding import ForceModel

    origins, vel, fields, sources = _plume_case(seed=4)
    t = oracle.topo(origins)
    model = ForceModel(combustion=1, burn_rate=0.5, heat_release=1.0, ignition_temp=0.0)
    _, _, created = t.hns_advance_model(vel, {"density": fields["density"]}, sources, 0.1, 10, 0.1, _params(), model)
    assert sorted(created) == ["fuel", "temperature"]
    _, _, created = t.hns_advance_model(vel, {"density": fields["density"]}, sources, 0.1, 10, 0.1, _params())
    assert sorted(created) == ["flame", "fuel", "temperature", "waste"]


def test_density_buoyancy_term(oracle):
    n = 4096
    rng = np.random.default_rng(7)
    vel = rng.uniform(-1, 1, size=(n, 3)).astype(np.float32)
    temp = rng.uniform(-0.5, 1.5, size=n).astype(np.float32)
    dens = rng.random(n, dtype=np.float32)
    out = np.zeros_like(vel)
    dt, amb, beta, alpha = np.float32(0.05), np.float32(0.25), np.float32(0.5), np.float32(0.1)
    lib = oracle.lib
    lib.hnso_buoyancy_density_f32.restype = None
    lib.hnso_buoyancy_density_f32.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 4 + [ctypes.c_float] * 4
    lib.hnso_buoyancy_density_f32(n, vel.ctypes.data, temp.ctypes.data, dens.ctypes.data, out.ctypes.data, dt, amb, beta,
                                  alpha)
    bt = np.where(temp > amb, np.maximum(np.float32(0), (temp - amb) * beta), np.float32(0)).astype(np.float32)
    fy = (bt - alpha * dens).astype(np.float32)
    want = vel.copy()
    want[:, 1] = (vel[:, 1] + fy * dt).astype(np.float32)
    assert np.array_equal(out, want)
    # alpha = 0: the reference's temperature_buoyancy.
    ref = np.zeros_like(vel)
    lib.hnso_temperature_buoyancy_f32.restype = None
    lib.hnso_temperature_buoyancy_f32.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 3 + [ctypes.c_float] * 3
    lib.hnso_temperature_buoyancy_f32(n, vel.ctypes.data, temp.ctypes.data, ref.ctypes.data, dt, amb, beta)
    lib.hnso_buoyancy_density_f32(n, vel.ctypes.data, temp.ctypes.data, dens.ctypes.data, out.ctypes.data, dt, amb, beta,
                                  np.float32(0))
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("combustion", [0, 1])
def test_fp64_model_close_to_fp32(oracle, combustion):
    from oracle.binding import ForceModel

    origins, vel, fields, sources = _plume_case(seed=5)
    t = oracle.topo(origins)
    model = ForceModel(combustion=combustion, burn_rate=0.5, heat_release=1.0, ignition_temp=0.0, density_buoyancy=0.1)
    params = _params()
    v32, s32, _ = t.hns_advance_model(vel, fields, sources, 0.1, 30, 1.0 / 24.0, params, model)
    v64, s64, _ = t.hns_advance_model(vel, fields, sources, 0.1, 30, 1.0 / 24.0, params, model, dtype=np.float64)
    assert v64.dtype == np.float64
    assert rel_err(v32, v64) < 1e-4
    for k in s32:
        assert rel_err(s32[k], s64[k]) < 1e-4, k
