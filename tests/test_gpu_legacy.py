"""The reference's own C++ entry points (include/hns_legacy.hpp), driven by a C++ program
the way the reference's SOPs call them, checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_err

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "tests", "legacy", "_build", "legacy_api_test")
TOL = 1e-5


def _load(d, name):
    path = os.path.join(d, name)
    if name.endswith(".i32"):
        return np.fromfile(path, np.int32).reshape(-1, 3)
    a = np.fromfile(path, np.float32)
    return a.reshape(-1, 3) if name.endswith(".v3") else a


@pytest.fixture(scope="module")
def run(tmp_path_factory):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(EXE):
        pytest.skip("legacy test program not built")
    d = str(tmp_path_factory.mktemp("legacy"))
    r = subprocess.run([EXE, d], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    return d


def test_sop_cook_two_frames(run, oracle):
    from hnanosolver_b200 import synth
    from oracle.binding import CombustionParams

    coords = _load(run, "in_coords.i32")
    origins = coords[::512].copy()
    assert np.array_equal(synth.sort_leaves_nanovdb(origins), origins)
    t = oracle.topo(origins)
    p = CombustionParams(expansionRate=0.1, temperatureRelease=0.5, buoyancyStrength=1.0, ambientTemp=0.4,
                         vorticityScale=0.5, factorScale=1.0, disturbanceEnable=1.0, substeps=2, gravity=1.0,
                         downloadVel=1)
    src = {"src_temperature": _load(run, "in_src_temperature.f32"), "src_fuel": _load(run, "in_src_fuel.f32"),
           "src_vel": _load(run, "in_src_vel.v3")}
    vel, state = _load(run, "in_velocity.v3"), {"density": _load(run, "in_density.f32"),
                                               "temperature": _load(run, "in_temperature.f32")}
    for _ in range(2):
        vel, sc, cr = t.hns_advance(vel, state, src, 0.1, 10, 1.0 / 24.0, p)
        state = {**sc, **cr}
    assert rel_err(_load(run, "advance_velocity.v3"), vel) <= TOL
    assert rel_err(_load(run, "advance_density.f32"), state["density"]) <= TOL
    assert rel_err(_load(run, "advance_temperature.f32"), state["temperature"]) <= TOL


def test_sop_operators(run, oracle):
    coords = _load(run, "in_coords.i32")
    t = oracle.topo(coords[::512].copy())
    vel, dens, temp = _load(run, "in_velocity.v3"), _load(run, "in_density.f32"), _load(run, "in_temperature.f32")
    div = t.divergence(vel, np.float32(1.0) / np.float32(0.1))
    assert rel_err(_load(run, "sopdiv_divergence.f32"), div) <= TOL
    inv = np.float32(1.0) / np.float32(0.1)
    # AdvectIndexGrid advects every float block, "divergence" included.
    assert rel_err(_load(run, "sop_divergence.f32"), t.advect_scalar(vel, div, 0.1, inv)) <= TOL
    assert rel_err(_load(run, "sop_density.f32"), t.advect_scalar(vel, dens, 0.1, inv)) <= TOL
    assert rel_err(_load(run, "sop_temperature.f32"), t.advect_scalar(vel, temp, 0.1, inv)) <= TOL
    v, _, _ = t.project(t.advect_vector(vel, 0.1, inv), 0.1, 20, -1.0)
    assert rel_err(_load(run, "sop_velocity.v3"), v) <= TOL
