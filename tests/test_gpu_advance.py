"""The all-in-one step (hns_advance, HNS_Advance semantics) against the oracle's
restatement of HNS_Advance (itself pinned to the reference's kernels by the golden
vectors), over several calls with substeps, sources, created fields and both branches of
the disturbance re-solve."""
import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _params(**kw):
    from oracle.binding import CombustionParams as OP

    from hnanosolver_b200.lib import CombustionParams

    p = OP.houdini_defaults()
    for k, v in kw.items():
        setattr(p, k, v)
    return p, CombustionParams.from_buffer_copy(bytes(p))


def test_advance_matches_golden(dev, golden_kernels):
    from hnanosolver_b200 import lib as hl

    g = golden_kernels
    _, params = _params()
    params = hl.CombustionParams.from_buffer_copy(g["advance_params"].tobytes())
    grid = hl.Grid(g["leaf_origins"], voxel_size=float(g["dx"]))
    grid.field_set("velocity", g["velocity"])
    grid.field_set("density", g["density"])
    grid.field_set("temperature", g["temperature"])
    for k in g:
        if k.startswith("advance_src_"):
            grid.field_set(k[len("advance_"):], g[k])
    grid.advance(int(g["advance_iterations"]), 0.1, params)
    assert rel_err(grid.field_get("velocity"), g["advance_velocity"]) <= TOL
    for name in ("density", "temperature", "fuel", "waste", "flame"):
        assert rel_err(grid.field_get(name), g["advance_out_" + name]) <= TOL, name
    assert np.all(grid.active_mask() == 1)
    grid.close()


@pytest.mark.parametrize("disturbance,substeps,xyz", [(1.0, 1, False), (0.0, 2, True), (1.0, 3, False)])
def test_advance_three_calls(dev, oracle, disturbance, substeps, xyz):
    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(80, 3, 8.0, 18.0, seed=4)
    dens, vel = synth.smoothed_fields(origins, seed=9, box_passes=2)
    vel = (vel * 5.0).astype(np.float32)
    n = len(dens)
    rng = np.random.default_rng(2)
    src = {"src_temperature": (rng.random(n) > 0.85).astype(np.float32) * 3.0,
           "src_fuel": (rng.random(n) > 0.85).astype(np.float32),
           "src_density": (rng.random(n) > 0.9).astype(np.float32)}
    if xyz:
        for c, a in zip("xyz", rng.uniform(-1, 1, (3, n)).astype(np.float32)):
            src["src_vel_" + c] = a
    else:
        src["src_vel"] = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    op, params = _params(ambientTemp=0.3, disturbanceEnable=disturbance, substeps=substeps, factorScale=1.0,
                         vorticityScale=0.7)
    grid = hl.Grid(origins, voxel_size=0.1)
    grid.field_set("velocity", vel)
    grid.field_set("density", dens)
    for k, a in src.items():
        grid.field_set(k, a)
    t = oracle.topo(origins)
    ov, state = vel, {"density": dens}
    for call in range(3):
        grid.advance(12, 1.0 / 24.0, params)
        ov, sc, cr = t.hns_advance(ov, state, src, 0.1, 12, 1.0 / 24.0, op)
        state = {**sc, **cr}  # fields created in this call persist and are advected next call
        assert rel_err(grid.field_get("velocity"), ov) <= TOL, call
        for name, ref in state.items():
            assert rel_err(grid.field_get(name), ref) <= TOL, (call, name)
    assert set(grid.field_names()) >= {"velocity", "density", "fuel", "waste", "temperature", "flame"}
    grid.close()


def test_advance_with_collider_matches_oracle(dev, oracle):
    """HNS_Advance with a "collision_sdf" field (a sphere collider, SDF in world units) over two
    calls of two substeps: the velocity, the scalars and the created fields against the oracle,
    whose collision branches are pinned to the reference's own kernels; the velocity inside the
    collider is 0."""
    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(48, 2, 8.0, 14.0, seed=3)
    dens, vel = synth.smoothed_fields(origins, seed=4, box_passes=1)
    vel = (vel * 20.0).astype(np.float32)
    dx = 0.1
    coords = synth.leaf_dense_coords(origins).astype(np.float64)
    centre = coords[len(coords) // 3] + 0.37
    sdf = ((np.linalg.norm(coords - centre, axis=1) - 5.0) * dx).astype(np.float32)
    p_or, params = _params(substeps=2, disturbanceEnable=0.0)
    grid = hl.Grid(origins, voxel_size=dx)
    grid.field_set("velocity", vel)
    grid.field_set("density", dens)
    grid.field_set("collision_sdf", sdf)
    t = oracle.topo(origins)
    v_ref, sc_ref = vel.copy(), {"density": dens.copy()}
    for _ in range(2):
        grid.advance(20, 0.1, params)
        v_ref, sc, cr = t.hns_advance(v_ref, sc_ref, {"collision_sdf": sdf}, dx, 20, 0.1, p_or)
        sc_ref = {**sc, **cr}
    got_v = grid.field_get("velocity")
    assert rel_err(got_v, v_ref) <= TOL
    for name, ref in sc_ref.items():
        assert rel_err(grid.field_get(name), ref) <= TOL, name
    assert np.all(got_v[sdf < 0] == 0.0)
    assert np.allclose(grid.field_get("collision_sdf"), sdf)  # the collider is not advected
    grid.close()


def test_field_transfers_through_staging(dev):
    """Host field uploads and downloads go through the pinned staging chunks (64 MB): a
    278 MB velocity field (several chunks and a partial one) and a scalar field round-trip
    exactly, and a small field (a direct copy) too."""
    from hnanosolver_b200 import lib as hl

    origins = synth.topology("shell512")
    g = hl.Grid(origins, voxel_size=0.1)
    n = g.num_voxels
    rng = np.random.default_rng(5)
    vel = rng.standard_normal((n, 3)).astype(np.float32)
    den = rng.random(n, dtype=np.float32)
    g.field_set("velocity", vel)
    g.field_set("density", den)
    assert np.array_equal(g.field_get("velocity"), vel)
    assert np.array_equal(g.field_get("density"), den)
    g.close()
    small = hl.Grid(synth.topology("box64"), voxel_size=0.1)
    d = rng.random(small.num_voxels, dtype=np.float32)
    small.field_set("density", d)
    assert np.array_equal(small.field_get("density"), d)
    small.close()
