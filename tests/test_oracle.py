"""The CPU oracle against the reference: golden vectors made by the reference's own
kernels (tests/golden/make_golden.py), the reference's known-answer tests restated on the
leaf-dense layout, and, where oracle/_ref is built, the reference kernels run live."""
import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

# The float oracle runs the reference's arithmetic in the reference's order; against the
# host-compiled reference it agrees to the last bit. 1e-6 leaves room for a compiler that
# contracts differently.
TOL = 1e-6


def test_topology_order_and_offsets(oracle, golden_topology):
    g = golden_topology
    srt = oracle.sort_leaves(g["input_leaf_origins_shuffled"])
    assert np.array_equal(srt, g["leaf_origins"])  # NanoVDB leaf order, bit-exact
    assert np.array_equal(synth.sort_leaves_nanovdb(g["input_leaf_origins_shuffled"]), g["leaf_origins"])
    t = oracle.topo(g["leaf_origins"])
    assert t.n + 1 == int(g["value_count"])
    assert np.array_equal(t.offsets(g["query"]), g["offsets"])  # ValueOnIndex offsets, bit-exact


def test_nanovdb_offset_kat(oracle):
    # externals/nanovdb/unittest/TestNanoVDB.cu:302-398: offsets count from 1, 0 is the
    # background, and offsetToGlobalCoord(CoordToOffset(ijk)) == ijk.
    t = oracle.topo(np.array([[0, 0, 0]], np.int32))
    assert list(t.offsets([[0, 0, 0], [0, 0, 1], [0, 0, 2], [0, 1, 0], [1, 0, 0], [8, 0, 0], [-1, 0, 0]])) == [
        1, 2, 3, 9, 65, 0, 0]
    c = t.coords()
    assert np.array_equal(t.offsets(c), np.arange(1, 513, dtype=np.uint64))


def _line_grids():
    """Tests/IndexGrid.cpp:157-282: density i at (i,0,0), velocity (i,i,i) at (0,i,0) for
    i < 15, on the leaf-dense layout of the domain's leaves."""
    origins = synth.sort_leaves_nanovdb(np.array([[0, 0, 0], [8, 0, 0], [0, 8, 0]], np.int32))
    coords = synth.leaf_dense_coords(origins)
    slot = {tuple(c): s for s, c in enumerate(coords)}
    dens = np.zeros(len(coords), np.float32)
    vel = np.zeros((len(coords), 3), np.float32)
    for i in range(15):
        dens[slot[(i, 0, 0)]] = i
        vel[slot[(0, i, 0)]] = (i, i, i)
    return origins, dens, vel


def test_sampler_kat(oracle):
    origins, dens, vel = _line_grids()
    t = oracle.topo(origins)
    # IndexSampler<float,0> exact reads (Tests/IndexGrid.cpp:278-281)
    pts = np.array([[i, 0, 0] for i in range(15)], np.float32)
    assert np.array_equal(t.sample_trilinear(dens, pts), np.arange(15, dtype=np.float32))
    # trilinear samples (Tests/IndexGrid.cpp:209-223)
    assert t.sample_trilinear(dens, [[0, 0, 0]])[0] == 0
    assert t.sample_trilinear(dens, [[1, 0, 0]])[0] == 1
    assert t.sample_trilinear(dens, [[1, 1, 0]])[0] == 0
    assert t.sample_trilinear(vel, [[1, 1, 0]])[0, 0] == 0
    assert t.sample_trilinear(vel, [[0, 1, 0]])[0, 0] == 1
    assert t.sample_trilinear(dens, [[0.5, 0, 0]])[0] == pytest.approx(0.5)
    assert t.sample_trilinear(dens, [[1.25, 0, 0]])[0] == pytest.approx(1.25)
    assert t.sample_trilinear(vel, [[0, 0.5, 0]])[0, 0] == pytest.approx(0.5)
    assert t.sample_trilinear(vel, [[0, 1.25, 0]])[0, 0] == pytest.approx(1.25)
    # out of the domain reads 0 (Tests/IndexGrid.cpp:212-213, 578-579)
    assert t.sample_trilinear(dens, [[-50, 3, 2]])[0] == 0


def test_layout_round_trip_kat(oracle):
    # Tests/IndexGrid.cpp:133-154: values doubled in the indexed arrays read back doubled.
    origins, dens, vel = _line_grids()
    t = oracle.topo(origins)
    d2, v2 = dens * 2, vel * 2
    assert t.sample_trilinear(d2, [[5, 0, 0]])[0] == 10
    assert t.sample_trilinear(d2, [[6, 0, 0]])[0] == 12
    assert t.sample_trilinear(v2, [[0, 5, 0]])[0, 0] == 10
    assert t.sample_trilinear(d2, [[5.5, 0, 0]])[0] == pytest.approx(11)
    assert t.sample_trilinear(v2, [[0, 5.5, 0]])[0, 0] == pytest.approx(11)


def test_kernels_against_golden(oracle, golden_kernels):
    g = golden_kernels
    t = oracle.topo(g["leaf_origins"])
    dt, dx = float(g["dt"]), float(g["dx"])
    inv = 1.0 / np.float32(dx)
    vel, dens, temp = g["velocity"], g["density"], g["temperature"]
    assert rel_err(t.advect_vector(vel, dt, inv), g["advect_vector"]) <= TOL
    a = t.advect_scalars(vel, [dens, temp], dt, inv)
    assert rel_err(a[0], g["advect_scalars_density"]) <= TOL
    assert rel_err(a[1], g["advect_scalars_temperature"]) <= TOL
    assert rel_err(t.advect_scalar(vel, dens, dt, inv), g["advect_scalar"]) <= TOL
    div = t.divergence(vel, inv)
    assert rel_err(div, g["divergence"]) <= TOL
    p = t.rbgs(div, np.zeros_like(div), dx, 12, 1.5)
    assert rel_err(p, g["rbgs_12_omega1p5"]) <= TOL
    assert rel_err(t.subtract_gradient(vel, g["rbgs_12_omega1p5"], inv), g["subtract_gradient"]) <= TOL
    assert rel_err(t.vorticity_confinement(vel, dt, inv, 0.3, 1.0), g["vorticity_fs1"]) <= TOL
    assert rel_err(t.vorticity_confinement(vel, dt, inv, 1.0, 0.5), g["vorticity_fs0p5"]) <= TOL
    pv, pd, pp = t.project(vel, dx, 15, -1.0)
    assert rel_err(pv, g["project_velocity"]) <= TOL
    assert rel_err(pd, g["project_divergence"]) <= TOL
    assert rel_err(pp, g["project_pressure"]) <= TOL


def test_factor_scale_truncation_gives_zero_force(oracle, golden_kernels):
    # int(0.5) == 0: the |omega| gradient is taken at the voxel itself (Kernel.cu:707-712).
    g = golden_kernels
    assert np.array_equal(g["vorticity_fs0p5"], g["velocity"])


def test_hns_advance_against_golden(oracle, golden_kernels):
    from oracle.binding import CombustionParams

    g = golden_kernels
    t = oracle.topo(g["leaf_origins"])
    params = CombustionParams.from_buffer_copy(g["advance_params"].tobytes())
    src = {k[len("advance_"):]: g[k] for k in g if k.startswith("advance_src_")}
    vel, sc, cr = t.hns_advance(g["velocity"], {"density": g["density"], "temperature": g["temperature"]}, src,
                                float(g["dx"]), int(g["advance_iterations"]), 0.1, params)
    assert rel_err(vel, g["advance_velocity"]) <= TOL
    for k, v in list(sc.items()) + list(cr.items()):
        assert rel_err(v, g["advance_out_" + k]) <= TOL, k


def test_fp64_oracle_close_to_fp32(oracle, golden_kernels):
    g = golden_kernels
    t = oracle.topo(g["leaf_origins"])
    v64 = g["velocity"].astype(np.float64)
    assert rel_err(t.advect_vector(v64, 0.1, 10.0), g["advect_vector"]) < 1e-5
    assert rel_err(t.divergence(v64, 10.0), g["divergence"]) < 1e-5


def test_oracle_matches_live_reference(oracle, ref_oracle):
    origins = synth.spheres_topology(64, 2, 6.0, 14.0, seed=5)
    dens, vel = synth.smoothed_fields(origins, seed=2, box_passes=1)
    vel = vel * 8.0
    t = oracle.topo(origins)
    g = ref_oracle.grid(synth.leaf_dense_coords(origins))
    assert np.array_equal(g.leaf_origins(), origins)
    assert rel_err(t.advect_vector(vel, 0.1, 10.0), g.advect_vector(vel, 0.1, 10.0)) <= TOL
    a, b = t.advect_scalars(vel, [dens], 0.1, 10.0)[0], g.advect_scalars(vel, [dens], 0.1, 10.0)[0]
    assert rel_err(a, b) <= TOL
    div = t.divergence(vel, 10.0)
    assert rel_err(t.rbgs(div, np.zeros_like(div), 0.1, 30, 1.7), g.rbgs(div, np.zeros_like(div), 0.1, 30, 1.7)) <= TOL


def collider_sdf(origins, centre, radius, dx):
    """Signed distance in world units to a sphere (centre and radius in voxels), per slot."""
    c = synth.leaf_dense_coords(origins).astype(np.float64)
    return ((np.linalg.norm(c - np.asarray(centre, dtype=np.float64), axis=1) - radius) * dx).astype(np.float32)


def test_advance_with_collision_matches_live_reference(oracle, ref_oracle):
    """HNS_Advance with a collider: the oracle's restatement of the collision branches
    (enforceCollisionBoundaries before the substeps and after each projection, the trace
    pull-backs and the near-wall blend of advect_vector / advect_scalars /
    subtractPressureGradient) against the reference's own kernels, two substeps."""
    from oracle.binding import CombustionParams

    origins = synth.spheres_topology(48, 2, 8.0, 14.0, seed=3)
    dens, vel = synth.smoothed_fields(origins, seed=4, box_passes=1)
    vel = (vel * 20.0).astype(np.float32)  # traces of up to a few voxels: some enter the collider
    dx = 0.1
    coords = synth.leaf_dense_coords(origins)
    centre = coords[len(coords) // 3].astype(np.float64) + 0.37
    sdf = collider_sdf(origins, centre, 5.0, dx)
    assert (sdf < 0).any() and ((sdf >= 0) & (sdf < 0.1)).any()
    params = CombustionParams.houdini_defaults()
    params.substeps = 2
    params.disturbanceEnable = 0.0
    t = oracle.topo(origins)
    g = ref_oracle.grid(coords)
    args = (vel, {"density": dens}, {"collision_sdf": sdf}, dx, 20, 0.1, params)
    v_o, s_o, c_o = t.hns_advance(*args)
    v_r, s_r, c_r = g.hns_advance(*args)
    assert rel_err(v_o, v_r) <= 1e-5
    assert rel_err(s_o["density"], s_r["density"]) <= 1e-5
    for k in c_o:
        assert rel_err(c_o[k], c_r[k]) <= 1e-5, k
    # The collider changed the result, and the velocity inside it is 0.
    v_n, _, _ = t.hns_advance(vel, {"density": dens}, {}, dx, 20, 0.1, params)
    assert rel_err(v_o, v_n) > 1e-3
    assert np.all(v_o[sdf < 0] == 0.0)
