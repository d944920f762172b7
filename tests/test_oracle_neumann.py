"""The oracle's zero-gradient (Neumann) walls on the CPU: the configurations' boundary, which
the reference does not have (it reads p = 0 outside the domain). Checked here:
  * the operator's null space: a pressure constant on a face-connected component has zero
    residual against a zero divergence;
  * the per-component mean removal: each component's divergence sums to zero (FP64), also on a
    grid of two separate components, while a Dirichlet solve needs no such step;
  * after the mean removal the singular system is consistent: red-black SOR drives the FP64
    residual below 1e-10 (a Dirichlet-0 solve reaches the same);
  * float and double agree."""
import numpy as np

from conftest import rel_err
from hnanosolver_b200 import synth


def _two_components():
    a = synth._box_leaves(24)
    b = synth._box_leaves(16) + np.array([48, 8, 8], np.int32)  # a gap of 24 voxels in x
    return synth.sort_leaves_nanovdb(np.concatenate([a, b]))


def test_constant_pressure_is_in_the_null_space(oracle):
    origins = synth.spheres_topology(48, 2, 8.0, 14.0, 5)
    t = oracle.topo(origins)
    n = 512 * len(origins)
    p = np.full(n, 3.25, np.float64)
    r2, b2 = t.residual_neumann(np.zeros(n), p, 0.1)
    assert r2 == 0.0 and b2 == 0.0
    r2d, _ = t.residual(np.zeros(n), p, 0.1)  # Dirichlet-0: a constant is not in the null space
    assert r2d > 0.0


def test_mean_removed_per_component(oracle):
    origins = _two_components()
    t = oracle.topo(origins)
    n = 512 * len(origins)
    rng = np.random.default_rng(1)
    div = rng.standard_normal(n) + 5.0
    out = t.remove_mean(div)
    coords = synth.leaf_dense_coords(origins)
    first = coords[:, 0] < 32
    assert first.sum() == 512 * 27 and (~first).sum() == 512 * 8
    assert abs(out[first].sum()) < 1e-8 * n and abs(out[~first].sum()) < 1e-8 * n
    np.testing.assert_allclose(out[first], div[first] - div[first].mean(), atol=1e-12)
    np.testing.assert_allclose(out[~first], div[~first] - div[~first].mean(), atol=1e-12)


def test_neumann_solve_converges_after_mean_removal(oracle):
    origins = _two_components()
    t = oracle.topo(origins)
    dens, vel = synth.smoothed_fields(origins, seed=2, box_passes=2)
    v = vel.astype(np.float64) * 4.0
    div = t.divergence(v, 10.0)
    assert abs(div.sum()) > 1e-6  # the raw divergence is not compatible
    b = t.remove_mean(div)
    p = t.rbgs_neumann(b, np.zeros_like(b), 0.1, 600, 1.8)
    r2, b2 = t.residual_neumann(b, p, 0.1)
    assert np.sqrt(r2 / b2) < 1e-10
    # Without the mean removal the same iterations stall.
    p2 = t.rbgs_neumann(div, np.zeros_like(div), 0.1, 600, 1.8)
    r2s, b2s = t.residual_neumann(div, p2, 0.1)
    assert np.sqrt(r2s / b2s) > 1e-3


def test_neumann_projection_float_matches_double(oracle):
    origins = synth.topology("box64")
    t = oracle.topo(origins)
    dens, vel = synth.smoothed_fields(origins, seed=0, box_passes=3)
    v32, d32, p32 = t.project_neumann(vel, np.float32(0.1), 40, np.float32(1.0))
    v64, d64, p64 = t.project_neumann(vel.astype(np.float64), 0.1, 40, 1.0)
    assert rel_err(v32, v64) < 1e-5
    assert rel_err(p32, p64) < 1e-4
    # The walls change the result against the reference's Dirichlet-0 projection.
    vd, _, _ = t.project(vel, np.float32(0.1), 40, np.float32(1.0))
    assert rel_err(v32, vd) > 1e-3
