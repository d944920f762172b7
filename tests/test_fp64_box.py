"""The FP64 box restatement of the plain step (fp64_box, the checker of the rollout adjoint
tests) against the FP64 oracle: several steps on a fully active box with traces that leave
the box, on the CPU."""
import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")


def test_fp64_box_step_matches_oracle(oracle):
    from fp64_box import Box, from_dense, to_dense

    origins = synth.sort_leaves_nanovdb(synth._box_leaves(24))
    dens, vel = synth.smoothed_fields(origins, seed=2, box_passes=3)
    vel = (vel * 8.0).astype(np.float64)  # about half a voxel per step: traces cross cells and leave the box
    dens = dens.astype(np.float64)
    coords = synth.leaf_dense_coords(origins)
    lo = coords.min(axis=0)
    dx, dt, iters, omega = 0.1, 0.1, 20, 1.3
    box = Box((24, 24, 24), lo, dx, torch.device("cpu"))
    tv, td = to_dense(vel, coords, lo, box.shape, "cpu"), to_dense(dens, coords, lo, box.shape, "cpu")
    t = oracle.topo(origins)
    v_ref, d_ref = vel.copy(), dens.copy()
    for _ in range(3):
        tv, (td,), _ = box.step(tv, [td], dt, iters, omega)
        d_ref = t.advect_scalar(v_ref, d_ref, dt, 1.0 / dx)
        v_ref, _, _ = t.project(t.advect_vector(v_ref, dt, 1.0 / dx), dx, iters, omega)
    assert rel_err(from_dense(td[0], coords, lo), d_ref) <= 1e-12
    assert rel_err(from_dense(tv[0], coords, lo), v_ref) <= 1e-12


def test_fp64_box_batch_is_independent():
    """A batch of states steps as the same states one at a time."""
    from fp64_box import Box

    box = Box((16, 16, 16), (0, 0, 0), 0.1, torch.device("cpu"))
    g = torch.Generator().manual_seed(0)
    v = torch.rand((3, 3, 16, 16, 16), generator=g, dtype=torch.float64) - 0.5
    d = torch.rand((3, 16, 16, 16), generator=g, dtype=torch.float64)
    vb, (db,), _ = box.step(v, [d], 0.1, 10, 1.0)
    for b in range(3):
        v1, (d1,), _ = box.step(v[b:b + 1], [d[b:b + 1]], 0.1, 10, 1.0)
        assert torch.equal(v1[0], vb[b]) and torch.equal(d1[0], db[b])


def test_fp64_box_frozen_replay():
    """Replaying a step's recorded decisions (trace cells, clamp selections) reproduces it
    exactly, and a small perturbation through the frozen decisions moves the result as little
    as through the free ones."""
    from fp64_box import Box

    box = Box((16, 16, 16), (0, 0, 0), 0.1, torch.device("cpu"))
    g = torch.Generator().manual_seed(1)
    v = (torch.rand((1, 3, 16, 16, 16), generator=g, dtype=torch.float64) - 0.5) * 4.0
    d = torch.rand((1, 16, 16, 16), generator=g, dtype=torch.float64)
    v1, (d1,), dec = box.step(v, [d], 0.1, 10, 1.0)
    v2, (d2,), _ = box.step(v, [d], 0.1, 10, 1.0, frozen=dec)
    assert torch.equal(v1, v2) and torch.equal(d1, d2)
    vp = v.clone()
    vp[0, 1, 5, 6, 7] += 1e-9
    va, (da,), _ = box.step(vp, [d], 0.1, 10, 1.0)
    vb, (db,), _ = box.step(vp, [d], 0.1, 10, 1.0, frozen=dec)
    assert float((da - db).abs().max()) <= 1e-14 and float((va - vb).abs().max()) <= 1e-14


def _sparse_box(origins, dx):
    from fp64_box import Box, active_mask

    coords = synth.leaf_dense_coords(origins)
    lo = coords.min(axis=0)
    shape = tuple(int(v) for v in coords.max(axis=0) - lo + 1)
    dev = torch.device("cpu")
    return Box(shape, lo, dx, dev, active=active_mask(coords, lo, shape, dev)), coords, lo


def test_fp64_sparse_step_matches_oracle(oracle):
    """A sparse grid (three spheres of leaves, traces leaving the grid) held as the box's mask:
    advection, divergence, red-black SOR and gradient against the FP64 oracle."""
    from fp64_box import from_dense, to_dense

    origins = synth.spheres_topology(48, 3, 6.0, 12.0, seed=4)
    dens, vel = synth.smoothed_fields(origins, seed=3, box_passes=2)
    vel = (vel * 8.0).astype(np.float64)
    dens = dens.astype(np.float64)
    dx, dt, iters, omega = 0.1, 0.1, 15, 1.4
    box, coords, lo = _sparse_box(origins, dx)
    assert int(box.active.sum()) == len(dens) < box.active.numel()
    tv, td = to_dense(vel, coords, lo, box.shape, "cpu"), to_dense(dens, coords, lo, box.shape, "cpu")
    t = oracle.topo(origins)
    v_ref, d_ref = vel.copy(), dens.copy()
    for _ in range(2):
        tv, (td,), _ = box.step(tv, [td], dt, iters, omega)
        d_ref = t.advect_scalar(v_ref, d_ref, dt, 1.0 / dx)
        v_ref, _, _ = t.project(t.advect_vector(v_ref, dt, 1.0 / dx), dx, iters, omega)
    assert rel_err(from_dense(td[0], coords, lo), d_ref) <= 1e-12
    assert rel_err(from_dense(tv[0], coords, lo), v_ref) <= 1e-12
    # Nothing leaks onto inactive voxels.
    assert float(td[0][~box.active].abs().max()) == 0.0 and float(tv[0][:, ~box.active].abs().max()) == 0.0


def test_fp64_exact_solve_residual(oracle):
    """solve_exact reaches its FP64 residual as the oracle measures it (p = 0 outside the grid),
    and red-black SOR approaches its solution."""
    from fp64_box import from_dense, to_dense

    origins = synth.spheres_topology(48, 3, 6.0, 12.0, seed=4)
    _, vel = synth.smoothed_fields(origins, seed=5, box_passes=2)
    dx = 0.1
    box, coords, lo = _sparse_box(origins, dx)
    t = oracle.topo(origins)
    div = t.divergence(vel.astype(np.float64), 1.0 / dx)
    p, it, res = box.solve_exact(to_dense(div, coords, lo, box.shape, "cpu")[0], tol=1e-12)
    assert res <= 1e-12 and it > 0
    r2, b2 = t.residual(div, from_dense(p, coords, lo), dx)
    assert np.sqrt(r2 / b2) <= 1e-11
    p_sor = t.rbgs(div, np.zeros_like(div), dx, 400, 1.8)
    assert rel_err(p_sor, from_dense(p, coords, lo)) <= 1e-6
