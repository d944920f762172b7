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
