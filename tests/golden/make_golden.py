"""Generates tests/golden/*.npz from the reference's own kernels.

Run where the reference checkout exists (it builds oracle/_ref from src/Cuda/Kernel.cu):
    python tests/golden/make_golden.py
The fixtures pin the CPU oracle (tests/test_oracle.py) and, through it, the CUDA kernels.
Inputs are seeded synthetic fields on small sparse grids; every output array is what the
reference's kernel, run as host C++, wrote for those inputs.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hnanosolver_b200 import synth  # noqa: E402
from oracle import binding  # noqa: E402


def golden_topology() -> np.ndarray:
    """Ten leaves on both sides of zero and across a 128-voxel lower-node boundary."""
    o = np.array([[0, 0, 0], [8, 0, 0], [0, 8, 0], [0, 0, 8], [-8, 0, 0], [-8, -8, 0], [0, -8, -8],
                  [120, 0, 0], [128, 0, 0], [-4096, 8, 0]], dtype=np.int32)
    return synth.sort_leaves_nanovdb(o)


def kernel_topology() -> np.ndarray:
    """A 3x3x2 block of leaves with two removed (16 leaves, 8192 voxels), with negative
    coordinates, so that domain walls and out-of-domain taps are exercised."""
    o = np.array([[x, y, z] for x in (-8, 0, 8) for y in (-8, 0, 8) for z in (0, 8)], dtype=np.int32)
    keep = ~(((o[:, 0] == 8) & (o[:, 1] == 8) & (o[:, 2] == 8)) | ((o[:, 0] == -8) & (o[:, 1] == 0) & (o[:, 2] == 0)))
    return synth.sort_leaves_nanovdb(o[keep])


def main() -> None:
    binding.build(ref=True)
    ref = binding.RefOracle(binding.REF_SO)

    # --- topology: leaf order and ValueOnIndex offsets ---
    origins = golden_topology()
    coords = synth.leaf_dense_coords(origins)
    rng = np.random.default_rng(0)
    shuffled = coords.reshape(-1, 512, 3)[rng.permutation(len(origins))].reshape(-1, 3)
    g = ref.grid(shuffled)  # the grid sorts leaves itself
    q = np.concatenate([coords[rng.choice(len(coords), 2000, replace=False)],
                        rng.integers(-4200, 300, size=(2000, 3)).astype(np.int32),
                        np.array([[7, 7, 7], [8, 0, 0], [-1, -1, -1], [-9, 0, 0], [127, 0, 0], [136, 0, 0]], np.int32)])
    np.savez_compressed(os.path.join(HERE, "topology.npz"), input_leaf_origins_shuffled=shuffled.reshape(-1, 512, 3)[:, 0],
                        leaf_origins=g.leaf_origins(), value_count=np.array(g.value_count()), query=q,
                        offsets=g.offsets(q))

    # --- kernels ---
    origins = kernel_topology()
    coords = synth.leaf_dense_coords(origins)
    g = ref.grid(coords)
    assert np.array_equal(g.leaf_origins(), origins)
    dens, vel = synth.smoothed_fields(origins, seed=7, box_passes=2)
    vel = (vel * 6.0).astype(np.float32)  # displacements of about a voxel at dt/dx = 1
    temp = (dens * 1.5).astype(np.float32)
    dt, dx = 0.1, 0.1
    inv = 1.0 / dx
    out = dict(leaf_origins=origins, density=dens, velocity=vel, temperature=temp, dt=np.float32(dt), dx=np.float32(dx))
    out["advect_vector"] = g.advect_vector(vel, dt, inv)
    a = g.advect_scalars(vel, [dens, temp], dt, inv)
    out["advect_scalars_density"], out["advect_scalars_temperature"] = a
    out["advect_scalar"] = g.advect_scalar(vel, dens, dt, inv)
    div = g.divergence(vel, inv)
    out["divergence"] = div
    out["rbgs_12_omega1p5"] = g.rbgs(div, np.zeros_like(div), dx, 12, 1.5)
    out["subtract_gradient"] = g.subtract_gradient(vel, out["rbgs_12_omega1p5"], inv)
    out["vorticity_fs1"] = g.vorticity_confinement(vel, dt, inv, 0.3, 1.0)
    out["vorticity_fs0p5"] = g.vorticity_confinement(vel, dt, inv, 1.0, 0.5)
    pv, pd, pp = g.project(vel, dx, 15, -1.0)
    out["project_velocity"], out["project_divergence"], out["project_pressure"] = pv, pd, pp

    # --- one HNS_Advance call, 2 substeps, Houdini defaults with a lower ambient ---
    params = binding.CombustionParams.houdini_defaults()
    params.ambientTemp = 0.5
    params.substeps = 2
    params.factorScale = 1.0
    n = len(coords)
    src = {
        "src_vel": rng.uniform(-1, 1, (n, 3)).astype(np.float32),
        "src_temperature": (rng.random(n) > 0.8).astype(np.float32) * 2.0,
        "src_fuel": (rng.random(n) > 0.8).astype(np.float32),
        "src_density": (rng.random(n) > 0.9).astype(np.float32),
    }
    scal = {"density": dens, "temperature": temp}
    v1, s1, c1 = g.hns_advance(vel, scal, src, dx, 8, 0.1, params)
    out["advance_params"] = np.frombuffer(bytes(params), dtype=np.uint8)
    out["advance_iterations"] = np.int32(8)
    for k, v in src.items():
        out["advance_" + k] = v
    out["advance_velocity"] = v1
    for k, v in list(s1.items()) + list(c1.items()):
        out["advance_out_" + k] = v
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), **out)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
