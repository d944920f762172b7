"""Seeded synthetic sparse grids and fields for the solver's workloads.

No public dataset is involved: these generators are the whole workload. Every topology
is a set of 8^3 leaves in NanoVDB leaf order (the order a ValueOnIndex grid assigns its
value offsets in, externals/nanovdb/tools/cuda/PointsToGrid.cuh:596-651), stored
leaf-dense: leaf i owns slots [512 i, 512 i + 512) and slot 512 i + n is the voxel at
origin + ((n>>6)&7, (n>>3)&7, n&7) (src/Utils/GridBuilder.hpp:164-174).

Workloads (seed 0 unless stated):
  box64      64^3 box, 512 leaves, 262,144 voxels (the CPU-runnable single step)
  plume256   256^3 box, leaves inside 8 seeded spheres of radius 20-60
  shell512   512^3 box, leaves within 16 voxels (plus the leaf half-diagonal) of a seeded
             radius-200 sphere: about 23M voxels
  box128     128^3 box, 4096 leaves, 2,097,152 voxels (the differentiable rollout)
  fire512    512^3 box, leaves inside 32 seeded spheres of radius 15-60 (a mid-size fire)
  fire1024   1024^3 box, leaves inside 32 seeded spheres of radius 30-120

fire_state() adds the fire workloads' fields and their sphere source (fuel and heat).
"""
from __future__ import annotations

import math

import numpy as np

LEAF_HALF_DIAGONAL = 4.0 * math.sqrt(3.0)


def local_offsets() -> np.ndarray:
    """(512, 3) local voxel coordinates of leaf slots, x-major (NanoVDB CoordToOffset)."""
    n = np.arange(512)
    return np.stack([(n >> 6) & 7, (n >> 3) & 7, n & 7], axis=1).astype(np.int32)


def leaf_dense_coords(origins: np.ndarray) -> np.ndarray:
    """(512 L, 3) int32 coordinates of every slot."""
    origins = np.asarray(origins, dtype=np.int32).reshape(-1, 3)
    return (origins[:, None, :] + local_offsets()[None]).reshape(-1, 3).astype(np.int32)


def sort_leaves_nanovdb(origins: np.ndarray) -> np.ndarray:
    """Leaf origins sorted into NanoVDB leaf order: 4096^3 root tiles in signed (x,y,z)
    order, then the upper node's 32^3 child index, then the lower node's 16^3 child index."""
    o = np.asarray(origins, dtype=np.int64).reshape(-1, 3)
    keys = []
    for d in (2, 1, 0):
        keys.append((o[:, d] >> 3) & 15)
    for d in (2, 1, 0):
        keys.append((o[:, d] >> 7) & 31)
    for d in (2, 1, 0):
        keys.append(o[:, d] >> 12)
    order = np.lexsort(keys)
    return np.ascontiguousarray(o[order].astype(np.int32))


def _box_leaves(extent: int) -> np.ndarray:
    r = np.arange(0, extent, 8)
    g = np.stack(np.meshgrid(r, r, r, indexing="ij"), axis=-1).reshape(-1, 3)
    return g.astype(np.int32)


def _leaf_centers(extent: int) -> np.ndarray:
    return _box_leaves(extent).astype(np.float64) + 3.5


def spheres(extent: int, count: int, rmin: float, rmax: float, seed: int):
    """The seeded spheres of spheres_topology: (centres (count, 3), radii (count,)), radius
    U(rmin, rmax), centre U(r, extent - r) per axis."""
    rng = np.random.default_rng(seed)
    radii = rng.uniform(rmin, rmax, size=count)
    centers = np.stack([rng.uniform(r, extent - r, size=3) for r in radii])
    return centers, radii


def spheres_topology(extent: int, count: int, rmin: float, rmax: float, seed: int) -> np.ndarray:
    """Leaves of an extent^3 box whose centre lies within r + half-diagonal of one of
    `count` seeded spheres (radius U(rmin, rmax), centre U(r, extent - r))."""
    centers, radii = spheres(extent, count, rmin, rmax, seed)
    leaves = _box_leaves(extent)
    lc = leaves.astype(np.float64) + 3.5
    keep = np.zeros(len(leaves), dtype=bool)
    for c, r in zip(centers, radii):
        keep |= np.linalg.norm(lc - c, axis=1) <= r + LEAF_HALF_DIAGONAL
    return sort_leaves_nanovdb(leaves[keep])


def shell_topology(extent: int = 512, radius: float = 200.0, band: float = 16.0, seed: int = 0) -> np.ndarray:
    """Leaves whose centre is within band + half-diagonal of a sphere of the given radius;
    the centre is the box centre jittered by a seeded U(-4, 4) per axis."""
    rng = np.random.default_rng(seed)
    center = np.full(3, extent / 2.0) + rng.uniform(-4.0, 4.0, size=3)
    leaves = _box_leaves(extent)
    d = np.linalg.norm(leaves.astype(np.float64) + 3.5 - center, axis=1)
    keep = np.abs(d - radius) <= band + LEAF_HALF_DIAGONAL
    return sort_leaves_nanovdb(leaves[keep])


# The sphere sets of the fire workloads: (extent, count, rmin, rmax).
SPHERE_WORKLOADS = {"plume256": (256, 8, 20.0, 60.0), "fire512": (512, 32, 15.0, 60.0),
                    "fire1024": (1024, 32, 30.0, 120.0)}


def topology(name: str, seed: int = 0) -> np.ndarray:
    if name == "box64":
        return sort_leaves_nanovdb(_box_leaves(64))
    if name == "box128":
        return sort_leaves_nanovdb(_box_leaves(128))
    if name == "plume256":
        return spheres_topology(256, 8, 20.0, 60.0, seed)
    if name == "shell512":
        return shell_topology(512, 200.0, 16.0, seed)
    if name in SPHERE_WORKLOADS:
        return spheres_topology(*SPHERE_WORKLOADS[name], seed)
    raise ValueError(f"unknown workload {name!r}")


# ---- fields ------------------------------------------------------------------------------

def value_noise(coords: np.ndarray, seed: int = 0, lattice: int = 8) -> np.ndarray:
    """Seeded value noise in [0, 1]: uniform lattice values every `lattice` voxels,
    trilinearly interpolated at the voxel coordinates."""
    c = np.asarray(coords, dtype=np.int64)
    lo = c.min(axis=0)
    q = (c - lo).astype(np.float64) / lattice
    i0 = np.floor(q).astype(np.int64)
    t = (q - i0).astype(np.float32)
    shape = tuple(int(s) + 2 for s in i0.max(axis=0))
    rng = np.random.default_rng(seed)
    lat = rng.random(shape, dtype=np.float32)
    out = np.zeros(len(c), dtype=np.float32)
    for a in (0, 1):
        wa = t[:, 0] if a else 1.0 - t[:, 0]
        for b in (0, 1):
            wb = t[:, 1] if b else 1.0 - t[:, 1]
            for cc in (0, 1):
                wc = t[:, 2] if cc else 1.0 - t[:, 2]
                out += wa * wb * wc * lat[i0[:, 0] + a, i0[:, 1] + b, i0[:, 2] + cc]
    return out


def box_filter(field: np.ndarray, coords: np.ndarray, times: int = 1) -> np.ndarray:
    """3x3x3 mean over the domain's voxels (out-of-domain samples excluded), `times` times.
    field: (N,) or (N, k), slots in the order of `coords`."""
    c = np.asarray(coords, dtype=np.int64)
    lo = c.min(axis=0) - 1
    dims = tuple(int(v) for v in (c.max(axis=0) - lo + 2))
    idx = tuple((c - lo).T)
    f = np.asarray(field, dtype=np.float32)
    squeeze = f.ndim == 1
    if squeeze:
        f = f[:, None]
    mask = np.zeros(dims, dtype=np.float32)
    mask[idx] = 1.0

    def box3(a):
        for ax in range(3):
            a = a + np.roll(a, 1, axis=ax) + np.roll(a, -1, axis=ax)
        return a

    count = box3(mask)
    out = np.empty_like(f)
    for k in range(f.shape[1]):
        g = np.zeros(dims, dtype=np.float32)
        g[idx] = f[:, k]
        for _ in range(times):
            g = box3(g) * mask
            g[idx] /= count[idx]
        out[:, k] = g[idx]
    return out[:, 0] if squeeze else out


def smoothed_fields(origins: np.ndarray, seed: int = 0, box_passes: int = 3):
    """Density = value noise in [0,1] box-filtered `box_passes` times; velocity = per-voxel
    U(-1,1)^3 box-filtered `box_passes` times (interleaved x,y,z, shape (N, 3))."""
    coords = leaf_dense_coords(origins)
    dens = box_filter(value_noise(coords, seed), coords, box_passes)
    rng = np.random.default_rng(seed + 1000)
    vel = rng.uniform(-1.0, 1.0, size=(len(coords), 3)).astype(np.float32)
    vel = box_filter(vel, coords, box_passes)
    return np.ascontiguousarray(dens, dtype=np.float32), np.ascontiguousarray(vel, dtype=np.float32)


def value_noise_leaves(origins: np.ndarray, seed: int = 0) -> np.ndarray:
    """value_noise(leaf_dense_coords(origins), seed) with the 8-voxel lattice, computed per
    leaf: every leaf lies in one lattice cell, so its 512 values are a fixed 512x8 weight
    matrix applied to the cell's 8 corner values."""
    o = np.asarray(origins, dtype=np.int64).reshape(-1, 3)
    lo = o.min(axis=0)
    cell = (o - lo) // 8
    shape = tuple(int(v) + 2 for v in cell.max(axis=0))
    rng = np.random.default_rng(seed)
    lat = rng.random(shape, dtype=np.float32)
    t = local_offsets().astype(np.float32) / 8.0
    w = np.empty((512, 8), dtype=np.float32)
    corners = np.empty((len(o), 8), dtype=np.float32)
    q = 0
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                w[:, q] = (t[:, 0] if a else 1 - t[:, 0]) * (t[:, 1] if b else 1 - t[:, 1]) * (t[:, 2] if c else 1 - t[:, 2])
                corners[:, q] = lat[cell[:, 0] + a, cell[:, 1] + b, cell[:, 2] + c]
                q += 1
    return (corners @ w.T).reshape(-1)


def noise_fields(origins: np.ndarray, seed: int = 0):
    """Cheap smooth fields for the large workloads: density = value noise in [0, 1]; each
    velocity component = 2 * (independent value noise) - 1. Shapes (N,) and (N, 3)."""
    dens = value_noise_leaves(origins, seed)
    vel = np.stack([2.0 * value_noise_leaves(origins, seed + 1 + k) - 1.0 for k in range(3)], axis=1)
    return np.ascontiguousarray(dens, dtype=np.float32), np.ascontiguousarray(vel, dtype=np.float32)


def sphere_mask(origins: np.ndarray, centre, radius: float) -> np.ndarray:
    """float32 per slot: 1 where the voxel lies within `radius` voxels of `centre`, else 0."""
    c = leaf_dense_coords(origins).astype(np.float64)
    return (np.linalg.norm(c - np.asarray(centre, dtype=np.float64), axis=1) <= radius).astype(np.float32)


def fire_state(name: str, seed: int = 0, source_radius: float = 10.0, fuel_rate: float = 1.0,
               temperature_rate: float = 2.0):
    """Initial state and sources of a fire workload (plume256, fire1024): velocity and density
    as noise_fields; temperature, fuel and flame zero; the sources src_fuel = fuel_rate and
    src_temperature = temperature_rate inside a sphere of source_radius voxels at the centre of
    the workload's first sphere, zero elsewhere. Returns (origins, fields, sources): fields
    maps velocity (N, 3) and density, temperature, fuel, flame (N,); sources maps src_fuel and
    src_temperature (N,). All float32."""
    extent, count, rmin, rmax = SPHERE_WORKLOADS[name]
    origins = topology(name, seed)
    centers, _ = spheres(extent, count, rmin, rmax, seed)
    dens, vel = noise_fields(origins, seed)
    n = len(dens)
    mask = sphere_mask(origins, centers[0], source_radius)
    fields = {"velocity": vel, "density": dens, "temperature": np.zeros(n, np.float32),
              "fuel": np.zeros(n, np.float32), "flame": np.zeros(n, np.float32)}
    sources = {"src_fuel": mask * np.float32(fuel_rate), "src_temperature": mask * np.float32(temperature_rate)}
    return origins, fields, sources
