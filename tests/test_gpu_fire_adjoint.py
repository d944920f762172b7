"""Adjoints of the fire step (hns_adjoint_advance, hns_adjoint_advance_mixed) through the C ABI,
as vector-Jacobian products against central finite differences (h = 1e-6) of the FP64 oracle's
step (hnso_hns_advance_model_f64), on a ragged sparse grid with traces that cross cells and
leave the domain: max |adjoint - finite difference| / max |finite difference| <= 1e-3 over
seeded entries of each input (velocity, density, temperature, fuel, and waste/flame for the
oxygen burn).

* FP32 step: `iterations` red-black iterations from p = 0 at HNS_Advance's omega, the same in
  the oracle; the rate/heat burn, the oxygen burn and no burn, with the density buoyancy.
* Mixed step: BF16/FP16 inputs (the oracle differentiates at their values), solves to 1e-5 taken
  as exact; the oracle's solves run to convergence (omega 1.9, 600 iterations)."""
import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FD_TOL = 1e-3
DX = 0.1
DT = 0.05


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _case(combustion):
    origins = synth.spheres_topology(40, 2, 8.0, 14.0, 3)
    dens, vel = synth.smoothed_fields(origins, seed=0, box_passes=3)
    coords = synth.leaf_dense_coords(origins)
    n = len(dens)
    centres, _ = synth.spheres(40, 2, 8.0, 14.0, 3)
    mask = synth.sphere_mask(origins, centres[0], 4.0)
    f = {"velocity": np.ascontiguousarray(vel * 8.0, dtype=np.float32), "density": dens,
         "temperature": (1.5 * synth.value_noise(coords, 41)).astype(np.float32),
         "fuel": (0.8 * synth.value_noise(coords, 42)).astype(np.float32),
         "flame": (0.5 * synth.value_noise(coords, 43)).astype(np.float32)}
    if combustion == 0:
        f["waste"] = (0.3 * synth.value_noise(coords, 44)).astype(np.float32)
    if combustion == 2:
        del f["fuel"]
    src = {"fuel": mask, "temperature": mask * np.float32(2.0)}
    return origins, n, f, src


def _params():
    from oracle.binding import CombustionParams as OP

    from hnanosolver_b200.lib import CombustionParams

    p = OP.houdini_defaults()
    p.buoyancyStrength, p.ambientTemp = 0.5, 0.3
    p.vorticityScale, p.factorScale = 0.3, 1.0
    p.disturbanceEnable, p.gravity = 0.0, 0.0
    p.temperatureRelease, p.expansionRate = 0.5, 0.2
    return p, CombustionParams.from_buffer_copy(bytes(p))


def _fd_check(t, fields, src, weights, grads, n, op, om, iterations, rng, count):
    """Central differences of sum(w * step(x)) of the FP64 oracle at `count` seeded entries of
    each input, against the adjoint's gradients."""
    keys = list(fields)
    s64 = {"src_" + k: np.asarray(v, np.float64) for k, v in src.items()}

    def loss(f):
        v, sc, _ = t.hns_advance_model(f["velocity"], {k: f[k] for k in keys if k != "velocity"}, s64, DX, iterations,
                                       DT, op, om, dtype=np.float64)
        out = {"velocity": v, **sc}
        return sum(float(np.sum(weights[k] * out[k])) for k in keys)

    base = {k: np.asarray(v, np.float64).copy() for k, v in fields.items()}
    worst = {}
    for k in keys:
        flat = base[k].reshape(-1)
        idx = rng.choice(flat.size, count, replace=False)
        fd = np.empty(count)
        for q, i in enumerate(idx):
            h = 1e-6
            xp = {kk: vv.copy() for kk, vv in base.items()}
            xm = {kk: vv.copy() for kk, vv in base.items()}
            xp[k].reshape(-1)[i] += h
            xm[k].reshape(-1)[i] -= h
            fd[q] = (loss(xp) - loss(xm)) / (2 * h)
        adj = grads[k].reshape(-1)[idx]
        worst[k] = float(np.max(np.abs(adj - fd)) / max(1e-30, np.max(np.abs(fd))))
    return worst


@pytest.mark.parametrize("combustion", [1, 0, 2])
def test_fire_adjoint_fp32_against_fd(dev, oracle, combustion):
    from oracle.binding import ForceModel as OM

    from hnanosolver_b200 import lib as hl

    origins, n, fields, src = _case(combustion)
    op, params = _params()
    om = OM(combustion=combustion, burn_rate=0.5, heat_release=1.0, ignition_temp=0.2, density_buoyancy=0.1)
    gm = hl.ForceModel(combustion=combustion, burn_rate=0.5, heat_release=1.0, ignition_temp=0.2, density_buoyancy=0.1)
    iterations = 20
    rng = np.random.default_rng(combustion + 7)
    weights = {k: rng.standard_normal(v.shape) for k, v in fields.items()}
    g = hl.Grid(origins, voxel_size=DX)
    fin = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev).reshape(-1) for k, v in fields.items()}
    sd = {k: torch.from_numpy(v).to(dev) for k, v in src.items()}
    ob = {k: torch.from_numpy(np.ascontiguousarray(w, dtype=np.float32)).to(dev).reshape(-1) for k, w in weights.items()}
    ib = {k: torch.zeros_like(v) for k, v in fin.items()}
    torch.cuda.synchronize()
    g.adjoint_advance(fin, sd, ob, ib, DT, iterations, params, gm)
    g.synchronize()
    grads = {k: v.double().cpu().numpy() for k, v in ib.items()}
    worst = _fd_check(oracle.topo(origins), fields, src, weights, grads, n, op, om, iterations, rng, 48)
    print(f"fire adjoint (FP32, combustion {combustion}) vs FD: {worst}")
    assert max(worst.values()) <= FD_TOL, worst
    g.close()


def test_fire_adjoint_mixed_against_fd(dev, oracle):
    from oracle.binding import ForceModel as OM

    from hnanosolver_b200 import lib as hl

    origins, n, fields, src = _case(1)
    op, params = _params()
    om = OM(combustion=1, burn_rate=0.5, heat_release=1.0, ignition_temp=0.2, density_buoyancy=0.1, omega=1.9)
    gm = hl.ForceModel(combustion=1, burn_rate=0.5, heat_release=1.0, ignition_temp=0.2, density_buoyancy=0.1)
    desc = hl.MixedDesc(dt=0.0, omega=1.9, tolerance=1e-6, max_outer=20, inner_iterations=30, flags=0)
    rng = np.random.default_rng(3)
    weights = {k: rng.standard_normal(v.shape) for k, v in fields.items()}
    g = hl.Grid(origins, voxel_size=DX)
    fin = {}
    for k, v in fields.items():
        t = torch.from_numpy(np.ascontiguousarray(v)).to(dev).reshape(-1)
        fin[k] = (t.to(torch.bfloat16) if k == "velocity" else t.to(torch.float16)).contiguous()
    sd = {k: torch.from_numpy(v).to(dev).to(torch.float16) for k, v in src.items()}
    ob = {k: torch.from_numpy(np.ascontiguousarray(w, dtype=np.float32)).to(dev).reshape(-1) for k, w in weights.items()}
    ib = {k: torch.zeros(v.numel(), device=dev) for k, v in fin.items()}
    torch.cuda.synchronize()
    g.adjoint_advance_mixed(fin, sd, ob, ib, DT, params, gm, desc)
    g.synchronize()
    grads = {k: v.double().cpu().numpy() for k, v in ib.items()}
    # The oracle differentiates at the BF16/FP16 values the step reads.
    at = {k: fin[k].double().cpu().numpy().reshape(fields[k].shape) for k in fields}
    src_at = {k: sd[k].double().cpu().numpy() for k in src}
    worst = _fd_check(oracle.topo(origins), at, src_at, weights, grads, n, op, om, 600, rng, 24)
    print(f"fire adjoint (mixed) vs FD: {worst}")
    assert max(worst.values()) <= FD_TOL, worst
    g.close()
