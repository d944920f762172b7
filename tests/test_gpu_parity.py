"""Parity of the CUDA kernels (through the C ABI) with the CPU oracle, on the golden
inputs, the 64^3 box and seeded sparse grids. Tolerance: max |gpu - oracle| / max |oracle|
<= 1e-5 for FP32 fields; topology and offsets bit-exact."""
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


def T(a, dev):
    """Uploads on torch's stream and waits: the library's own stream does not wait for torch's."""
    t = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    torch.cuda.synchronize()
    return t


def H(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def grids():
    yield "golden", None
    yield "box64", synth.topology("box64")
    yield "spheres", synth.spheres_topology(96, 3, 8.0, 20.0, seed=11)


@pytest.fixture(scope="module", params=["golden", "box64", "spheres"])
def case(request, golden_kernels, oracle, dev):
    from hnanosolver_b200 import lib as hl

    if request.param == "golden":
        g = golden_kernels
        origins, vel, dens = g["leaf_origins"], g["velocity"], g["density"]
    else:
        origins = dict(grids())[request.param]
        dens, vel = synth.smoothed_fields(origins, seed=3, box_passes=2)
        vel = (vel * 8.0).astype(np.float32)
    grid = hl.Grid(origins, voxel_size=0.1, device=0)
    yield dict(grid=grid, topo=oracle.topo(origins), origins=origins, vel=vel, dens=dens)
    grid.close()


def test_offsets_bit_exact(case):
    coords = synth.leaf_dense_coords(case["origins"])
    rng = np.random.default_rng(1)
    q = np.concatenate([coords, rng.integers(coords.min() - 20, coords.max() + 20, size=(50000, 3)).astype(np.int32)])
    assert np.array_equal(case["grid"].index_offsets(q), case["topo"].offsets(q))
    assert case["grid"].is_nanovdb_order()


def test_offsets_golden(golden_topology, dev):
    from hnanosolver_b200 import lib as hl

    g = golden_topology
    grid = hl.Grid(g["leaf_origins"], voxel_size=1.0)
    assert np.array_equal(grid.index_offsets(g["query"]), g["offsets"])
    grid.close()


def test_advect_vec3(case, dev):
    g, t = case["grid"], case["topo"]
    v = T(case["vel"], dev)
    out = torch.empty_like(v)
    g.advect_vec3(v, out, 0.1)
    g.synchronize()
    assert rel_err(H(out), t.advect_vector(case["vel"], 0.1, 10.0)) <= TOL


def test_advect_scalar(case, dev):
    g, t = case["grid"], case["topo"]
    v, d = T(case["vel"], dev), T(case["dens"], dev)
    out = torch.empty_like(d)
    g.advect_scalar(v, d, out, 0.1)
    g.synchronize()
    assert rel_err(H(out), t.advect_scalar(case["vel"], case["dens"], 0.1, 10.0)) <= TOL


def test_advect_scalars_slot0_fallback(case, dev):
    g, t = case["grid"], case["topo"]
    fields = [case["dens"], (case["dens"] * 3.0 - 1.0).astype(np.float32)]
    v = T(case["vel"], dev)
    ins = [T(f, dev) for f in fields]
    outs = [torch.empty_like(x) for x in ins]
    g.advect_scalars(v, ins, outs, 0.1)
    g.synchronize()
    ref = t.advect_scalars(case["vel"], fields, 0.1, 10.0)
    for o, r in zip(outs, ref):
        assert rel_err(H(o), r) <= TOL


def test_divergence(case, dev):
    g, t = case["grid"], case["topo"]
    v = T(case["vel"], dev)
    div = torch.empty(len(case["vel"]), device=dev)
    g.divergence(v, div)
    g.synchronize()
    assert rel_err(H(div), t.divergence(case["vel"], 10.0)) <= TOL


@pytest.mark.parametrize("iters,omega,zero", [(1, 1.0, True), (7, 1.5, True), (8, 1.9, False), (40, 1.0, True)])
def test_rbgs(case, dev, iters, omega, zero):
    from hnanosolver_b200 import lib as hl

    g, t = case["grid"], case["topo"]
    div = t.divergence(case["vel"], 10.0)
    p0 = np.zeros_like(div) if zero else (case["dens"] * 0.01).astype(np.float32)
    p = T(p0, dev)
    g.rbgs(T(div, dev), p, iters, omega, hl.SOLVE_ZERO_INIT if zero else 0)
    g.synchronize()
    assert rel_err(H(p), t.rbgs(div, p0, 0.1, iters, omega)) <= TOL


def test_subtract_gradient(case, dev):
    g, t = case["grid"], case["topo"]
    p = (case["dens"] * 0.05).astype(np.float32)
    out = torch.empty(case["vel"].shape, device=dev)
    g.subtract_gradient(T(case["vel"], dev), T(p, dev), out)
    g.synchronize()
    assert rel_err(H(out), t.subtract_gradient(case["vel"], p, 10.0)) <= TOL


@pytest.mark.parametrize("fs", [0.5, 1.0, 2.0])
def test_vorticity(case, dev, fs):
    g, t = case["grid"], case["topo"]
    out = torch.empty(case["vel"].shape, device=dev)
    g.vorticity_confinement(T(case["vel"], dev), out, 0.1, 0.3, fs)
    g.synchronize()
    assert rel_err(H(out), t.vorticity_confinement(case["vel"], 0.1, 10.0, 0.3, fs)) <= TOL


def test_project(case, dev):
    g, t = case["grid"], case["topo"]
    v = T(case["vel"], dev)
    info = g.project(v, 25, -1.0)
    ref_v, ref_div, ref_p = t.project(case["vel"], 0.1, 25, -1.0)
    assert rel_err(H(v), ref_v) <= TOL
    r2, b2 = t.residual(ref_div, ref_p, 0.1)
    assert info.iterations == 25
    assert info.residual == pytest.approx(np.sqrt(r2 / b2), rel=1e-3)
    assert info.initial_residual == pytest.approx(1.0, rel=1e-9)


@pytest.mark.parametrize("kernel,form", [(0, None), (1, None), (2, 0), (2, 1)])
@pytest.mark.parametrize("iters,zero", [(1, True), (6, False), (11, True)])
def test_rbgs_kernels_bit_exact(case, dev, kernel, form, iters, zero):
    """The FP32 red-black kernels (plain-load halo tile, bulk async copies into a staged tile,
    colour-split leaves launched per colour or as one persistent launch) equal the oracle."""
    from conftest import bit_exact
    from hnanosolver_b200 import lib as hl

    g, t = case["grid"], case["topo"]
    g.set_option(hl.OPT_RBGS_KERNEL, kernel)
    g.set_option(hl.OPT_SPLIT_SOLVE, hl.SPLIT_PER_COLOUR if form is None else form)
    div = t.divergence(case["vel"], 10.0)
    p0 = np.zeros_like(div) if zero else (case["dens"] * 0.01).astype(np.float32)
    p = T(p0, dev)
    g.rbgs(T(div, dev), p, iters, 1.8, hl.SOLVE_ZERO_INIT if zero else 0)
    g.device_status()
    assert bit_exact(H(p), t.rbgs(div, p0, 0.1, iters, 1.8))
    g.set_option(hl.OPT_RBGS_KERNEL, hl.RBGS_SPLIT)
    g.set_option(hl.OPT_SPLIT_SOLVE, hl.SPLIT_PER_COLOUR)


def test_rbgs_unaligned_pointers_fall_back(case, dev):
    from conftest import bit_exact

    g, t = case["grid"], case["topo"]
    n = len(case["dens"])
    div = t.divergence(case["vel"], 10.0)
    buf = torch.zeros(2 * n + 8, device=dev)
    dv = buf[1:n + 1]          # 4-byte offset: not 16-byte aligned
    dv.copy_(T(div, dev))
    p = buf[n + 3:2 * n + 3]
    g.rbgs(dv, p, 5, 1.6, 1)
    g.device_status()
    assert bit_exact(H(p), t.rbgs(div, np.zeros_like(div), 0.1, 5, 1.6))
