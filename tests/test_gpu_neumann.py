"""Zero-gradient (Neumann) walls on the GPU (HNS_SOLVE_NEUMANN) against the oracle's restatement
(tests/test_oracle_neumann.py): max |gpu - oracle| / max |oracle| <= 1e-5.

  * hns_project: divergence, its mean removed per face-connected component in FP64, red-black
    SOR with the in-domain neighbour average, gradient with the wall's ghost pressure equal to
    the voxel's own: on the CPU-runnable single step's 64^3 box (40 iterations, omega 1.0) and on
    a grid of two separate components;
  * hns_rbgs with the flag relaxes the given divergence (no mean removal);
  * hns_step_plain solves to a tolerance with the walls; the reported FP64 residual equals the
    oracle's for the returned pressure's iteration count;
  * the forms the walls do not support say so (refined and mixed solves, the static projection)."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5
NEUMANN = 2


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _two_components():
    a = synth._box_leaves(24)
    b = synth._box_leaves(16) + np.array([48, 8, 8], np.int32)
    return synth.sort_leaves_nanovdb(np.concatenate([a, b]))


@pytest.mark.parametrize("topo", ["box64", "two"])
def test_neumann_projection_matches_oracle(dev, oracle, topo):
    from hnanosolver_b200 import lib as hl

    origins = synth.topology("box64") if topo == "box64" else _two_components()
    dens, vel = synth.smoothed_fields(origins, seed=0, box_passes=3)
    vel = (vel * 4.0).astype(np.float32)
    g = hl.Grid(origins, voxel_size=0.1)
    v = torch.from_numpy(vel).to(dev)
    torch.cuda.synchronize()
    info = g.project(v, 40, omega=1.0, flags=NEUMANN)
    g.synchronize()
    t = oracle.topo(origins)
    ov, od, op = t.project_neumann(vel, np.float32(0.1), 40, np.float32(1.0))
    assert rel_err(v.cpu().numpy(), ov) <= TOL
    r2, b2 = t.residual_neumann(od, op, np.float32(0.1))
    assert info.residual == pytest.approx(np.sqrt(r2 / b2), rel=1e-5)
    assert info.residual < info.initial_residual
    # The reference's walls give another field.
    v2 = torch.from_numpy(vel).to(dev)
    torch.cuda.synchronize()
    g.project(v2, 40, omega=1.0)
    g.synchronize()
    assert rel_err(v2.cpu().numpy(), ov) > 1e-3
    g.close()


def test_neumann_rbgs_matches_oracle(dev, oracle):
    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(64, 3, 8.0, 16.0, 4)
    n = 512 * len(origins)
    rng = np.random.default_rng(2)
    div = rng.standard_normal(n).astype(np.float32)
    p0 = rng.standard_normal(n).astype(np.float32)
    g = hl.Grid(origins, voxel_size=0.1)
    d, p = torch.from_numpy(div).to(dev), torch.from_numpy(p0).to(dev)
    torch.cuda.synchronize()
    g.rbgs(d, p, 7, 1.6, NEUMANN)
    g.synchronize()
    ref = oracle.topo(origins).rbgs_neumann(div, p0, np.float32(0.1), 7, np.float32(1.6))
    assert rel_err(p.cpu().numpy(), ref) <= TOL
    g.close()


def test_neumann_step_to_tolerance(dev, oracle):
    from hnanosolver_b200 import lib as hl

    origins = _two_components()
    dens, vel = synth.smoothed_fields(origins, seed=1, box_passes=2)
    vel = (vel * 4.0).astype(np.float32)
    g = hl.Grid(origins, voxel_size=0.1)
    vi, di = torch.from_numpy(vel).to(dev), torch.from_numpy(dens).to(dev)
    vo, do = torch.empty_like(vi), torch.empty_like(di)
    desc = hl.StepDesc(dt=0.1, max_iterations=2000, omega=1.8, tolerance=1e-5, check_every=10, flags=NEUMANN)
    torch.cuda.synchronize()
    info = g.step_plain(vi, vo, [di], [do], desc, info=True)
    assert info.residual <= 1e-5 and 0 < info.iterations < 2000
    t = oracle.topo(origins)
    adv = t.advect_vector(vel, 0.1, 10.0)
    ov, od, op = t.project_neumann(adv, np.float32(0.1), info.iterations, np.float32(1.8))
    assert rel_err(vo.cpu().numpy(), ov) <= TOL
    g.close()


def test_neumann_unsupported_forms(dev):
    from hnanosolver_b200 import lib as hl

    origins = synth.topology("box64")
    n = 512 * len(origins)
    g = hl.Grid(origins, voxel_size=0.1)
    v = torch.zeros(3 * n, device=dev)
    vo, d, do = torch.empty_like(v), torch.zeros(n, device=dev), torch.empty(n, device=dev)
    desc = hl.StepDesc(dt=0.1, max_iterations=0, omega=1.9, tolerance=1e-5, check_every=10,
                       flags=NEUMANN | hl.SOLVE_REFINE, max_outer=4, inner_iterations=10)
    with pytest.raises(hl.HnsError) as e:
        g.step_plain(v, vo, [d], [do], desc)
    assert e.value.status == 7
    si = hl.SolveInfo()
    assert hl.lib.hns_project_static(g._h, ctypes.c_void_p(v.data_ptr()), 4, -1.0, NEUMANN, ctypes.byref(si)) == 7
    g.close()
