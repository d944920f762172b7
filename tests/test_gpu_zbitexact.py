"""Bit-exactness of the FP32 CUDA path against the oracle.

libhns is compiled without implicit FMA contraction, and its kernels apply the reference's
operations in the reference's order, so on the same inputs every FP32 output should equal
the oracle's (which equals the reference's kernels run as host C++) to the last bit. The
parity bar of the other tests is 1e-5 relative; this file checks the stronger property."""
import numpy as np
import pytest

from conftest import bit_exact
from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def test_operators_bit_exact(dev, oracle, golden_kernels):
    from hnanosolver_b200 import lib as hl

    g = golden_kernels
    origins, vel, dens = g["leaf_origins"], g["velocity"], g["density"]
    grid = hl.Grid(origins, voxel_size=0.1)
    t = oracle.topo(origins)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    v, d = T(vel), T(dens)
    out3, out1 = torch.empty_like(v), torch.empty_like(d)
    checks = {}
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    grid.advect_vec3(v, out3, 0.1)
    grid.synchronize()
    checks["advect_vec3"] = bit_exact(out3.cpu().numpy(), t.advect_vector(vel, 0.1, 10.0))
    grid.advect_scalar(v, d, out1, 0.1)
    grid.synchronize()
    checks["advect_scalar"] = bit_exact(out1.cpu().numpy(), t.advect_scalar(vel, dens, 0.1, 10.0))
    grid.advect_scalars(v, [d], [out1], 0.1)
    grid.synchronize()
    checks["advect_scalars"] = bit_exact(out1.cpu().numpy(), t.advect_scalars(vel, [dens], 0.1, 10.0)[0])
    div = t.divergence(vel, 10.0)
    grid.divergence(v, out1)
    grid.synchronize()
    checks["divergence"] = bit_exact(out1.cpu().numpy(), div)
    p = torch.zeros_like(d)
    grid.rbgs(T(div), p, 13, 1.7, hl.SOLVE_ZERO_INIT)
    grid.synchronize()
    checks["rbgs"] = bit_exact(p.cpu().numpy(), t.rbgs(div, np.zeros_like(div), 0.1, 13, 1.7))
    grid.vorticity_confinement(v, out3, 0.1, 0.3, 1.0)
    grid.synchronize()
    checks["vorticity"] = bit_exact(out3.cpu().numpy(), t.vorticity_confinement(vel, 0.1, 10.0, 0.3, 1.0))
    vv = T(vel)
    grid.project(vv, 9, -1.0)
    checks["project"] = bit_exact(vv.cpu().numpy(), t.project(vel, 0.1, 9, -1.0)[0])
    grid.close()
    assert all(checks.values()), checks


def test_advance_rollout_bit_exact(dev, oracle):
    from oracle.binding import CombustionParams as OP

    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(80, 3, 8.0, 18.0, seed=4)
    dens, vel = synth.smoothed_fields(origins, seed=9, box_passes=2)
    vel = (vel * 5.0).astype(np.float32)
    n = len(dens)
    rng = np.random.default_rng(2)
    src = {"src_temperature": (rng.random(n) > 0.85).astype(np.float32) * 3.0,
           "src_fuel": (rng.random(n) > 0.85).astype(np.float32),
           "src_vel": rng.uniform(-1, 1, (n, 3)).astype(np.float32)}
    op = OP.houdini_defaults()
    op.ambientTemp, op.factorScale, op.substeps = 0.3, 1.0, 2
    grid = hl.Grid(origins, voxel_size=0.1)
    grid.field_set("velocity", vel)
    grid.field_set("density", dens)
    for k, a in src.items():
        grid.field_set(k, a)
    t = oracle.topo(origins)
    ov, state = vel, {"density": dens}
    for call in range(3):
        grid.advance(12, 1.0 / 24.0, hl.CombustionParams.from_buffer_copy(bytes(op)))
        ov, sc, cr = t.hns_advance(ov, state, src, 0.1, 12, 1.0 / 24.0, op)
        state = {**sc, **cr}
    assert bit_exact(grid.field_get("velocity"), ov)
    for name, ref in state.items():
        assert bit_exact(grid.field_get(name), ref), name
    grid.close()
