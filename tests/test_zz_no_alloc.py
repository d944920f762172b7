"""hns_project_static (solver scratch in a fixed device array, no allocation) against
hns_project, called through the C ABI. Tolerance: max |static - project| / max |project|
<= 1e-5 on the projected velocity, and the same FP64 residuals, on two calls in a row with
different inputs and odd/even iteration counts. Also checked: the call leaves the device's
free memory unchanged, a call without `info` and a zero-iteration call, and a call right
after another grid's call (the shared array keeps the last call's contents). This file is
collected last so that the static array is also exercised after every other test has run
in the process.

The library runs on the context's own (non-blocking) stream, while torch uploads and clones
on its current stream: every input is made on torch's stream and synchronised before the C ABI
reads it."""
import ctypes

import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5
MAX_VOXELS = 1 << 20


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def project_static(hl, grid, vel, iterations, omega, info=True):
    si = hl.SolveInfo()
    st = hl.lib.hns_project_static(grid._h, ctypes.c_void_p(vel.data_ptr()), iterations, omega, 0,
                                   ctypes.byref(si) if info else None)
    return st, si


def _velocity(dev, origins, seed):
    _, vel = synth.smoothed_fields(origins, seed=seed, box_passes=2)
    return torch.from_numpy((vel * 8.0).astype(np.float32)).to(dev)


@pytest.mark.parametrize("topo", ["box64", "spheres"])
def test_static_projection_matches_project_twice(dev, topo):
    from hnanosolver_b200 import lib as hl

    origins = synth.topology("box64") if topo == "box64" else synth.spheres_topology(96, 3, 8.0, 20.0, seed=11)
    grid = hl.Grid(origins, voxel_size=0.1, device=0)
    try:
        for call, (seed, iterations) in enumerate([(5, 41), (6, 40)]):
            v0 = _velocity(dev, origins, seed)
            want = v0.clone()
            got = v0.clone()
            torch.cuda.synchronize()
            info_want = grid.project(want, iterations, omega=-1.0)
            st, info_got = project_static(hl, grid, got, iterations, -1.0)
            assert st == 0, (call, hl.lib.hns_last_error())
            grid.synchronize()
            w, g = want.cpu().numpy(), got.cpu().numpy()
            assert rel_err(g, w) <= TOL, (call, rel_err(g, w))
            assert info_got.iterations == iterations
            assert info_got.residual == pytest.approx(info_want.residual, rel=1e-6)
            assert info_got.initial_residual == pytest.approx(info_want.initial_residual, rel=1e-6)
            assert info_got.residual < info_got.initial_residual
        assert hl.lib.hns_device_status(grid._h) == 0
    finally:
        grid.close()


def test_static_projection_allocates_nothing(dev):
    """After one warm-up call (which loads the module holding the array), a call on a fresh
    context leaves the device's free memory exactly as it was."""
    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(96, 3, 8.0, 20.0, seed=12)
    warm = hl.Grid(origins, voxel_size=0.1, device=0)
    v = _velocity(dev, origins, 7)
    torch.cuda.synchronize()
    assert project_static(hl, warm, v, 6, -1.0)[0] == 0
    warm.synchronize()
    warm.close()
    grid = hl.Grid(origins, voxel_size=0.1, device=0)
    try:
        torch.cuda.synchronize()
        free_before, _ = torch.cuda.mem_get_info(dev)
        st, info = project_static(hl, grid, v, 9, -1.0)
        assert st == 0, hl.lib.hns_last_error()
        st, _ = project_static(hl, grid, v, 8, -1.0, info=False)
        assert st == 0, hl.lib.hns_last_error()
        grid.synchronize()
        free_after, _ = torch.cuda.mem_get_info(dev)
        assert free_after == free_before
        assert info.iterations == 9
    finally:
        grid.close()


def test_static_projection_without_info_and_zero_iterations(dev):
    """info = NULL (no residuals, no synchronisation) and iterations = 0 right after calls on
    another grid: zero iterations leave p = 0, so the velocity is unchanged; an odd count
    after a different grid's call equals hns_project without info."""
    from hnanosolver_b200 import lib as hl

    other = synth.topology("box64")
    origins = synth.spheres_topology(96, 3, 8.0, 20.0, seed=13)
    g_other = hl.Grid(other, voxel_size=0.1, device=0)
    grid = hl.Grid(origins, voxel_size=0.1, device=0)
    try:
        vo = _velocity(dev, other, 8)
        torch.cuda.synchronize()
        assert project_static(hl, g_other, vo, 41, -1.0)[0] == 0  # fills the shared array
        g_other.synchronize()

        v0 = _velocity(dev, origins, 9)
        same = v0.clone()
        torch.cuda.synchronize()
        st, _ = project_static(hl, grid, same, 0, -1.0, info=False)
        assert st == 0, hl.lib.hns_last_error()
        grid.synchronize()
        assert torch.equal(same, v0)

        assert project_static(hl, g_other, vo, 40, -1.0)[0] == 0
        g_other.synchronize()
        want, got = v0.clone(), v0.clone()
        torch.cuda.synchronize()
        grid.project(want, 17, omega=-1.0, info=False)
        st, _ = project_static(hl, grid, got, 17, -1.0, info=False)
        assert st == 0, hl.lib.hns_last_error()
        grid.synchronize()
        assert rel_err(got.cpu().numpy(), want.cpu().numpy()) <= TOL
    finally:
        grid.close()
        g_other.close()


def test_static_projection_rejects_grids_above_the_limit(dev):
    from hnanosolver_b200 import lib as hl

    # 16 x 16 x 9 leaves = 2304 leaves = 1,179,648 voxels > 2^20.
    ii, jj, kk = np.meshgrid(np.arange(16), np.arange(16), np.arange(9), indexing="ij")
    origins = (np.stack([ii, jj, kk], -1).reshape(-1, 3) * 8).astype(np.int32)
    grid = hl.Grid(origins, voxel_size=0.1, device=0)
    try:
        assert grid.num_voxels > MAX_VOXELS
        vel = torch.zeros(3 * grid.num_voxels, device=dev)
        torch.cuda.synchronize()
        st, _ = project_static(hl, grid, vel, 4, -1.0)
        assert st == 7  # HNS_ERR_UNSUPPORTED
        msg = hl.lib.hns_last_error().decode()
        assert "1048576" in msg and "hns_project" in msg
    finally:
        grid.close()
