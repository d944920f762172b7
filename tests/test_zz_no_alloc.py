"""hns_project_static (solver scratch in a fixed device array, no allocation) against
hns_project, called through the C ABI. Tolerance: max |static - project| / max |project|
<= 1e-5 on the projected velocity, and the same FP64 residuals, on two calls in a row with
different inputs and odd/even iteration counts. This file is collected last so that the
static array is also exercised after every other test has run in the process."""
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


def project_static(hl, grid, vel, iterations, omega):
    si = hl.SolveInfo()
    st = hl.lib.hns_project_static(grid._h, ctypes.c_void_p(vel.data_ptr()), iterations, omega, 0, ctypes.byref(si))
    return st, si


@pytest.mark.parametrize("topo", ["box64", "spheres"])
def test_static_projection_matches_project_twice(dev, topo):
    from hnanosolver_b200 import lib as hl

    origins = synth.topology("box64") if topo == "box64" else synth.spheres_topology(96, 3, 8.0, 20.0, seed=11)
    grid = hl.Grid(origins, voxel_size=0.1, device=0)
    try:
        for call, (seed, iterations) in enumerate([(5, 41), (6, 40)]):
            _, vel = synth.smoothed_fields(origins, seed=seed, box_passes=2)
            v0 = torch.from_numpy((vel * 8.0).astype(np.float32)).to(dev)
            want = v0.clone()
            info_want = grid.project(want, iterations, omega=-1.0)
            got = v0.clone()
            st, info_got = project_static(hl, grid, got, iterations, -1.0)
            assert st == 0, (call, hl.lib.hns_last_error())
            torch.cuda.synchronize()
            w, g = want.cpu().numpy(), got.cpu().numpy()
            assert rel_err(g, w) <= TOL, (call, rel_err(g, w))
            assert info_got.iterations == iterations
            assert info_got.residual == pytest.approx(info_want.residual, rel=1e-6)
            assert info_got.initial_residual == pytest.approx(info_want.initial_residual, rel=1e-6)
            assert info_got.residual < info_got.initial_residual
        assert hl.lib.hns_device_status(grid._h) == 0
    finally:
        grid.close()


def test_static_projection_rejects_grids_above_the_limit(dev):
    from hnanosolver_b200 import lib as hl

    # 16 x 16 x 9 leaves = 2304 leaves = 1,179,648 voxels > 2^20.
    ii, jj, kk = np.meshgrid(np.arange(16), np.arange(16), np.arange(9), indexing="ij")
    origins = (np.stack([ii, jj, kk], -1).reshape(-1, 3) * 8).astype(np.int32)
    grid = hl.Grid(origins, voxel_size=0.1, device=0)
    try:
        assert grid.num_voxels > MAX_VOXELS
        vel = torch.zeros(3 * grid.num_voxels, device=dev)
        st, _ = project_static(hl, grid, vel, 4, -1.0)
        assert st == 7  # HNS_ERR_UNSUPPORTED
        msg = hl.lib.hns_last_error().decode()
        assert "1048576" in msg and "hns_project" in msg
    finally:
        grid.close()
