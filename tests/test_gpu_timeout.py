"""The timeout paths of the bounded device-side waits, made to run out on purpose.

rbgs_stream_kernel (the FP32 red-black iteration) waits for each leaf's bulk copies on an
mbarrier with a bounded number of polls. The test hook HNS_OPT_WAIT_POLLS lowers the limit of
that first wait to 0 polls, so every CTA gives up at its first leaf: it raises the device error
flag, still waits for its copies in flight with the normal limit (no copy is writing when the
CTA exits), and returns. Nothing hangs or faults: hns_device_status reports HNS_ERR_TIMEOUT
once and clears it, and the next call with the default limit is clean and gives the same bits
as a context that never timed out.

The persistent inner solve of the mixed-precision step orders its leaf groups by progress
counters, each wait bounded. With the same hook every wait's target is out of reach: the first
waits give up after 0 polls, raise the flag and the abort word, every CTA returns, and the step
ends (unconverged) instead of hanging; the next step with the default is clean and bit-exact."""
import numpy as np
import pytest

from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def test_bounded_copy_wait_gives_up_then_recovers(dev):
    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(96, 3, 8.0, 20.0, seed=12)
    dens, vel = synth.smoothed_fields(origins, seed=3, box_passes=1)
    n = len(dens)
    clean = hl.Grid(origins, voxel_size=0.1)
    grid = hl.Grid(origins, voxel_size=0.1)
    for g in (clean, grid):  # the staged kernel, whose copies the bounded wait guards
        g.set_option(hl.OPT_RBGS_KERNEL, hl.RBGS_BULK)
    v = torch.from_numpy(vel).to(dev)
    div = torch.empty(n, device=dev)
    p_ref = torch.zeros(n, device=dev)
    torch.cuda.synchronize()
    clean.divergence(v, div)
    clean.rbgs(div, p_ref, 6, 1.7)
    clean.synchronize()

    grid.set_option(hl.OPT_WAIT_POLLS, 0)
    p = torch.zeros(n, device=dev)
    torch.cuda.synchronize()
    grid.rbgs(div, p, 6, 1.7)  # the launches themselves succeed
    st = hl.lib.hns_device_status(grid._h)
    assert st == 8, hl.STATUS_NAMES.get(st)  # HNS_ERR_TIMEOUT
    assert b"device-side wait" in hl.lib.hns_last_error()
    assert hl.lib.hns_device_status(grid._h) == 0  # reported once, then cleared
    assert not torch.equal(p, p_ref)  # the solve did not finish

    grid.set_option(hl.OPT_WAIT_POLLS, -1)
    p2 = torch.zeros(n, device=dev)
    torch.cuda.synchronize()
    grid.rbgs(div, p2, 6, 1.7)
    assert hl.lib.hns_device_status(grid._h) == 0
    assert torch.equal(p2, p_ref)
    with pytest.raises(hl.HnsError):
        grid.set_option(hl.OPT_WAIT_POLLS, -2)
    grid.close()
    clean.close()
    assert np.isfinite(p2.cpu().numpy()).all()


def test_persistent_inner_solve_wait_gives_up_then_recovers(dev):
    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(96, 3, 8.0, 20.0, seed=12)
    dens, vel = synth.smoothed_fields(origins, seed=3, box_passes=1)
    st = hl.MixedDesc(dt=0.1, max_outer=4, inner_iterations=12, omega=1.8, tolerance=1e-5, flags=0)

    def step(g):
        vb = torch.from_numpy(vel).to(dev).to(torch.bfloat16)
        dh = torch.from_numpy(dens).to(dev).to(torch.float16)
        vo, do = torch.empty_like(vb), torch.empty_like(dh)
        torch.cuda.synchronize()
        try:
            g.step_mixed(vb, vo, [dh], [do], st)
        except hl.HnsError as e:
            assert e.status == 6  # HNS_ERR_NOT_CONVERGED at most
        p = torch.empty(g.num_voxels, dtype=torch.float64, device=dev)
        g.refine_pressure(p)
        torch.cuda.synchronize()
        return vo.cpu(), p.cpu()

    clean = hl.Grid(origins, voxel_size=0.1)
    clean.set_option(hl.OPT_SPLIT_SOLVE, hl.SPLIT_PERSISTENT)
    ref = step(clean)
    assert hl.lib.hns_device_status(clean._h) == 0
    clean.close()

    grid = hl.Grid(origins, voxel_size=0.1)
    grid.set_option(hl.OPT_SPLIT_SOLVE, hl.SPLIT_PERSISTENT)
    grid.set_option(hl.OPT_WAIT_POLLS, 0)
    step(grid)
    s = hl.lib.hns_device_status(grid._h)
    assert s == 8, hl.STATUS_NAMES.get(s)  # HNS_ERR_TIMEOUT
    assert hl.lib.hns_device_status(grid._h) == 0
    grid.set_option(hl.OPT_WAIT_POLLS, -1)
    got = step(grid)
    assert hl.lib.hns_device_status(grid._h) == 0
    assert torch.equal(got[0], ref[0]) and torch.equal(got[1], ref[1])
    grid.close()
