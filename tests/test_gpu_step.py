"""The plain step (HNanoAdvect + HNanoAdvectVelocity + HNanoProjectNonDivergent chain)
against the oracle, its host-buffer form, and the device-side convergence stop."""
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


@pytest.fixture(scope="module")
def box64():
    origins = synth.topology("box64")
    dens, vel = synth.smoothed_fields(origins, seed=0, box_passes=3)
    return origins, dens, vel


def _desc(**kw):
    from hnanosolver_b200.lib import StepDesc

    d = dict(dt=0.1, max_iterations=40, omega=1.0, tolerance=0.0, check_every=0, flags=0)
    d.update(kw)
    return StepDesc(**d)


def test_step_plain_box64_matches_oracle(dev, oracle, box64):
    """The CPU-runnable single step: 64^3 box, dt 0.1, dx 0.1, 40 iterations, omega 1."""
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = box64
    g = hl.Grid(origins, voxel_size=0.1)
    v_in, d_in = torch.from_numpy(vel).to(dev), torch.from_numpy(dens).to(dev)
    v_out, d_out = torch.empty_like(v_in), torch.empty_like(d_in)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    info = g.step_plain(v_in, v_out, [d_in], [d_out], _desc(), info=True)
    t = oracle.topo(origins)
    ref_d = t.advect_scalar(vel, dens, 0.1, 10.0)
    ref_v, ref_div, ref_p = t.project(t.advect_vector(vel, 0.1, 10.0), 0.1, 40, 1.0)
    torch.cuda.synchronize()
    assert rel_err(d_out.cpu().numpy(), ref_d) <= TOL
    assert rel_err(v_out.cpu().numpy(), ref_v) <= TOL
    r2, b2 = t.residual(ref_div, ref_p, 0.1)
    assert info.iterations == 40
    assert info.residual == pytest.approx(np.sqrt(r2 / b2), rel=1e-3)
    g.close()


def test_step_plain_host_equals_device(dev, box64):
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = box64
    g = hl.Grid(origins, voxel_size=0.1)
    v_in, d_in = torch.from_numpy(vel).to(dev), torch.from_numpy(dens).to(dev)
    v_out, d_out = torch.empty_like(v_in), torch.empty_like(d_in)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    g.step_plain(v_in, v_out, [d_in], [d_out], _desc(max_iterations=12, omega=1.6))
    g.synchronize()
    hv, hd = vel.copy(), dens.copy()
    g.step_plain_host(hv, [hd], _desc(max_iterations=12, omega=1.6))
    assert np.array_equal(hv, v_out.cpu().numpy())
    assert np.array_equal(hd, d_out.cpu().numpy())
    g.close()


@pytest.mark.parametrize("check_every", [2, 6, 10])
def test_convergence_stop_equals_fixed_iterations(dev, check_every):
    """With a tolerance, the solve stops on the device at a check boundary; its result is
    bit-identical to running that many iterations without checks, and meets the tolerance."""
    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(96, 3, 8.0, 20.0, seed=11)
    dens, vel = synth.smoothed_fields(origins, seed=3, box_passes=2)
    g = hl.Grid(origins, voxel_size=0.1)
    v_in, d_in = torch.from_numpy(vel).to(dev), torch.from_numpy(dens).to(dev)
    v_a, d_a = torch.empty_like(v_in), torch.empty_like(d_in)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    info = g.step_plain(v_in, v_a, [d_in], [d_a], _desc(max_iterations=600, omega=1.8, tolerance=1e-4,
                                                         check_every=check_every), info=True)
    assert info.iterations < 600 and info.iterations % check_every == 0
    assert g.last_solve().iterations == info.iterations
    v_b, d_b = torch.empty_like(v_in), torch.empty_like(d_in)
    info_b = g.step_plain(v_in, v_b, [d_in], [d_b], _desc(max_iterations=info.iterations, omega=1.8), info=True)
    torch.cuda.synchronize()
    assert torch.equal(v_a, v_b)
    assert info.residual == pytest.approx(info_b.residual, rel=1e-9)  # FP64 atomics: summation order varies
    assert info.residual <= 1e-4
    g.close()


def test_not_converged_status(dev):
    from hnanosolver_b200 import lib as hl

    origins = synth.topology("box64")
    dens, vel = synth.smoothed_fields(origins, seed=1, box_passes=1)
    g = hl.Grid(origins, voxel_size=0.1)
    v_in, d_in = torch.from_numpy(vel).to(dev), torch.from_numpy(dens).to(dev)
    v_out, d_out = torch.empty_like(v_in), torch.empty_like(d_in)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    with pytest.raises(hl.HnsError) as e:
        g.step_plain(v_in, v_out, [d_in], [d_out], _desc(max_iterations=4, tolerance=1e-9, check_every=2), info=True)
    assert e.value.status == 6
    g.close()


def test_profile_counts_solver_launches(dev, box64):
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = box64
    g = hl.Grid(origins, voxel_size=0.1)
    v_in, d_in = torch.from_numpy(vel).to(dev), torch.from_numpy(dens).to(dev)
    v_out, d_out = torch.empty_like(v_in), torch.empty_like(d_in)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    g.profile_read()
    g.profile_enable(True)
    g.step_plain(v_in, v_out, [d_in], [d_out], _desc(max_iterations=16))
    p = g.profile_read()
    assert p.solver_launches == 32  # red-black half-sweeps: two per iteration on the colour-split default
    assert p.phase_count[hl.PHASES["solve"]] == 1 and p.phase_ms[hl.PHASES["solve"]] > 0
    g.close()
