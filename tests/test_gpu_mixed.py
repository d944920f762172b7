"""Mixed precision (BF16 velocity, FP16 scalars, FP64 iterative refinement of the pressure
solve) against the FP64 oracle, and the FP32 refinement it is compared with.

Error statements checked here (a 160^3 shell, about 1.3M voxels):
  * the refined solve's residual ||b - L p|| / ||b||, recomputed by the oracle in FP64 from
    the returned FP64 pressure, is <= the 1e-5 tolerance;
  * the projected velocity differs from the FP64 oracle's (same BF16-rounded inputs, exact
    FP64 solve to 1e-10) by <= 2e-2 of its max (BF16 storage: 8 significant bits);
  * the advected density differs from the FP64 oracle's by <= 2e-3 of its max (FP16)."""
import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.fixture(scope="module")
def shell():
    origins = synth.shell_topology(160, 60.0, 8.0, seed=2)
    dens, vel = synth.noise_fields(origins, seed=5)
    return origins, dens, vel


def test_conversions_round_to_nearest(dev, shell):
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    g = hl.Grid(origins, voxel_size=0.1)
    v = torch.from_numpy(vel).to(dev).reshape(-1)
    b = torch.empty(v.numel(), dtype=torch.bfloat16, device=dev)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    g.convert(v, hl.DTYPE_F32, b, hl.DTYPE_BF16, v.numel())
    d = torch.from_numpy(dens).to(dev)
    h = torch.empty(d.numel(), dtype=torch.float16, device=dev)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    g.convert(d, hl.DTYPE_F32, h, hl.DTYPE_F16, d.numel())
    back = torch.empty_like(v)
    g.convert(b, hl.DTYPE_BF16, back, hl.DTYPE_F32, v.numel())
    g.synchronize()
    assert torch.equal(b, v.to(torch.bfloat16))
    assert torch.equal(h, d.to(torch.float16))
    assert torch.equal(back, v.to(torch.bfloat16).float())
    g.close()


def _mixed(g, dev, dens, vel, tol=1e-5, inner=40, outer=8, flags=0):
    from hnanosolver_b200 import lib as hl

    vb = torch.from_numpy(vel).to(dev).to(torch.bfloat16).contiguous()
    dh = torch.from_numpy(dens).to(dev).to(torch.float16).contiguous()
    vo, do = torch.empty_like(vb), torch.empty_like(dh)
    desc = hl.MixedDesc(dt=0.1, omega=1.9, tolerance=tol, max_outer=outer, inner_iterations=inner, flags=flags)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    info = g.step_mixed(vb, vo, [dh], [do], desc, info=True)
    return vb, dh, vo, do, info


def test_mixed_step_against_fp64_oracle(dev, oracle, shell):
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    g = hl.Grid(origins, voxel_size=0.1)
    vb, dh, vo, do, info = _mixed(g, dev, dens, vel)
    assert info.residual <= 1e-5
    t = oracle.topo(origins)
    v_in = vb.float().cpu().numpy()
    # The right-hand side the kernels solved: FP32 advection of the BF16 inputs (the oracle's
    # float path is the kernels' arithmetic), stored as BF16, then its FP32 divergence.
    adv = torch.from_numpy(t.advect_vector(v_in, 0.1, 10.0)).to(torch.bfloat16).float().numpy()
    div32 = t.divergence(adv, np.float32(10.0))
    # The residual claim, recomputed by the oracle in FP64 from the returned FP64 pressure.
    p = torch.empty(len(dens), dtype=torch.float64, device=dev)
    outer, res = g.refine_pressure(p)
    dx32 = float(np.float32(0.1))  # the library's voxel size is a float
    r2, b2 = t.residual(div32.astype(np.float64), p.cpu().numpy(), dx32)
    assert np.sqrt(r2 / b2) <= 1e-5
    assert np.sqrt(r2 / b2) == pytest.approx(res, rel=1e-6)
    # The gradient subtraction to the bit: the BF16 advected velocity minus the FP32-rounded
    # FP64 central difference of the returned pressure (0 outside the domain), rounded to BF16.
    p64 = p.cpu().numpy()
    ijk = t.coords()
    hh = 0.5 * float(np.float32(10.0))
    expect = adv.astype(np.float32).copy()
    for ax in range(3):
        e = np.zeros(3, dtype=np.int32)
        e[ax] = 1
        off_p = t.offsets(ijk + e).astype(np.int64)
        off_m = t.offsets(ijk - e).astype(np.int64)
        pp = np.where(off_p == 0, 0.0, p64[np.maximum(off_p - 1, 0)])
        pm = np.where(off_m == 0, 0.0, p64[np.maximum(off_m - 1, 0)])
        expect[:, ax] = expect[:, ax] - ((pp - pm) * hh).astype(np.float32)
    expect_bf16 = torch.from_numpy(expect).to(torch.bfloat16)
    assert torch.equal(vo.cpu().view(-1, 3), expect_bf16)
    # The scalar advection to the bit: the oracle's FP32 MacCormack step of the FP16 density
    # along the BF16 velocity, rounded to FP16.
    d_in = dh.float().cpu().numpy()
    expect_d = torch.from_numpy(t.advect_scalar(v_in, d_in, 0.1, 10.0)).to(torch.float16)
    assert torch.equal(do.cpu(), expect_d)
    # Field error against the FP64 oracle (same BF16/FP16 inputs, FP64 advection, FP64 solve
    # to a residual far below 1e-5).
    v64 = v_in.astype(np.float64)
    adv64 = t.advect_vector(v64, 0.1, 10.0)
    div64 = t.divergence(adv64, 10.0)
    p64 = t.rbgs(div64, np.zeros_like(div64), 0.1, 1200, 1.9)
    r2, b2 = t.residual(div64, p64, 0.1)
    assert np.sqrt(r2 / b2) < 1e-9
    ref_v = t.subtract_gradient(adv64, p64, 10.0)
    assert rel_err(vo.float().cpu().numpy(), ref_v) <= 2e-2
    ref_d = t.advect_scalar(v64, dh.float().cpu().numpy().astype(np.float64), 0.1, 10.0)
    assert rel_err(do.float().cpu().numpy(), ref_d) <= 2e-3
    g.close()


@pytest.mark.parametrize("nscalars", [0, 3])
def test_mixed_step_scalar_counts(dev, oracle, shell, nscalars):
    """The mixed advection reads the velocity and the first scalar as interleaved voxel records
    and further scalars from their own arrays: with no scalar the projected velocity is the one
    of the single-scalar step, and with three each advected scalar is the oracle's FP32
    MacCormack step of its FP16 input along the BF16 velocity, to the bit."""
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    g = hl.Grid(origins, voxel_size=0.1)
    vb = torch.from_numpy(vel).to(dev).to(torch.bfloat16).contiguous()
    rng = np.random.default_rng(3)
    fields = [dens] + [rng.random(len(dens), dtype=np.float32) for _ in range(2)]
    hs = [torch.from_numpy(f).to(dev).to(torch.float16).contiguous() for f in fields[:nscalars]]
    outs = [torch.empty_like(h) for h in hs]
    vo = torch.empty_like(vb)
    desc = hl.MixedDesc(dt=0.1, omega=1.9, tolerance=1e-5, max_outer=8, inner_iterations=40, flags=0)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    info = g.step_mixed(vb, vo, hs, outs, desc, info=True)
    assert info.residual <= 1e-5
    vb1, dh1, vo1, do1, _ = _mixed(g, dev, dens, vel)
    torch.cuda.synchronize()
    assert torch.equal(vo.cpu(), vo1.cpu())
    t = oracle.topo(origins)
    v_in = vb.float().cpu().numpy()
    for h, o in zip(hs, outs):
        expect = torch.from_numpy(t.advect_scalar(v_in, h.float().cpu().numpy(), 0.1, 10.0)).to(torch.float16)
        assert torch.equal(o.cpu(), expect)
    g.close()


def test_mixed_advection_long_traces(dev, oracle, shell):
    """Traces of up to four voxels per axis leave the shared-memory leaf tile of the advection
    (the leaf and a one-voxel halo) and take the leaf-table path: the density is still the
    oracle's FP32 MacCormack step of its FP16 input to the bit, and the velocity and density
    equal those of the records kernel (the path of a step with three scalars)."""
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    g = hl.Grid(origins, voxel_size=0.1)
    vb, dh, vo, do, _ = _mixed(g, dev, dens, vel * 4.0, tol=1e-3)
    t = oracle.topo(origins)
    v_in = vb.float().cpu().numpy()
    assert np.abs(v_in).max() > 3.0  # traces longer than the tile's halo
    expect_d = torch.from_numpy(t.advect_scalar(v_in, dh.float().cpu().numpy(), 0.1, 10.0)).to(torch.float16)
    assert torch.equal(do.cpu(), expect_d)
    hs = [dh, dh.clone(), dh.clone()]
    outs = [torch.empty_like(dh) for _ in hs]
    vo3 = torch.empty_like(vb)
    desc = hl.MixedDesc(dt=0.1, omega=1.9, tolerance=1e-3, max_outer=8, inner_iterations=40, flags=0)
    torch.cuda.synchronize()
    g.step_mixed(vb, vo3, hs, outs, desc)
    torch.cuda.synchronize()
    assert torch.equal(vo3.cpu(), vo.cpu())
    assert torch.equal(outs[0].cpu(), do.cpu())
    g.close()


def test_unaligned_arrays_match_aligned(dev, shell):
    """Velocity and scalar arrays that are only element-aligned (2 bytes for BF16/FP16, 4 for
    FP32) take element-wise loads in the advection, divergence and gradient kernels instead of
    the vector forms; the steps give the same bits as on aligned arrays."""
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    n = len(dens)
    g = hl.Grid(origins, voxel_size=0.1)
    vb, dh, vo, do, _ = _mixed(g, dev, dens, vel)

    def shifted(t):  # the same values at an address one element past an aligned one
        buf = torch.empty(t.numel() + 1, dtype=t.dtype, device=dev)
        view = buf[1:]
        view.copy_(t.reshape(-1))
        return view

    # The library runs on its own stream: the copies torch makes on its stream must be done
    # before each call reads them.
    vb_u, dh_u = shifted(vb), shifted(dh)
    vo_u, do_u = shifted(torch.zeros_like(vb)), shifted(torch.zeros_like(dh))
    torch.cuda.synchronize()
    desc = hl.MixedDesc(dt=0.1, omega=1.9, tolerance=1e-5, max_outer=8, inner_iterations=40, flags=0)
    g.step_mixed(vb_u, vo_u, [dh_u], [do_u], desc)
    torch.cuda.synchronize()
    assert torch.equal(vo_u.cpu(), vo.reshape(-1).cpu()) and torch.equal(do_u.cpu(), do.cpu())

    # The FP32 step with the refined solve (its gradient reads the FP64 pressure with vector
    # loads of velocity when the array is 16-byte aligned).
    v32 = torch.from_numpy(vel).to(dev).reshape(-1).contiguous()
    d32 = torch.from_numpy(dens).to(dev).contiguous()
    sd = hl.StepDesc(dt=0.1, max_iterations=0, omega=1.9, tolerance=1e-5, check_every=10,
                     flags=hl.SOLVE_REFINE, max_outer=10, inner_iterations=40)
    va, da = torch.empty_like(v32), torch.empty_like(d32)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    g.step_plain(v32, va, [d32], [da], sd)
    torch.cuda.synchronize()
    vi, di = shifted(v32), shifted(d32)
    vu, du = shifted(torch.zeros_like(v32)), shifted(torch.zeros_like(d32))
    torch.cuda.synchronize()
    g.step_plain(vi, vu, [di], [du], sd)
    torch.cuda.synchronize()
    assert torch.equal(vu.cpu(), va.cpu()) and torch.equal(du.cpu(), da.cpu())
    assert n > 0
    g.close()


def test_mixed_host_equals_device(dev, shell):
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    g = hl.Grid(origins, voxel_size=0.1)
    vb, dh, vo, do, info = _mixed(g, dev, dens, vel)
    hv = vb.float().cpu().numpy().copy()
    hd = dh.float().cpu().numpy().copy()
    desc = hl.MixedDesc(dt=0.1, omega=1.9, tolerance=1e-5, max_outer=8, inner_iterations=40, flags=0)
    info_h = g.step_mixed_host(hv, [hd], desc, info=True)
    assert np.array_equal(hv, vo.float().cpu().numpy())
    assert np.array_equal(hd, do.float().cpu().numpy())
    assert info_h.iterations == info.iterations
    g.close()


def test_fp32_refined_reaches_tolerance_plain_fp32_cannot(dev, shell):
    """Plain FP32 SOR at omega 1.9 stalls above 1e-5 on this grid (its rounding floor);
    the same solve inside FP64 refinement reaches it."""
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    g = hl.Grid(origins, voxel_size=0.1)
    v_in, d_in = torch.from_numpy(vel).to(dev), torch.from_numpy(dens).to(dev)
    v_out, d_out = torch.empty_like(v_in), torch.empty_like(d_in)
    desc = hl.StepDesc(dt=0.1, max_iterations=0, omega=1.9, tolerance=1e-6, check_every=10,
                       flags=hl.SOLVE_REFINE, max_outer=10, inner_iterations=40)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    info = g.step_plain(v_in, v_out, [d_in], [d_out], desc, info=True)
    assert info.residual <= 1e-6
    plain = hl.StepDesc(dt=0.1, max_iterations=3000, omega=1.9, tolerance=1e-6, check_every=10, flags=0)
    with pytest.raises(hl.HnsError) as e:
        g.step_plain(v_in, v_out, [d_in], [d_out], plain, info=True)
    assert e.value.status == 6
    g.close()


@pytest.mark.parametrize("grid", ["shell", "spheres"])
def test_inner_solve_layouts_bit_exact(dev, shell, grid):
    """The FP16 inner solve on colour-split leaves (the default, as one persistent launch per
    inner solve or one launch per colour), on colour-packed rows and on the plain slot order
    relax every voxel with the same arithmetic, so the whole mixed step -- refined pressure,
    outer iteration count, projected velocity, advected density -- is identical to the bit.
    The sparse spheres exercise missing neighbour leaves (face rings and z rings left at 0)."""
    from hnanosolver_b200 import lib as hl

    if grid == "shell":
        origins, dens, vel = shell
    else:
        origins = synth.spheres_topology(96, 3, 8.0, 20.0, seed=11)
        dens, vel = synth.noise_fields(origins, seed=7)
    out = {}
    forms = [(hl.INNER_ROWS, None), (hl.INNER_PACKED, None), (hl.INNER_SPLIT, hl.SPLIT_PER_COLOUR),
             (hl.INNER_SPLIT, hl.SPLIT_PERSISTENT)]
    for layout in forms:
        g = hl.Grid(origins, voxel_size=0.1)
        g.set_option(hl.OPT_INNER_LAYOUT, layout[0])
        if layout[1] is not None:
            g.set_option(hl.OPT_SPLIT_SOLVE, layout[1])
        vb, dh, vo, do, info = _mixed(g, dev, dens, vel, inner=30, outer=12)
        p = torch.empty(g.num_voxels, dtype=torch.float64, device=dev)
        outer, res = g.refine_pressure(p)
        g.device_status()  # raises HNS_ERR_TIMEOUT if a bounded copy wait gave up
        torch.cuda.synchronize()
        out[layout] = (vo.cpu(), do.cpu(), p.cpu(), outer, res, info.iterations)
        g.close()
    a = out[forms[0]]
    for layout in forms[1:]:
        b = out[layout]
        assert a[3] == b[3] and a[5] == b[5]
        assert a[4] == pytest.approx(b[4], rel=1e-12)  # FP64 atomics: summation order varies
        assert torch.equal(a[2], b[2])
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
        assert b[4] <= 1e-5


@pytest.mark.parametrize("inner_solve", ["red-black", "multigrid"])
def test_outer_forecast_short_grids_bit_exact(dev, shell, inner_solve):
    """A context forecasts the refinement's outer iterations from the checks of its earlier
    solves; the outer iterations past the forecast run their kernels on short grids (one wave,
    looping over the leaves), and under multigrid each runs as a graph whose device-side
    condition skips it after convergence. Whether those iterations find the solve converged (a
    forecast at or above the need) or still have work (a forecast below it), the step is the
    same to the bit as on a fresh context, which has no forecast."""
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    mg = inner_solve == "multigrid"

    def solve(g, tol):
        vb, dh, vo, do, info = _mixed(g, dev, dens, vel, tol=tol, inner=2 if mg else 30, outer=12,
                                      flags=hl.SOLVE_MULTIGRID if mg else 0)
        p = torch.empty(g.num_voxels, dtype=torch.float64, device=dev)
        outer, res = g.refine_pressure(p)
        torch.cuda.synchronize()
        return vo.cpu(), do.cpu(), p.cpu(), outer, res

    fresh = hl.Grid(origins, voxel_size=0.1)
    ref = solve(fresh, 1e-6)
    fresh.close()
    assert ref[4] <= 1e-6

    g = hl.Grid(origins, voxel_size=0.1)
    loose = solve(g, 1e-3)  # forecast: the few outer iterations of a loose tolerance
    assert loose[3] < ref[3]
    under = solve(g, 1e-6)  # iterations past that forecast still have work on short grids
    over = solve(g, 1e-6)   # forecast = the need: the iterations past it return at once
    g.close()
    for got in (under, over):
        assert got[3] == ref[3]
        assert got[4] == pytest.approx(ref[4], rel=1e-12)  # FP64 atomics: summation order varies
        assert torch.equal(got[2], ref[2])
        assert torch.equal(got[0], ref[0]) and torch.equal(got[1], ref[1])


@pytest.mark.parametrize("grid", ["spheres", "box", "shell"])
def test_multigrid_inner_solve_reaches_the_tolerance(dev, oracle, grid):
    """HNS_SOLVE_MULTIGRID: V-cycles (two per outer step for the mixed step, one for the FP32
    refined step) in place of the red-black iterations. The FP64 residual of the returned pressure, recomputed by the oracle, is within the tolerance,
    and the projected velocity agrees with the red-black refinement's to the accuracy that a
    1e-5 relative residual allows; the FP32 refined step takes the flag too."""
    from hnanosolver_b200 import lib as hl

    if grid == "spheres":
        origins = synth.spheres_topology(96, 3, 8.0, 20.0, seed=11)
    elif grid == "shell":
        origins = synth.shell_topology(160, 60.0, 8.0, seed=2)
    else:
        origins = synth.topology("box64")
    dens, vel = synth.noise_fields(origins, seed=7)
    g = hl.Grid(origins, voxel_size=0.1)
    vb = torch.from_numpy(vel).to(dev).to(torch.bfloat16).contiguous()
    dh = torch.from_numpy(dens).to(dev).to(torch.float16).contiguous()
    outs = {}
    for flags in (0, hl.SOLVE_MULTIGRID):
        vo, do = torch.empty_like(vb), torch.empty_like(dh)
        desc = hl.MixedDesc(dt=0.1, omega=1.9, tolerance=1e-5, max_outer=40, inner_iterations=2 if flags else 30,
                            flags=flags)
        torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
        info = g.step_mixed(vb, vo, [dh], [do], desc, info=True)
        assert info.residual <= 1e-5
        p = torch.empty(g.num_voxels, dtype=torch.float64, device=dev)
        g.refine_pressure(p)
        torch.cuda.synchronize()
        outs[flags] = (vo.float().cpu().numpy(), p.cpu().numpy())
    t = oracle.topo(origins)
    adv = torch.from_numpy(t.advect_vector(vb.float().cpu().numpy(), 0.1, 10.0)).to(torch.bfloat16).float().numpy()
    div = t.divergence(adv, np.float32(10.0)).astype(np.float64)
    r2, b2 = t.residual(div, outs[hl.SOLVE_MULTIGRID][1], float(np.float32(0.1)))  # the library's voxel size is a float
    assert np.sqrt(r2 / b2) <= 1e-5 * (1 + 1e-6)
    assert rel_err(outs[hl.SOLVE_MULTIGRID][0], outs[0][0]) <= 2e-2
    v = torch.from_numpy(vel).to(dev)
    d = torch.from_numpy(dens).to(dev)
    sd = hl.StepDesc(dt=0.1, max_iterations=0, omega=1.9, tolerance=1e-5, check_every=0,
                     flags=hl.SOLVE_REFINE | hl.SOLVE_MULTIGRID, max_outer=40, inner_iterations=30)
    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    info = g.step_plain(v, torch.empty_like(v), [d], [torch.empty_like(d)], sd, info=True)
    assert info.residual <= 1e-5
    g.close()



@pytest.mark.parametrize("grid", ["four_leaves", "spheres", "box", "shell512"])
def test_multigrid_coarse_cluster_bit_exact(dev, grid):
    """The multigrid cycle's coarsest level (one cell per leaf) solved by one thread-block cluster
    launch that holds the level in shared memory (the default) and by two launches per SOR sweep
    relaxes the same cells with the same arithmetic: the mixed step's refined pressure, outer
    iteration count, projected velocity and advected density are identical to the bit. Cases:
    fewer leaves than the cluster has CTAs (some CTAs hold none), sparse spheres (missing
    neighbours), a box, and the 45,198-leaf shell of the bench (2,825 leaves per CTA of 16)."""
    from hnanosolver_b200 import lib as hl

    if grid == "four_leaves":
        origins = synth.sort_leaves_nanovdb(np.array([[0, 0, 0], [8, 0, 0], [0, 8, 0], [8, 8, 8]], dtype=np.int32))
    elif grid == "spheres":
        origins = synth.spheres_topology(96, 3, 8.0, 20.0, seed=11)
    elif grid == "box":
        origins = synth.topology("box64")
    else:
        origins = synth.topology("shell512")
    dens, vel = synth.noise_fields(origins, seed=7)
    vb = torch.from_numpy(vel).to(dev).to(torch.bfloat16).contiguous()
    dh = torch.from_numpy(dens).to(dev).to(torch.float16).contiguous()
    out = {}
    for form in (hl.COARSE_LAUNCHES, hl.COARSE_CLUSTER):
        g = hl.Grid(origins, voxel_size=0.1)
        g.set_option(hl.OPT_COARSE_SOLVE, form)
        vo, do = torch.empty_like(vb), torch.empty_like(dh)
        desc = hl.MixedDesc(dt=0.1, omega=1.9, tolerance=1e-5, max_outer=40, inner_iterations=2,
                            flags=hl.SOLVE_MULTIGRID)
        torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
        info = g.step_mixed(vb, vo, [dh], [do], desc, info=True)
        p = torch.empty(g.num_voxels, dtype=torch.float64, device=dev)
        outer, res = g.refine_pressure(p)
        torch.cuda.synchronize()
        out[form] = (vo.cpu(), do.cpu(), p.cpu(), outer, info.residual)
        g.close()
    a, b = out[hl.COARSE_LAUNCHES], out[hl.COARSE_CLUSTER]
    assert a[3] == b[3]
    assert torch.equal(a[2], b[2])
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    assert b[4] <= 1e-5


@pytest.mark.parametrize("flags", [0, 8])
def test_l2_persistence_same_results(dev, shell, flags):
    """HNS_OPT_L2_PERSIST (the inner solve's FP16 correction array marked persisting in L2 for
    the solve's launches; the default where it fits) changes caching only: the mixed step with
    red-black (flags 0) or multigrid (HNS_SOLVE_MULTIGRID = 8) inner solves gives the same
    pressure, outer count, velocity and density to the bit as with ordinary caching."""
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    out = {}
    for persist in (0, 1):
        g = hl.Grid(origins, voxel_size=0.1)
        g.set_option(hl.OPT_L2_PERSIST, persist)
        vb, dh, vo, do, info = _mixed(g, dev, dens, vel, inner=2 if flags else 30, outer=12, flags=flags)
        p = torch.empty(g.num_voxels, dtype=torch.float64, device=dev)
        outer, res = g.refine_pressure(p)
        torch.cuda.synchronize()
        out[persist] = (vo.cpu(), do.cpu(), p.cpu(), outer)
        g.close()
    a, b = out[0], out[1]
    assert a[3] == b[3]
    assert torch.equal(a[2], b[2]) and torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


def test_multigrid_step_captured_in_a_graph(dev, shell):
    """The multigrid mixed step enqueued into a caller's CUDA graph capture (the cluster launch
    of the coarsest level, the L2 window and the PDL chain captured; no forecast and no spare
    graphs under capture) and replayed gives the eager step's velocity and density to the bit."""
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    g = hl.Grid(origins, voxel_size=0.1)
    s = torch.cuda.Stream()
    g.set_stream(s.cuda_stream)
    vb = torch.from_numpy(vel).to(dev).to(torch.bfloat16).contiguous()
    dh = torch.from_numpy(dens).to(dev).to(torch.float16).contiguous()
    vo, do = torch.empty_like(vb), torch.empty_like(dh)
    desc = hl.MixedDesc(dt=0.1, omega=1.9, tolerance=1e-5, max_outer=8, inner_iterations=2,
                        flags=hl.SOLVE_MULTIGRID)
    torch.cuda.synchronize()
    g.step_mixed(vb, vo, [dh], [do], desc)  # eager: scratch, tables and limits made here
    s.synchronize()
    want_v, want_d = vo.clone(), do.clone()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s, capture_error_mode="relaxed"):
        g.step_mixed(vb, vo, [dh], [do], desc)
    vo.zero_()
    do.zero_()
    torch.cuda.synchronize()
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(vo, want_v) and torch.equal(do, want_d)
    del graph
    g.close()


def test_two_live_grids_of_different_sizes(dev, shell):
    """Two contexts of different leaf counts on one device, stepped alternately with multigrid
    inner solves: the cluster kernel's shared-memory limit and the persisting-L2 limit are
    process-wide settings that a context only raises, so the smaller grid set up second does not
    break the larger one's next step, which repeats its first to the bit."""
    from hnanosolver_b200 import lib as hl

    origins, dens, vel = shell
    small = synth.topology("box64")
    sd, sv = synth.noise_fields(small, seed=3)
    big_g = hl.Grid(origins, voxel_size=0.1)
    small_g = hl.Grid(small, voxel_size=0.1)
    first = _mixed(big_g, dev, dens, vel, inner=2, outer=12, flags=hl.SOLVE_MULTIGRID)
    torch.cuda.synchronize()
    _mixed(small_g, dev, sd, sv, inner=2, outer=12, flags=hl.SOLVE_MULTIGRID)
    again = _mixed(big_g, dev, dens, vel, inner=2, outer=12, flags=hl.SOLVE_MULTIGRID)
    torch.cuda.synchronize()
    assert torch.equal(first[2], again[2]) and torch.equal(first[3], again[3])
    big_g.close()
    small_g.close()
