"""The all-in-one step on reduced-precision storage (hns_advance_mixed: BF16 velocity, FP16
density/temperature/fuel/flame/waste, FP32 arithmetic, FP64-refined pressure solves) against
the FP64 oracle (hnso_hns_advance_model_f64 on the same BF16/FP16 inputs, its solves run with
omega 1.9 for enough iterations to converge far below the tolerance).

Error statements checked per call (each call starts both sides from the device's previous
output, so the errors do not compound), as max |mixed - FP64| / max |FP64|:
  * velocity <= 2e-2: three BF16 roundings (advection, confinement, buoyancy) of 8
    significant bits, and the solve's 1e-5 residual;
  * scalars <= 5e-3: FP16 storage (11 significant bits) of the burned and advected fields;
  * the refined solve's own FP64 residual <= 1e-5 for every solve (the convergence log).
The measured errors are printed (pytest -s)."""
import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5
VEL_TOL = 2e-2
SCALAR_TOL = 5e-3


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _params(**kw):
    from oracle.binding import CombustionParams as OP

    from hnanosolver_b200.lib import CombustionParams

    p = OP.houdini_defaults()
    p.buoyancyStrength = 0.5
    p.ambientTemp = 0.0
    p.vorticityScale = 0.3
    p.factorScale = 1.0
    p.disturbanceEnable = 0.0
    p.gravity = 0.0
    for k, v in kw.items():
        setattr(p, k, v)
    return p, CombustionParams.from_buffer_copy(bytes(p))


def _to_dev(dev, fields):
    out = {}
    for k, a in fields.items():
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev)
        out[k] = (t.to(torch.bfloat16) if k == "velocity" else t.to(torch.float16)).reshape(-1).contiguous()
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    return out


def _host64(t, n):
    a = t.double().cpu().numpy()
    return a.reshape(n, 3) if a.size == 3 * n else a


@pytest.mark.parametrize("combustion,alpha,substeps,disturbance,factor,multigrid",
                         [(1, 0.1, 1, 0.0, 1.0, False), (0, 0.1, 1, 0.0, 1.0, False), (1, 0.0, 2, 1.0, 1.0, False),
                          (2, 0.1, 1, 0.0, 1.0, False), (1, 0.1, 1, 0.0, 2.0, False), (1, 0.1, 1, 0.0, 1.0, True),
                          (0, 0.1, 1, 0.0, 1.0, True), (1, 0.0, 2, 1.0, 1.0, True)])
def test_fire_mixed_against_fp64_oracle(dev, oracle, combustion, alpha, substeps, disturbance, factor, multigrid):
    from oracle.binding import ForceModel as OM

    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(80, 3, 8.0, 18.0, seed=6)
    dens, vel = synth.smoothed_fields(origins, seed=11, box_passes=2)
    n = len(dens)
    coords = synth.leaf_dense_coords(origins)
    centres, _ = synth.spheres(80, 3, 8.0, 18.0, 6)
    mask = synth.sphere_mask(origins, centres[0], 6.0)
    # Smooth fields (value noise), so that the error statement measures precision rather than
    # the displacement of a per-voxel discontinuity by a BF16-rounded velocity.
    state = {"velocity": (vel * 5.0).astype(np.float32), "density": dens,
             "temperature": (1.5 * synth.value_noise(coords, 21)).astype(np.float32),
             "fuel": np.maximum(0.0, synth.value_noise(coords, 22) - 0.3).astype(np.float32),
             "flame": np.zeros(n, np.float32)}
    if combustion == 0:
        state["waste"] = (0.3 * synth.value_noise(coords, 23)).astype(np.float32)
    if combustion == 2:
        del state["fuel"]
    sources = {"fuel": mask, "temperature": mask * np.float32(2.0)}
    op, params = _params(substeps=substeps, disturbanceEnable=disturbance, factorScale=factor)
    om = OM(combustion=combustion, burn_rate=0.5, heat_release=1.0, ignition_temp=0.0, density_buoyancy=alpha,
            omega=1.9)
    gm = hl.ForceModel(combustion=combustion, burn_rate=0.5, heat_release=1.0, ignition_temp=0.0,
                       density_buoyancy=alpha)
    if multigrid:  # two V-cycles per outer step
        desc = hl.MixedDesc(dt=0.0, omega=1.9, tolerance=TOL, max_outer=12, inner_iterations=2, flags=hl.SOLVE_MULTIGRID)
    else:
        desc = hl.MixedDesc(dt=0.0, omega=1.9, tolerance=TOL, max_outer=12, inner_iterations=30, flags=0)
    grid = hl.Grid(origins, voxel_size=0.1)
    t = oracle.topo(origins)
    cur = _to_dev(dev, state)
    src = _to_dev(dev, sources)
    dt = 1.0 / 24.0
    grid.solve_log(capacity=0, reset=True)
    for call in range(3):
        nxt = {k: torch.empty_like(v) for k, v in cur.items()}
        torch.cuda.synchronize()
        info = grid.advance_mixed(cur, nxt, src, dt, params, gm, desc, info=True)
        assert info.residual <= TOL
        grid.synchronize()
        # The FP64 oracle from the same (BF16/FP16-valued) inputs.
        h = {k: _host64(v, n) for k, v in cur.items()}
        s64 = {"src_" + k: _host64(v, n) for k, v in src.items()}
        scal = {k: v for k, v in h.items() if k != "velocity"}
        v64, sc64, made = t.hns_advance_model(h["velocity"], scal, s64, 0.1, 3000, dt, op, om, dtype=np.float64)
        assert not made
        errs = {"velocity": rel_err(_host64(nxt["velocity"], n), v64)}
        for k in sc64:
            errs[k] = rel_err(_host64(nxt[k], n), sc64[k])
        print(f"call {call}: field errors vs FP64 {errs}, residual {info.residual:.2e}")
        assert errs["velocity"] <= VEL_TOL, errs
        for k in sc64:
            assert errs[k] <= SCALAR_TOL, (k, errs)
        cur = nxt
    count, entries = grid.solve_log()
    assert count == 3 * substeps * (2 if disturbance > 0 else 1)
    assert all(e.residual <= TOL for e in entries)
    grid.close()


def test_fire_mixed_rejects_bad_fields(dev):
    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(64, 2, 8.0, 14.0, seed=8)
    n = 512 * len(origins)
    grid = hl.Grid(origins, voxel_size=0.1)
    v = torch.zeros(3 * n, dtype=torch.bfloat16, device=dev)
    v2 = torch.zeros_like(v)
    h = [torch.zeros(n, dtype=torch.float16, device=dev) for _ in range(4)]
    _, params = _params()
    desc = hl.MixedDesc(dt=0.0, omega=1.9, tolerance=TOL, max_outer=4, inner_iterations=10, flags=0)
    rate = hl.ForceModel(combustion=1, burn_rate=0.5, heat_release=1.0)
    cases = [
        ({"velocity": v}, {"velocity": v2}, rate),                                     # no temperature
        ({"velocity": v, "temperature": h[0]}, {"velocity": v2, "temperature": h[1]}, rate),  # rate burn, no fuel
        ({"velocity": v, "temperature": h[0]}, {"velocity": v, "temperature": h[1]}, None),   # velocity aliases
        ({"velocity": v, "temperature": h[0], "density": h[2]}, {"velocity": v2, "temperature": h[1]}, None),
    ]
    for fin, fout, model in cases:
        with pytest.raises(hl.HnsError) as e:
            grid.advance_mixed(fin, fout, None, 0.1, params, model if model is not None else hl.ForceModel(combustion=2),
                               desc)
        assert e.value.status == 1
    grid.close()


def test_fire_mixed_host_equals_device(dev):
    """hns_advance_mixed_host (FP32 host arrays, converted on the device) gives the device form's
    result on the same rounded inputs, to the bit."""
    from hnanosolver_b200 import lib as hl

    origins = synth.spheres_topology(80, 3, 8.0, 18.0, seed=9)
    dens, vel = synth.smoothed_fields(origins, seed=4, box_passes=2)
    coords = synth.leaf_dense_coords(origins)
    centres, _ = synth.spheres(80, 3, 8.0, 18.0, 9)
    mask = synth.sphere_mask(origins, centres[0], 6.0)
    host = {"velocity": (vel * 5.0).astype(np.float32), "density": dens,
            "temperature": (1.5 * synth.value_noise(coords, 31)).astype(np.float32),
            "fuel": np.maximum(0.0, synth.value_noise(coords, 32) - 0.3).astype(np.float32),
            "flame": np.zeros(len(dens), np.float32)}
    sources = {"fuel": mask, "temperature": mask * np.float32(2.0)}
    _, params = _params()
    model = hl.ForceModel(combustion=1, burn_rate=0.5, heat_release=1.0, density_buoyancy=0.1)
    desc = hl.MixedDesc(dt=0.0, omega=1.9, tolerance=TOL, max_outer=12, inner_iterations=30, flags=0)
    grid = hl.Grid(origins, voxel_size=0.1)
    cur = _to_dev(dev, host)
    src = _to_dev(dev, sources)
    nxt = {k: torch.empty_like(v) for k, v in cur.items()}
    torch.cuda.synchronize()
    grid.advance_mixed(cur, nxt, src, 1.0 / 24.0, params, model, desc)
    grid.synchronize()
    hf = {k: np.ascontiguousarray(v.reshape(-1)).copy() for k, v in host.items()}
    info = grid.advance_mixed_host(hf, sources, 1.0 / 24.0, params, model, desc, info=True)
    assert info.residual <= TOL
    for k, t in nxt.items():
        assert np.array_equal(hf[k], t.float().cpu().numpy()), k
    grid.close()
