"""Adjoint kernels (hns_adjoint_*), through the C ABI.

- Linear operators (divergence, gradient subtraction, the red-black solve from p = 0, the
  projection): the adjoint is the transpose of the forward kernel, <A x, y> = <x, A^T y>.
- Nonlinear operators (MacCormack advection of a scalar and of the velocity, vorticity
  confinement, the whole plain step): vector-Jacobian products against central finite
  differences of the FP64 oracle, on a ragged sparse grid, at 64 seeded entries per input.
- Rollouts: K plain steps differentiated through a torch.autograd.Function that keeps a
  checkpoint every few steps and recomputes the rest in the backward pass; the loss is
  1/2 |rho_K - rho_target|^2 and its gradients with respect to the initial density and
  velocity are checked against central finite differences of the FP64 box restatement of
  the step (fp64_box, itself pinned to the oracle): with h = 1e-3 through the unperturbed
  trajectory's branch decisions (trace cells, MacCormack clamp selections), the derivative
  the adjoint takes, and with h = 1e-6 through the free function. Free differences with
  h = 1e-3 straddle clamp switches and cell crossings (the step is only piecewise smooth)
  and differ from every derivative by up to a few percent, so they are not a check.
"""
import numpy as np
import pytest

from conftest import rel_err
from hnanosolver_b200 import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FD_TOL = 1e-3  # max |adjoint - finite difference| / max |finite difference|
DOT_TOL = 1e-5  # |<A x, y> - <x, A^T y>| / sum |terms|
DX, INV_DX = 0.1, 10.0


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.fixture(scope="module")
def ragged():
    """42 leaves around two seeded spheres in a 40^3 box (21,504 voxels, ragged walls).
    Velocities scaled to about half a voxel per step so that traces cross cells and leave
    the domain."""
    origins = synth.spheres_topology(40, 2, 8.0, 14.0, 3)
    dens, vel = synth.smoothed_fields(origins, seed=0, box_passes=3)
    return origins, dens, np.ascontiguousarray(vel * 8.0, dtype=np.float32)


def _grid(origins):
    """A grid whose calls run on torch's current stream, so that they are ordered with the
    torch operations (zeroing, copies) around them."""
    from hnanosolver_b200 import lib as hl

    g = hl.Grid(origins, voxel_size=DX)
    # torch's default stream has handle 0, which hns_set_stream reads as "the grid's own
    # stream"; that stream is the legacy default stream, cudaStreamLegacy = (cudaStream_t)1.
    g.set_stream(torch.cuda.current_stream().cuda_stream or 1)
    return g


def _t(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _np(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.float64)


def _dot(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(a @ b), float(np.abs(a * b).sum())


def _assert_transpose(lhs, rhs):
    (x, sx), (y, sy) = lhs, rhs
    assert abs(x - y) <= DOT_TOL * max(sx, sy), (x, y, sx)


def _fd(field_fn, w, x, flat_idx, h=1e-6):
    """Central differences of sum(w * field_fn(x)) at x along the flat entries flat_idx, with
    the difference of the two perturbed fields taken before the sum."""
    x = np.array(x, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    g = np.empty(len(flat_idx))
    for q, i in enumerate(flat_idx):
        xp, xm = x.copy(), x.copy()
        xp.flat[i] += h
        xm.flat[i] -= h
        g[q] = float(np.sum(w * (field_fn(xp) - field_fn(xm)))) / (2.0 * h)
    return g


def _entries(rng, n, vec3):
    s = rng.choice(n, 64, replace=False)
    return 3 * s + rng.integers(0, 3, 64) if vec3 else s


# ---- linear operators: transposes ---------------------------------------------------------


def test_divergence_adjoint_is_transpose(dev, ragged):
    origins = ragged[0]
    g = _grid(origins)
    n = 512 * len(origins)
    rng = np.random.default_rng(11)
    v = rng.standard_normal((n, 3)).astype(np.float32)
    w = rng.standard_normal(n).astype(np.float32)
    div = torch.empty(n, device=dev)
    g.divergence(_t(v, dev), div)
    vb = torch.zeros((n, 3), device=dev)
    g.adjoint_divergence(_t(w, dev), vb)
    _assert_transpose(_dot(_np(div), w), _dot(v, _np(vb)))
    g.close()


def test_gradient_adjoint_is_transpose(dev, ragged):
    origins = ragged[0]
    g = _grid(origins)
    n = 512 * len(origins)
    rng = np.random.default_rng(12)
    p = rng.standard_normal(n).astype(np.float32)
    u = rng.standard_normal((n, 3)).astype(np.float32)
    out = torch.empty((n, 3), device=dev)
    g.subtract_gradient(torch.zeros((n, 3), device=dev), _t(p, dev), out)  # out = -grad p
    pb, vb = torch.zeros(n, device=dev), torch.zeros((n, 3), device=dev)
    g.adjoint_subtract_gradient(_t(u, dev), vb, pb)
    _assert_transpose(_dot(_np(out), u), _dot(p, _np(pb)))
    assert np.array_equal(_np(vb), u.astype(np.float64))  # d out / d vel = I
    g.close()


@pytest.mark.parametrize("iterations,omega", [(1, 1.0), (7, 1.4), (40, 1.6)])
def test_rbgs_adjoint_is_transpose(dev, ragged, iterations, omega):
    from hnanosolver_b200 import lib as hl

    origins = ragged[0]
    g = _grid(origins)
    n = 512 * len(origins)
    rng = np.random.default_rng(13)
    b = rng.standard_normal(n).astype(np.float32)
    w = rng.standard_normal(n).astype(np.float32)
    p = torch.empty(n, device=dev)
    g.rbgs(_t(b, dev), p, iterations, omega, flags=hl.SOLVE_ZERO_INIT)
    db = torch.zeros(n, device=dev)
    g.adjoint_rbgs(_t(w, dev), db, iterations, omega)
    _assert_transpose(_dot(_np(p), w), _dot(b, _np(db)))
    g.close()


def test_project_adjoint_is_transpose(dev, ragged):
    origins = ragged[0]
    g = _grid(origins)
    n = 512 * len(origins)
    rng = np.random.default_rng(14)
    v = rng.standard_normal((n, 3)).astype(np.float32)
    w = rng.standard_normal((n, 3)).astype(np.float32)
    vp = _t(v, dev).clone()
    g.project(vp, 20, 1.2, info=False)
    wb = _t(w, dev).clone()
    g.adjoint_project(wb, 20, 1.2)
    _assert_transpose(_dot(_np(vp), w), _dot(v, _np(wb)))
    g.close()


def test_adjoint_rejects_bad_arguments(dev, ragged):
    from hnanosolver_b200 import lib as hl

    g = _grid(ragged[0])
    n = 512 * len(ragged[0])
    a = torch.zeros(n, device=dev)
    with pytest.raises(hl.HnsError):
        g.adjoint_rbgs(a, a.clone(), -1, 1.0)
    with pytest.raises(hl.HnsError):
        g.adjoint_divergence(a, None)
    g.close()


# ---- nonlinear operators: finite differences of the FP64 oracle ---------------------------


def test_advect_scalar_adjoint_matches_fd(dev, oracle, ragged):
    origins, dens, vel = ragged
    g = _grid(origins)
    n, dt = len(dens), 0.1
    rng = np.random.default_rng(21)
    w = rng.standard_normal(n).astype(np.float32)
    in_bar, vel_bar = torch.zeros(n, device=dev), torch.zeros((n, 3), device=dev)
    g.adjoint_advect_scalar(_t(vel, dev), _t(dens, dev), _t(w, dev), in_bar, vel_bar, dt)
    t = oracle.topo(origins)
    v64, d64 = vel.astype(np.float64), dens.astype(np.float64)
    si, vi = _entries(rng, n, False), _entries(rng, n, True)
    fd_in = _fd(lambda x: t.advect_scalar(v64, x, dt, INV_DX), w, d64, si)
    fd_vel = _fd(lambda x: t.advect_scalar(x, d64, dt, INV_DX), w, v64, vi)
    assert rel_err(_np(in_bar).ravel()[si], fd_in) <= FD_TOL
    assert rel_err(_np(vel_bar).ravel()[vi], fd_vel) <= FD_TOL
    g.close()


def test_advect_vec3_adjoint_matches_fd(dev, oracle, ragged):
    origins, _, vel = ragged
    g = _grid(origins)
    n, dt = len(vel), 0.1
    rng = np.random.default_rng(22)
    w = rng.standard_normal((n, 3)).astype(np.float32)
    vel_bar = torch.zeros((n, 3), device=dev)
    g.adjoint_advect_vec3(_t(vel, dev), _t(w, dev), vel_bar, dt)
    t = oracle.topo(origins)
    vi = _entries(rng, n, True)
    fd = _fd(lambda x: t.advect_vector(x, dt, INV_DX), w, vel.astype(np.float64), vi)
    assert rel_err(_np(vel_bar).ravel()[vi], fd) <= FD_TOL
    g.close()


@pytest.mark.parametrize("factor_scale", [1.0, 2.0, 0.5])
def test_confinement_adjoint_matches_fd(dev, oracle, ragged, factor_scale):
    """eps 0.3, dt 1/24; the |omega| gradient is taken int(factor_scale) voxels away (0.5 gives
    offset 0: no force and a zero adjoint beyond the identity)."""
    origins, _, vel = ragged
    g = _grid(origins)
    n, dt, scale = len(vel), 1.0 / 24.0, 0.3
    rng = np.random.default_rng(23)
    w = rng.standard_normal((n, 3)).astype(np.float32)
    vel_bar = torch.zeros((n, 3), device=dev)
    g.adjoint_vorticity_confinement(_t(vel, dev), _t(w, dev), vel_bar, dt, scale, factor_scale)
    t = oracle.topo(origins)
    vi = _entries(rng, n, True)
    fd = _fd(lambda x: t.vorticity_confinement(x, dt, INV_DX, scale, factor_scale), w, vel.astype(np.float64), vi)
    got = _np(vel_bar).ravel()[vi]
    assert rel_err(got, fd) <= FD_TOL
    if factor_scale < 1.0:
        assert np.allclose(got, w.astype(np.float64).ravel()[vi], rtol=0, atol=1e-6)
    g.close()


def test_step_adjoint_matches_fd(dev, oracle, ragged):
    """hns_adjoint_step_plain: advect (velocity and density) then project, 20 iterations."""
    origins, dens, vel = ragged
    g = _grid(origins)
    n, dt, iters, omega = len(dens), 0.1, 20, 1.0
    rng = np.random.default_rng(24)
    wv = rng.standard_normal((n, 3)).astype(np.float32)
    wd = rng.standard_normal(n).astype(np.float32)
    vb, db = torch.zeros((n, 3), device=dev), torch.zeros(n, device=dev)
    g.adjoint_step_plain(_t(vel, dev), [_t(dens, dev)], _t(wv, dev), [_t(wd, dev)], vb, [db], dt, iters, omega)
    t = oracle.topo(origins)
    v64, d64 = vel.astype(np.float64), dens.astype(np.float64)

    def step(v, d):
        out_v, _, _ = t.project(t.advect_vector(v, dt, INV_DX), DX, iters, omega)
        return out_v, t.advect_scalar(v, d, dt, INV_DX)

    def both(v, d):
        out_v, out_d = step(v, d)
        return np.concatenate([out_v.ravel(), out_d])

    w = np.concatenate([wv.ravel(), wd])
    si, vi = _entries(rng, n, False), _entries(rng, n, True)
    fd_d = _fd(lambda x: both(v64, x), w, d64, si)
    fd_v = _fd(lambda x: both(x, d64), w, v64, vi)
    assert rel_err(_np(db)[si], fd_d) <= FD_TOL
    assert rel_err(_np(vb).ravel()[vi], fd_v) <= FD_TOL
    g.close()


# ---- rollouts: a checkpointing autograd.Function ------------------------------------------


def _step(grid, v, d, desc):
    v2, d2 = torch.empty_like(v), torch.empty_like(d)
    grid.step_plain(v, v2, [d], [d2], desc)
    return v2, d2


class Rollout(torch.autograd.Function):
    """`steps` plain steps of (velocity, density) through the C ABI. The forward keeps the
    state at every `every`-th step; the backward walks the segments in reverse, recomputes the
    inputs of a segment's steps from its checkpoint, and runs hns_adjoint_step_plain on them
    in reverse order."""

    recomputed = 0

    @staticmethod
    def forward(ctx, vel0, dens0, grid, steps, every, desc):
        v, d = vel0.detach().contiguous(), dens0.detach().contiguous()
        ckpt = []
        for k in range(steps):
            if k % every == 0:
                ckpt.append((v.clone(), d.clone()))
            v, d = _step(grid, v, d, desc)
        ctx.grid, ctx.steps, ctx.every, ctx.desc, ctx.ckpt = grid, steps, every, desc, ckpt
        return v, d

    @staticmethod
    def backward(ctx, gv, gd):
        g, desc = ctx.grid, ctx.desc
        vb, db = gv.contiguous().clone(), gd.contiguous().clone()
        for seg in reversed(range(len(ctx.ckpt))):
            k0 = seg * ctx.every
            k1 = min(k0 + ctx.every, ctx.steps)
            states = [ctx.ckpt[seg]]
            for _ in range(k0, k1 - 1):
                states.append(_step(g, *states[-1], desc))
                Rollout.recomputed += 1
            for v_in, d_in in reversed(states):
                vin_bar, din_bar = torch.zeros_like(vb), torch.zeros_like(db)
                g.adjoint_step_plain(v_in, [d_in], vb, [db], vin_bar, [din_bar], desc.dt, desc.max_iterations,
                                     desc.omega)
                vb, db = vin_bar, din_bar
        ctx.ckpt = None
        return vb, db, None, None, None, None


def _desc(dt, iters, omega):
    from hnanosolver_b200.lib import StepDesc

    return StepDesc(dt=dt, max_iterations=iters, omega=omega, tolerance=0.0, check_every=0, flags=0)


def _rollout_grads(dev, origins, dens, vel, target, steps, every, desc):
    g = _grid(origins)
    v0 = _t(vel, dev).requires_grad_(True)
    d0 = _t(dens, dev).requires_grad_(True)
    vK, dK = Rollout.apply(v0, d0, g, steps, every, desc)
    loss = 0.5 * ((dK - _t(target, dev)) ** 2).sum()
    loss.backward()
    out = _np(v0.grad), _np(d0.grad), _np(dK)
    g.close()
    return out


class _BoxRollout:
    """The rollout of the loss 1/2 |rho_K - target|^2 in the FP64 box restatement, with the
    unperturbed trajectory's decisions (trace cells, clamp selections) recorded per step."""

    def __init__(self, dev, origins, dens, vel, target, steps, iters, omega, dt):
        from fp64_box import Box, from_dense, to_dense

        coords = synth.leaf_dense_coords(origins)
        lo = coords.min(axis=0)
        shape = tuple(int(s) for s in coords.max(axis=0) - lo + 1)
        assert np.prod(shape) == len(coords), "the FP64 box restatement needs a fully active box"
        self.box = Box(shape, lo, DX, dev)
        self.V = to_dense(vel, coords, lo, shape, dev)
        self.D = to_dense(dens, coords, lo, shape, dev)
        self.T = to_dense(target, coords, lo, shape, dev)
        self.rel = (coords - lo).astype(np.int64)
        self.steps, self.iters, self.omega, self.dt = steps, iters, omega, dt
        self.batch = max(1, min(64, (1 << 25) // len(coords)))  # 2 x batch states of at most 2^26 voxels
        d, self.decisions = self.run(self.V, self.D, record=True)
        self.base = from_dense(d[0], coords, lo)

    def run(self, v, d, record=False, frozen=False):
        rec = []
        for k in range(self.steps):
            v, (d,), dec = self.box.step(v, [d], self.dt, self.iters, self.omega,
                                         self.decisions[k] if frozen else None)
            if record:
                rec.append(dec)
        return d, rec

    def fd(self, entries, h, frozen):
        """Central differences (step h) of the loss along each entry ('v', slot, component) or
        ('d', slot, 0), a batch of perturbed states at a time; with `frozen` the perturbed
        rollouts replay the unperturbed decisions, which makes the loss smooth in h."""
        out = np.empty(len(entries))
        for b0 in range(0, len(entries), self.batch):
            chunk = entries[b0:b0 + self.batch]
            B = len(chunk)
            vp, dp = self.V.repeat(2 * B, 1, 1, 1, 1), self.D.repeat(2 * B, 1, 1, 1)
            for q, (kind, s, c) in enumerate(chunk):
                x, y, z = (int(a) for a in self.rel[s])
                for sgn, row in ((1.0, q), (-1.0, B + q)):
                    if kind == "v":
                        vp[row, c, x, y, z] += sgn * h
                    else:
                        dp[row, x, y, z] += sgn * h
            dk, _ = self.run(vp, dp, frozen=frozen)
            a, m = dk[:B], dk[B:]
            # L(+) - L(-) = 1/2 sum (a - m)(a + m - 2 target), without cancellation.
            diff = 0.5 * ((a - m) * (a + m - 2.0 * self.T)).sum(dim=(1, 2, 3))
            out[b0:b0 + B] = (diff / (2.0 * h)).cpu().numpy()
        return out


def _rollout_case(dev, extent, steps, iters, every, n_slots, n_free, seed=5):
    """Adjoint gradients of a rollout against (1) central differences with h = 1e-3 through the
    unperturbed trajectory's decisions, at n_slots seeded voxels (density and the three
    velocity components), and (2) plain central differences with h = 1e-6 at the first n_free
    of them. Returns the relative errors {(kind, which): err}."""
    origins = synth.sort_leaves_nanovdb(synth._box_leaves(extent))
    dens, vel = synth.smoothed_fields(origins, seed=0, box_passes=3)
    target, _ = synth.smoothed_fields(origins, seed=1, box_passes=3)
    dt, omega = 0.1, 1.0
    desc = _desc(dt, iters, omega)
    Rollout.recomputed = 0
    gv, gd, dK = _rollout_grads(dev, origins, dens, vel, target, steps, every, desc)
    assert Rollout.recomputed == steps - (steps + every - 1) // every
    box = _BoxRollout(dev, origins, dens, vel, target, steps, iters, omega, dt)
    assert rel_err(dK, box.base) <= 1e-4  # the FP32 rollout follows the FP64 one
    rng = np.random.default_rng(seed)
    slots = rng.choice(len(dens), n_slots, replace=False)
    errs = {}
    for kind, sl, h, frozen in (("frozen", slots, 1e-3, True), ("free", slots[:n_free], 1e-6, False)):
        ents = [("d", int(s), 0) for s in sl] + [("v", int(s), c) for s in sl for c in range(3)]
        fd = box.fd(ents, h, frozen)
        adj_v = np.array([gv[s, c] for _, s, c in ents[len(sl):]])
        errs[(kind, "density")] = rel_err(gd[sl], fd[:len(sl)])
        errs[(kind, "velocity")] = rel_err(adj_v, fd[len(sl):])
    print(f"box{extent} rollout: " + ", ".join(f"{k[0]} {k[1]} {v:.2e}" for k, v in errs.items()))
    return errs


def test_rollout_adjoint_box32_matches_fd(dev):
    """16 steps, 60 iterations, a checkpoint every 4 steps, 32^3 fully active box; all 64
    seeded voxels for both differences."""
    errs = _rollout_case(dev, 32, 16, 60, 4, 64, 64)
    assert max(errs.values()) <= FD_TOL, errs


def test_rollout_adjoint_box128_matches_fd(dev):
    """The differentiable-rollout configuration: 128^3 fully active (2,097,152 voxels), 16
    steps of advect + project with 60 iterations, a checkpoint every 4 steps, loss
    1/2 |rho_K - rho_target|^2; central differences with h = 1e-3 at 64 seeded voxels
    (density and the three velocity components), plain h = 1e-6 differences at 16 of them."""
    errs = _rollout_case(dev, 128, 16, 60, 4, 64, 16)
    assert max(errs.values()) <= FD_TOL, errs


def test_rollout_checkpoint_interval_does_not_change_gradients(dev):
    origins = synth.sort_leaves_nanovdb(synth._box_leaves(32))
    dens, vel = synth.smoothed_fields(origins, seed=0, box_passes=3)
    target, _ = synth.smoothed_fields(origins, seed=1, box_passes=3)
    desc = _desc(0.1, 30, 1.0)
    g1 = _rollout_grads(dev, origins, dens, vel, target, 8, 1, desc)
    g3 = _rollout_grads(dev, origins, dens, vel, target, 8, 3, desc)
    assert rel_err(g3[0], g1[0]) <= 1e-5 and rel_err(g3[1], g1[1]) <= 1e-5
