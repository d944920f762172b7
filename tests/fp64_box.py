"""FP64 restatement, in torch, of the plain step on a box of voxels: MacCormack advection
of the velocity (advect_vector, src/Cuda/Kernel.cu:349-426) and of scalars (advect_scalar,
src/Cuda/Kernel.cu:294-344), divergence (Kernel.cu:432-453), red-black SOR from p = 0
(Kernel.cu:459-489, driven as in src/Cuda/HNanoSolver.cu:366-373) and gradient subtraction
(Kernel.cu:495-541), with every read outside the box 0. The box is fully active, or holds a
sparse grid as a mask of its active voxels (`active`), every read of an inactive voxel 0 as the
reference reads outside its index grid.

Test infrastructure only: it is the checker that makes central finite differences of long
rollouts affordable (a batch of perturbed states steps at once on the device), and it follows
the FP64 oracle (oracle/hns_oracle_impl.h) formula for formula; test_oracle pins it against
that oracle. A field is a dense array over the box, 0 at inactive voxels: scalars (B, X, Y, Z),
velocity (B, 3, X, Y, Z), index (x, y, z) = coordinate - box origin. `solve_exact` (conjugate
gradients to an FP64 residual of 1e-12) gives the projection the iterative solves approach, the
reference point of the field error of a step solved to a tolerance.
"""
import numpy as np
import torch
import torch.nn.functional as F

PAD = 4  # taps up to PAD voxels outside the box read the zero padding; further ones are clamped onto it
NBRS = ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1))  # the clamp's neighbour order


def _index(coords, lo, device) -> torch.Tensor:
    if isinstance(coords, torch.Tensor):
        return coords.to(device=device, dtype=torch.int64) - torch.as_tensor(np.asarray(lo, dtype=np.int64), device=device)
    return torch.as_tensor(np.asarray(coords, dtype=np.int64) - np.asarray(lo, dtype=np.int64), device=device)


def to_dense(values, coords, lo, shape, device, dtype=torch.float64) -> torch.Tensor:
    """Slot-ordered values ((N,) or (N, 3), numpy or torch) -> (1, X, Y, Z) or (1, 3, X, Y, Z)."""
    if isinstance(values, torch.Tensor):
        v = values.to(device=device, dtype=dtype)
    else:
        v = torch.as_tensor(np.asarray(values, dtype=np.float64), device=device, dtype=dtype)
    c = _index(coords, lo, device)
    if v.ndim == 1:
        out = torch.zeros((1,) + tuple(shape), device=device, dtype=dtype)
        out[0, c[:, 0], c[:, 1], c[:, 2]] = v
    else:
        out = torch.zeros((1, 3) + tuple(shape), device=device, dtype=dtype)
        out[0, :, c[:, 0], c[:, 1], c[:, 2]] = v.T
    return out


def from_dense(d: torch.Tensor, coords, lo, numpy: bool = True):
    """(X, Y, Z) or (3, X, Y, Z) -> slot-ordered (N,) or (N, 3) float64 (numpy, or a tensor on
    d's device)."""
    c = _index(coords, lo, d.device)
    out = d[c[:, 0], c[:, 1], c[:, 2]] if d.ndim == 3 else d[:, c[:, 0], c[:, 1], c[:, 2]].T
    return out.cpu().numpy() if numpy else out


def active_mask(coords, lo, shape, device) -> torch.Tensor:
    """The box's active voxels (X, Y, Z) bool, from the grid's voxel coordinates."""
    c = _index(coords, lo, device)
    m = torch.zeros(tuple(shape), dtype=torch.bool, device=device)
    m[c[:, 0], c[:, 1], c[:, 2]] = True
    return m


class Box:
    """Operators on a dense box of the given shape whose first voxel has coordinate `lo`;
    `active` (X, Y, Z) bool marks the grid's voxels (None: all). Inputs are 0 at inactive
    voxels, and so are the outputs."""

    def __init__(self, shape, lo, dx: float, device, active=None):
        self.shape = tuple(int(s) for s in shape)
        self.lo = tuple(int(v) for v in lo)
        self.dx = float(dx)
        self.inv_dx = 1.0 / self.dx
        self.device = device
        X, Y, Z = self.shape
        ax = [torch.arange(n, device=device, dtype=torch.float64) + o for n, o in zip(self.shape, self.lo)]
        self.gx, self.gy, self.gz = torch.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
        par = (self.gx + self.gy + self.gz).long() & 1
        self.active = active
        self.colour = [par == 0, par == 1] if active is None else [(par == 0) & active, (par == 1) & active]

    def _mask(self, f):
        return f if self.active is None else torch.where(self.active, f, torch.zeros((), dtype=f.dtype, device=f.device))

    # ---- reads ----
    @staticmethod
    def _pad1(f):
        return F.pad(f, (1, 1, 1, 1, 1, 1))

    def _nbr(self, fp, di, dj, dk):
        """fp padded by one voxel (..., X+2, Y+2, Z+2) -> the field at (i+di, j+dj, k+dk)."""
        X, Y, Z = self.shape
        return fp[..., 1 + di:1 + di + X, 1 + dj:1 + dj + Y, 1 + dk:1 + dk + Z]

    def _taps(self, x, y, z, floors=None):
        """Flat indices into the PAD-padded volume and fractions of the cells `floors` (default
        floor(x, y, z)); with frozen cells the fractions may leave [0, 1) and the sample
        extends the cell's trilinear polynomial. Returns (taps, floors)."""
        X, Y, Z = self.shape
        sx, sy, sz = X + 2 * PAD, Y + 2 * PAD, Z + 2 * PAD
        fx, fy, fz = floors if floors is not None else (torch.floor(x), torch.floor(y), torch.floor(z))
        tx, ty, tz = x - fx, y - fy, z - fz
        ix = fx.long() - self.lo[0] + PAD
        iy = fy.long() - self.lo[1] + PAD
        iz = fz.long() - self.lo[2] + PAD
        shape = x.shape
        idx = {}
        for a in (0, 1):
            for b in (0, 1):
                for c in (0, 1):
                    # A tap beyond the padding is clamped onto the padding's outer layer (zeros).
                    qx = (ix + a).clamp(0, sx - 1)
                    qy = (iy + b).clamp(0, sy - 1)
                    qz = (iz + c).clamp(0, sz - 1)
                    idx[(a, b, c)] = (((qx * sy) + qy) * sz + qz).expand(shape).reshape(shape[0], -1)
        return (idx, tx, ty, tz), (fx, fy, fz)

    def _sample(self, f, taps):
        """Lerp-chain trilinear sample (z, then y, then x) of scalar field f (B, X, Y, Z)."""
        idx, tx, ty, tz = taps
        B = f.shape[0]
        fp = F.pad(f, (PAD,) * 6).reshape(B, -1)

        def v(a, b, c):
            return torch.gather(fp, 1, idx[(a, b, c)]).reshape(f.shape)

        def lerp(a, b, w):
            return a + w * (b - a)

        z0 = lerp(v(0, 0, 0), v(0, 0, 1), tz)
        z1 = lerp(v(0, 1, 0), v(0, 1, 1), tz)
        z2 = lerp(v(1, 0, 0), v(1, 0, 1), tz)
        z3 = lerp(v(1, 1, 0), v(1, 1, 1), tz)
        return lerp(lerp(z0, z1, ty), lerp(z2, z3, ty), tx)

    # ---- advection ----
    def _clamp(self, po, pf, pb, sel=None):
        """MacCormack correction clamped to [min, max] of the centre, its 6 face neighbours and
        the forward sample. Returns (value, selection): which candidate the clamp returned
        (0 centre, 1..6 the neighbours -x, +x, -y, +y, -z, +z, 7 the forward sample, 8 the
        correction). With `sel` given the same candidates are returned whatever the values."""
        corr = pf + 0.5 * (po - pb)
        pp = self._pad1(po)
        cands = [po] + [self._nbr(pp, *d) for d in NBRS] + [pf, corr]
        if sel is not None:
            return torch.gather(torch.stack(cands), 0, sel.expand(po.shape).unsqueeze(0)).squeeze(0), sel
        C = torch.stack(cands[:8])
        mn, imn = C.min(dim=0)
        mx, imx = C.max(dim=0)
        out = torch.maximum(mn, torch.minimum(corr, mx))
        sel = torch.where(corr > mx, imx, torch.where(corr < mn, imn, torch.full_like(imn, 8)))
        return out, sel

    def advect(self, vel, scalars, dt, frozen=None):
        """MacCormack advection of vel (B, 3, X, Y, Z) and of each scalar along it. Returns
        (velocity, [scalars], decisions): the cells of both traces and the clamp selections.
        With `frozen` (decisions of an earlier call, batch 1) those are reused."""
        sdt = dt * self.inv_dx
        fr = frozen or {}
        bx = self.gx - vel[:, 0] * sdt
        by = self.gy - vel[:, 1] * sdt
        bz = self.gz - vel[:, 2] * sdt
        tb, fb = self._taps(bx, by, bz, fr.get("back"))
        vf = torch.stack([self._sample(vel[:, c], tb) for c in range(3)], dim=1)
        tf, ff = self._taps(bx + vf[:, 0] * sdt, by + vf[:, 1] * sdt, bz + vf[:, 2] * sdt, fr.get("fwd"))
        vsel, vout = [], []
        for c in range(3):
            o, sc = self._clamp(vel[:, c], vf[:, c], self._sample(vel[:, c], tf), fr["vel"][c] if fr else None)
            vout.append(o)
            vsel.append(sc)
        ssel, souts = [], []
        for q, s in enumerate(scalars):
            o, sc = self._clamp(s, self._sample(s, tb), self._sample(s, tf), fr["scalars"][q] if fr else None)
            souts.append(o)
            ssel.append(sc)
        souts = [self._mask(o) for o in souts]
        return self._mask(torch.stack(vout, dim=1)), souts, {"back": fb, "fwd": ff, "vel": vsel, "scalars": ssel}

    # ---- projection ----
    def divergence(self, vel):
        out = torch.zeros_like(vel[:, 0])
        for c, d in enumerate(((1, 0, 0), (0, 1, 0), (0, 0, 1))):
            u = vel[:, c]
            up = self._pad1(u)
            p = (u + self._nbr(up, *d)) * 0.5
            m = (u + self._nbr(up, -d[0], -d[1], -d[2])) * 0.5
            out = out + (p - m)
        return self._mask(out * self.inv_dx)

    def rbgs(self, div, iterations, omega):
        """Red-black SOR from p = 0 (colour 0 first), p + omega (pgs - p) written as
        (1 - omega) p + omega / 6 (sum - div dx^2), in place in a zero-bordered buffer."""
        X, Y, Z = self.shape
        P = torch.zeros((div.shape[0], X + 2, Y + 2, Z + 2), dtype=div.dtype, device=div.device)
        p = P[:, 1:-1, 1:-1, 1:-1]
        w6 = omega / 6.0
        c = div * (w6 * self.dx * self.dx)
        s = torch.empty_like(div)
        for _ in range(iterations):
            for colour in (0, 1):
                torch.add(P[:, 2:, 1:-1, 1:-1], P[:, :-2, 1:-1, 1:-1], out=s)
                s.add_(P[:, 1:-1, 2:, 1:-1]).add_(P[:, 1:-1, :-2, 1:-1]).add_(P[:, 1:-1, 1:-1, 2:])
                s.add_(P[:, 1:-1, 1:-1, :-2])
                s.mul_(w6).sub_(c).add_(p, alpha=1.0 - omega)
                torch.where(self.colour[colour], s, p, out=p)
        return p.contiguous()

    def subtract_gradient(self, vel, p):
        h = 0.5 * self.inv_dx
        pp = self._pad1(p)
        g = [(self._nbr(pp, *d) - self._nbr(pp, -d[0], -d[1], -d[2])) * h
             for d in ((1, 0, 0), (0, 1, 0), (0, 0, 1))]
        return self._mask(vel - torch.stack(g, dim=1))

    def project(self, vel, iterations, omega):
        return self.subtract_gradient(vel, self.rbgs(self.divergence(vel), iterations, omega))

    def laplacian(self, p):
        """L p = the six face neighbours' sum - 6 p (0 outside the grid), at the active voxels."""
        pp = self._pad1(p)
        s = self._nbr(pp, 1, 0, 0) + self._nbr(pp, -1, 0, 0) + self._nbr(pp, 0, 1, 0) + self._nbr(pp, 0, -1, 0)
        s = s + self._nbr(pp, 0, 0, 1) + self._nbr(pp, 0, 0, -1)
        return self._mask(s - 6.0 * p)

    def solve_exact(self, div, tol: float = 1e-12, max_iterations: int = 20000):
        """p with L p = div dx^2 to a relative FP64 residual |b - L p| / |b| <= tol, by conjugate
        gradients on -L (symmetric positive definite with p = 0 outside the grid), from p = 0.
        Returns (p, iterations, relative residual)."""
        b = -div * (self.dx * self.dx)
        p = torch.zeros_like(b)
        r = b.clone()
        d = r.clone()
        bb = float((b * b).sum())
        if bb == 0.0:
            return p, 0, 0.0
        rr = bb
        it = 0
        while it < max_iterations and rr > tol * tol * bb:
            q = -self.laplacian(d)
            a = rr / float((d * q).sum())
            p.add_(d, alpha=a)
            r.sub_(q, alpha=a)
            rr_new = float((r * r).sum())
            d.mul_(rr_new / rr).add_(r)
            rr = rr_new
            it += 1
        res = self.laplacian(p) - div * (self.dx * self.dx)
        return p, it, float(torch.sqrt((res * res).sum() / bb))

    def project_exact(self, vel, tol: float = 1e-12):
        """The projection with the exact solve. Returns (velocity, iterations, residual)."""
        p, it, res = self.solve_exact(self.divergence(vel), tol)
        return self.subtract_gradient(vel, p), it, res

    def step(self, vel, scalars, dt, iterations, omega, frozen=None):
        """The plain step: advect (velocity and scalars along the incoming velocity), project.
        Returns (velocity, [scalars], decisions), decisions as in advect."""
        v, s, dec = self.advect(vel, scalars, dt, frozen)
        return self.project(v, iterations, omega), s, dec
