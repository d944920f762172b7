/* Precision-generic body of the CPU oracle (test infrastructure only).
 *
 * Included twice by hns_oracle.c, with R = float / S = _f32 and R = double / S = _f64.
 * Each function restates one reference kernel; the citation is on the function. The
 * arithmetic follows the reference's operation order so that the float build matches the
 * reference to rounding; the double build is the FP64 oracle the error statements use.
 */
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, S)

/* Nearest read, 0 outside the domain: IndexSampler<T,0> (src/Utils/Stencils.hpp:74-93). */
static inline R FN(near_s)(const hnso_topo* t, const R* d, int32_t i, int32_t j, int32_t k) {
    const uint64_t off = hnso_offset(t, i, j, k);
    return off == 0 ? (R)0 : d[off - 1];
}

static inline void FN(near_v)(const hnso_topo* t, const R* d, int32_t i, int32_t j, int32_t k, R v[3]) {
    const uint64_t off = hnso_offset(t, i, j, k);
    if (off == 0) {
        v[0] = v[1] = v[2] = (R)0;
    } else {
        v[0] = d[3 * (off - 1)];
        v[1] = d[3 * (off - 1) + 1];
        v[2] = d[3 * (off - 1) + 2];
    }
}

static inline R FN(lerp)(R a, R b, R w) { return a + w * (b - a); }

/* Trilinear sample: floor, fractional part, then lerp along z, y, x
 * (TrilinearSampler::sample, src/Utils/Stencils.hpp:118-153). */
static R FN(tri_s)(const hnso_topo* t, const R* d, R x, R y, R z) {
    const int32_t i = (int32_t)floor(x), j = (int32_t)floor(y), k = (int32_t)floor(z);
    const R tx = x - (R)i, ty = y - (R)j, tz = z - (R)k;
    const R v000 = FN(near_s)(t, d, i, j, k), v001 = FN(near_s)(t, d, i, j, k + 1);
    const R v010 = FN(near_s)(t, d, i, j + 1, k), v011 = FN(near_s)(t, d, i, j + 1, k + 1);
    const R v100 = FN(near_s)(t, d, i + 1, j, k), v101 = FN(near_s)(t, d, i + 1, j, k + 1);
    const R v110 = FN(near_s)(t, d, i + 1, j + 1, k), v111 = FN(near_s)(t, d, i + 1, j + 1, k + 1);
    const R z0 = FN(lerp)(v000, v001, tz), z1 = FN(lerp)(v010, v011, tz);
    const R z2 = FN(lerp)(v100, v101, tz), z3 = FN(lerp)(v110, v111, tz);
    const R y0 = FN(lerp)(z0, z1, ty), y1 = FN(lerp)(z2, z3, ty);
    return FN(lerp)(y0, y1, tx);
}

static void FN(tri_v)(const hnso_topo* t, const R* d, R x, R y, R z, R out[3]) {
    const int32_t i = (int32_t)floor(x), j = (int32_t)floor(y), k = (int32_t)floor(z);
    const R tx = x - (R)i, ty = y - (R)j, tz = z - (R)k;
    R v[2][2][2][3];
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c) FN(near_v)(t, d, i + a, j + b, k + c, v[a][b][c]);
    for (int q = 0; q < 3; ++q) {
        const R z0 = FN(lerp)(v[0][0][0][q], v[0][0][1][q], tz), z1 = FN(lerp)(v[0][1][0][q], v[0][1][1][q], tz);
        const R z2 = FN(lerp)(v[1][0][0][q], v[1][0][1][q], tz), z3 = FN(lerp)(v[1][1][0][q], v[1][1][1][q], tz);
        const R y0 = FN(lerp)(z0, z1, ty), y1 = FN(lerp)(z2, z3, ty);
        out[q] = FN(lerp)(y0, y1, tx);
    }
}

void FN(hnso_sample_trilinear_scalar)(const hnso_topo* t, const R* data, const R* xyz, int64_t n, R* out) {
    for (int64_t q = 0; q < n; ++q) out[q] = FN(tri_s)(t, data, xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]);
}

void FN(hnso_sample_trilinear_vec3)(const hnso_topo* t, const R* data, const R* xyz, int64_t n, R* out) {
    for (int64_t q = 0; q < n; ++q) FN(tri_v)(t, data, xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2], out + 3 * q);
}

static inline void FN(coord_of)(const hnso_topo* t, int64_t slot, int32_t* i, int32_t* j, int32_t* k) {
    const int32_t* o = hnso_leaf_origin(t, slot >> 9);
    const int32_t n = (int32_t)(slot & 511);
    *i = o[0] + ((n >> 6) & 7);
    *j = o[1] + ((n >> 3) & 7);
    *k = o[2] + (n & 7);
}

static inline R FN(fmin_)(R a, R b) { return a < b ? a : (b < a ? b : (a != a ? b : a)); }
static inline R FN(fmax_)(R a, R b) { return a > b ? a : (b > a ? b : (a != a ? b : a)); }

/* ---- collision (src/Cuda/Kernel.cu:81-158) ----
 * isInCollision: the trilinear SDF sample (0 outside the domain) below 0. */
static int FN(in_collision)(const hnso_topo* t, const R* sdf, R x, R y, R z) { return FN(tri_s)(t, sdf, x, y, z) < (R)0; }

/* getSDFNormal: central differences of the SDF at the voxel's face neighbours times
 * 0.5 inv_dx, normalised when longer than 1e-6, else 0. */
static void FN(sdf_normal)(const hnso_topo* t, const R* sdf, int32_t i, int32_t j, int32_t k, R inv_dx, R n[3]) {
    const R h = (R)0.5 * inv_dx;
    const R g[3] = {(FN(near_s)(t, sdf, i + 1, j, k) - FN(near_s)(t, sdf, i - 1, j, k)) * h,
                    (FN(near_s)(t, sdf, i, j + 1, k) - FN(near_s)(t, sdf, i, j - 1, k)) * h,
                    (FN(near_s)(t, sdf, i, j, k + 1) - FN(near_s)(t, sdf, i, j, k - 1)) * h};
    const R len = SQRT(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    const R inv = len > (R)1e-6f ? (R)1 / len : (R)0; /* Vec3f / s is (1 / s) * v */
    for (int q = 0; q < 3; ++q) n[q] = inv * g[q];
}

/* v (1 - blend) + blend (v - n (v . n)): applyNoSlipBoundary blended in. */
static void FN(no_slip_blend)(R v[3], const R n[3], R blend) {
    const R vdotn = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
    R tg[3];
    for (int q = 0; q < 3; ++q) tg[q] = v[q] - n[q] * vdotn;
    for (int q = 0; q < 3; ++q) v[q] = v[q] * ((R)1 - blend) + tg[q] * blend;
}

/* The velocity treatment after advect_vector (margin 0.1, blend 1 - sdf / 1.5) and after
 * subtractPressureGradient and in enforceCollisionBoundaries (margin 0.1, blend
 * 1 - sdf / 0.1): inside the collider (sdf < 0) the velocity is 0; within the margin the
 * normal component is blended out. */
static void FN(collide)(const hnso_topo* t, const R* sdf, int64_t s, int32_t i, int32_t j, int32_t k, R inv_dx, R ramp,
                        R v[3]) {
    const R d = sdf[s];
    if (d < (R)0) {
        v[0] = v[1] = v[2] = (R)0;
    } else if (d < (R)0.1f) {
        R n[3];
        FN(sdf_normal)(t, sdf, i, j, k, inv_dx, n);
        FN(no_slip_blend)(v, n, (R)1 - d / ramp);
    }
}

/* enforceCollisionBoundaries (src/Cuda/Kernel.cu:133-158), in place. */
void FN(hnso_enforce_collision)(const hnso_topo* t, R* vel, const R* sdf, R inv_dx) {
    const int64_t N = hnso_topo_num_voxels(t);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        FN(collide)(t, sdf, s, i, j, k, inv_dx, (R)0.1f, vel + 3 * s);
    }
}

/* advect_vector (src/Cuda/Kernel.cu:349-426): MacCormack back/forward trace with trilinear
 * velocity, clamped to [min,max] of centre, 6 face neighbours and the forward sample. With a
 * collision SDF (sdf non-NULL): a trace point inside the collider is pulled back (the back
 * position to the voxel, the forward one to the back position) and the result gets the
 * collision treatment (margin 0.1, blend 1 - sdf / 1.5). */
static void FN(advect_vector_impl)(const hnso_topo* t, const R* vel, R* out, R dt, R inv_dx, const R* sdf) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R sdt = dt * inv_dx;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        R vo[3], vf[3], vb[3], back[3], fwd[3], corr[3], mn[3], mx[3];
        FN(near_v)(t, vel, i, j, k, vo);
        back[0] = (R)i - vo[0] * sdt;
        back[1] = (R)j - vo[1] * sdt;
        back[2] = (R)k - vo[2] * sdt;
        if (sdf && FN(in_collision)(t, sdf, back[0], back[1], back[2])) back[0] = (R)i, back[1] = (R)j, back[2] = (R)k;
        FN(tri_v)(t, vel, back[0], back[1], back[2], vf);
        for (int q = 0; q < 3; ++q) fwd[q] = back[q] + vf[q] * sdt;
        if (sdf && FN(in_collision)(t, sdf, fwd[0], fwd[1], fwd[2]))
            for (int q = 0; q < 3; ++q) fwd[q] = back[q];
        FN(tri_v)(t, vel, fwd[0], fwd[1], fwd[2], vb);
        for (int q = 0; q < 3; ++q) {
            corr[q] = vf[q] + (R)0.5 * (vo[q] - vb[q]);
            mn[q] = mx[q] = vo[q];
        }
        for (int dim = 0; dim < 3; ++dim) {
            for (int off = -1; off <= 1; off += 2) {
                R vn[3];
                FN(near_v)(t, vel, i + (dim == 0 ? off : 0), j + (dim == 1 ? off : 0), k + (dim == 2 ? off : 0), vn);
                for (int q = 0; q < 3; ++q) {
                    mn[q] = FN(fmin_)(mn[q], vn[q]);
                    mx[q] = FN(fmax_)(mx[q], vn[q]);
                }
            }
        }
        for (int q = 0; q < 3; ++q) {
            mn[q] = FN(fmin_)(mn[q], vf[q]);
            mx[q] = FN(fmax_)(mx[q], vf[q]);
            corr[q] = FN(fmax_)(mn[q], FN(fmin_)(corr[q], mx[q]));
        }
        if (sdf) FN(collide)(t, sdf, s, i, j, k, inv_dx, (R)1.5f, corr);
        for (int q = 0; q < 3; ++q) out[3 * s + q] = corr[q];
    }
}

void FN(hnso_advect_vector)(const hnso_topo* t, const R* vel, R* out, R dt, R inv_dx) {
    FN(advect_vector_impl)(t, vel, out, dt, inv_dx, NULL);
}

/* Index of a tap for advect_scalars: offset 0 (outside the domain) reads array index 0,
 * i.e. slot 0's value, not zero (src/Cuda/Kernel.cu:229-230, 256-257). */
static inline int64_t FN(tap)(const hnso_topo* t, int32_t i, int32_t j, int32_t k) {
    const uint64_t off = hnso_offset(t, i, j, k);
    return off == 0 ? 0 : (int64_t)(off - 1);
}

static void FN(interp_setup)(const hnso_topo* t, R x, R y, R z, int64_t idx[8], R w[8]) {
    const int32_t i0 = (int32_t)floor(x), j0 = (int32_t)floor(y), k0 = (int32_t)floor(z);
    const int32_t i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
    const R tx = x - (R)i0, ty = y - (R)j0, tz = z - (R)k0;
    const R itx = (R)1 - tx, ity = (R)1 - ty, itz = (R)1 - tz;
    const R w00 = itx * ity, w10 = tx * ity, w01 = itx * ty, w11 = tx * ty;
    w[0] = w00 * itz;
    w[1] = w10 * itz;
    w[2] = w01 * itz;
    w[3] = w11 * itz;
    w[4] = w00 * tz;
    w[5] = w10 * tz;
    w[6] = w01 * tz;
    w[7] = w11 * tz;
    idx[0] = FN(tap)(t, i0, j0, k0);
    idx[1] = FN(tap)(t, i1, j0, k0);
    idx[2] = FN(tap)(t, i0, j1, k0);
    idx[3] = FN(tap)(t, i1, j1, k0);
    idx[4] = FN(tap)(t, i0, j0, k1);
    idx[5] = FN(tap)(t, i1, j0, k1);
    idx[6] = FN(tap)(t, i0, j1, k1);
    idx[7] = FN(tap)(t, i1, j1, k1);
}

/* advect_scalars (src/Cuda/Kernel.cu:163-289), no collision: the back-trace uses the
 * voxel's own velocity, the re-trace the weight-sum trilinear velocity; per field a
 * fused-multiply-add weight sum, MacCormack correction and 7+1 point clamp. */
static void FN(advect_scalars_impl)(const hnso_topo* t, const R* vel, const R* const* in, R* const* out, int nfields,
                                    R dt, R inv_dx, const R* sdf) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R sdt = dt * inv_dx;
    static const int offs[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        const int64_t orig = FN(tap)(t, i, j, k);
        const R* vc = vel + 3 * orig;
        R back[3] = {(R)i - vc[0] * sdt, (R)j - vc[1] * sdt, (R)k - vc[2] * sdt};
        /* With a collision SDF, trace points inside the collider are pulled back (Kernel.cu:192-195, 245-248). */
        if (sdf && FN(in_collision)(t, sdf, back[0], back[1], back[2])) back[0] = (R)i, back[1] = (R)j, back[2] = (R)k;
        int64_t bi[8], fi[8], nb[6];
        R bw[8], fw[8];
        FN(interp_setup)(t, back[0], back[1], back[2], bi, bw);
        R vf[3] = {0, 0, 0};
        for (int q = 0; q < 8; ++q)
            for (int c = 0; c < 3; ++c) vf[c] = vf[c] + vel[3 * bi[q] + c] * bw[q];
        R fwd[3] = {back[0] + vf[0] * sdt, back[1] + vf[1] * sdt, back[2] + vf[2] * sdt};
        if (sdf && FN(in_collision)(t, sdf, fwd[0], fwd[1], fwd[2]))
            for (int q = 0; q < 3; ++q) fwd[q] = back[q];
        FN(interp_setup)(t, fwd[0], fwd[1], fwd[2], fi, fw);
        for (int q = 0; q < 6; ++q) nb[q] = FN(tap)(t, i + offs[q][0], j + offs[q][1], k + offs[q][2]);
        for (int f = 0; f < nfields; ++f) {
            const R* d = in[f];
            const R po = d[orig];
            R pf = 0, pb = 0;
            for (int q = 0; q < 8; ++q) {
                pf = FMA(d[bi[q]], bw[q], pf);
                pb = FMA(d[fi[q]], fw[q], pb);
            }
            const R corr = FMA((R)0.5, po - pb, pf);
            R mn = po, mx = po;
            for (int q = 0; q < 6; ++q) {
                mn = FN(fmin_)(mn, d[nb[q]]);
                mx = FN(fmax_)(mx, d[nb[q]]);
            }
            mn = FN(fmin_)(mn, pf);
            mx = FN(fmax_)(mx, pf);
            out[f][s] = FN(fmax_)(mn, FN(fmin_)(corr, mx));
        }
    }
}

void FN(hnso_advect_scalars)(const hnso_topo* t, const R* vel, const R* const* in, R* const* out, int nfields, R dt,
                             R inv_dx) {
    FN(advect_scalars_impl)(t, vel, in, out, nfields, dt, inv_dx, NULL);
}

/* advect_scalar (src/Cuda/Kernel.cu:294-344), the HNanoAdvect kernel: samplers read 0
 * outside the domain; lerp-chain trilinear for the field and the velocity. */
void FN(hnso_advect_scalar)(const hnso_topo* t, const R* vel, const R* in, R* out, R dt, R inv_dx) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R sdt = dt * inv_dx;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        const R po = FN(near_s)(t, in, i, j, k);
        R vc[3], vf[3];
        FN(near_v)(t, vel, i, j, k, vc);
        const R back[3] = {(R)i - vc[0] * sdt, (R)j - vc[1] * sdt, (R)k - vc[2] * sdt};
        const R pf = FN(tri_s)(t, in, back[0], back[1], back[2]);
        FN(tri_v)(t, vel, back[0], back[1], back[2], vf);
        const R fwd[3] = {back[0] + vf[0] * sdt, back[1] + vf[1] * sdt, back[2] + vf[2] * sdt};
        const R pb = FN(tri_s)(t, in, fwd[0], fwd[1], fwd[2]);
        const R corr = pf + (R)0.5 * (po - pb);
        R mn = po, mx = po;
        for (int dim = 0; dim < 3; ++dim) {
            for (int off = -1; off <= 1; off += 2) {
                const R v = FN(near_s)(t, in, i + (dim == 0 ? off : 0), j + (dim == 1 ? off : 0), k + (dim == 2 ? off : 0));
                mn = FN(fmin_)(mn, v);
                mx = FN(fmax_)(mx, v);
            }
        }
        mn = FN(fmin_)(mn, pf);
        mx = FN(fmax_)(mx, pf);
        out[s] = FN(fmax_)(mn, FN(fmin_)(corr, mx));
    }
}

/* divergence (src/Cuda/Kernel.cu:432-453): central difference written through face
 * averages, velocity 0 outside the domain. */
void FN(hnso_divergence)(const hnso_topo* t, const R* vel, R* div, R inv_dx) {
    const int64_t N = hnso_topo_num_voxels(t);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        const R* c = vel + 3 * s;
        R n[3];
        FN(near_v)(t, vel, i + 1, j, k, n);
        const R xp = (c[0] + n[0]) * (R)0.5;
        FN(near_v)(t, vel, i - 1, j, k, n);
        const R xm = (c[0] + n[0]) * (R)0.5;
        FN(near_v)(t, vel, i, j + 1, k, n);
        const R yp = (c[1] + n[1]) * (R)0.5;
        FN(near_v)(t, vel, i, j - 1, k, n);
        const R ym = (c[1] + n[1]) * (R)0.5;
        FN(near_v)(t, vel, i, j, k + 1, n);
        const R zp = (c[2] + n[2]) * (R)0.5;
        FN(near_v)(t, vel, i, j, k - 1, n);
        const R zm = (c[2] + n[2]) * (R)0.5;
        div[s] = (xp - xm + yp - ym + zp - zm) * inv_dx;
    }
}

/* One colour of redBlackGaussSeidelUpdate (src/Cuda/Kernel.cu:459-489): colour
 * (i+j+k)&1, pressure 0 outside the domain with a fixed 1/6 (Dirichlet-0 walls). */
void FN(hnso_rbgs_sweep)(const hnso_topo* t, const R* div, R* p, R dx, int color, R omega) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R dx2 = dx * dx;
    const R inv6 = (R)INV6;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        if (((i + j + k) & 1) != color) continue;
        const R sum = FN(near_s)(t, p, i + 1, j, k) + FN(near_s)(t, p, i - 1, j, k) + FN(near_s)(t, p, i, j + 1, k) +
                      FN(near_s)(t, p, i, j - 1, k) + FN(near_s)(t, p, i, j, k + 1) + FN(near_s)(t, p, i, j, k - 1);
        const R pgs = (sum - div[s] * dx2) * inv6;
        const R pold = p[s];
        p[s] = pold + omega * (pgs - pold);
    }
}

/* The pressure loop of HNS_Advance (src/Cuda/HNanoSolver.cu:366-373): iterations x
 * (colour 0, colour 1). */
void FN(hnso_rbgs)(const hnso_topo* t, const R* div, R* p, R dx, int iterations, R omega) {
    for (int it = 0; it < iterations; ++it) {
        FN(hnso_rbgs_sweep)(t, div, p, dx, 0, omega);
        FN(hnso_rbgs_sweep)(t, div, p, dx, 1, omega);
    }
}

/* Poisson residual of the system the sweeps relax, accumulated in double:
 * r = div*dx^2 - (sum of 6 neighbours - 6 p), with p = 0 outside. Returns sum r^2 and
 * sum (div*dx^2)^2. */
void FN(hnso_residual)(const hnso_topo* t, const R* div, const R* p, R dx, double* r2, double* b2) {
    const int64_t N = hnso_topo_num_voxels(t);
    const double h2 = (double)dx * (double)dx;
    double sr = 0.0, sb = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : sr, sb)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        const double lap = (double)FN(near_s)(t, p, i + 1, j, k) + (double)FN(near_s)(t, p, i - 1, j, k) +
                           (double)FN(near_s)(t, p, i, j + 1, k) + (double)FN(near_s)(t, p, i, j - 1, k) +
                           (double)FN(near_s)(t, p, i, j, k + 1) + (double)FN(near_s)(t, p, i, j, k - 1) -
                           6.0 * (double)p[s];
        const double b = (double)div[s] * h2;
        sr += (b - lap) * (b - lap);
        sb += b * b;
    }
    *r2 = sr;
    *b2 = sb;
}

/* ---- zero-gradient (Neumann) walls: the configurations' boundary, an extension ----------
 * The reference reads p = 0 outside the domain with a fixed 1/6 (Dirichlet-0). With zero-
 * gradient walls the pressure outside equals that of the voxel inside, so a voxel's update
 * averages its n in-domain face neighbours: p += omega ((sum of those - div dx^2) / n - p),
 * the sum in the order x+, x-, y+, y-, z+, z-. The operator is singular, one constant per
 * face-connected component of leaves, so the divergence's mean is removed per component in
 * FP64 first (FN(hnso_remove_mean)). */
static int FN(inside)(const hnso_topo* t, int32_t i, int32_t j, int32_t k) { return hnso_offset(t, i, j, k) != 0; }

void FN(hnso_rbgs_sweep_neumann)(const hnso_topo* t, const R* div, R* p, R dx, int color, R omega) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R dx2 = dx * dx;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        if (((i + j + k) & 1) != color) continue;
        const int32_t d[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        R sum = 0;
        int cnt = 0;
        for (int q = 0; q < 6; ++q) {
            if (!FN(inside)(t, i + d[q][0], j + d[q][1], k + d[q][2])) continue;
            sum = cnt == 0 ? FN(near_s)(t, p, i + d[q][0], j + d[q][1], k + d[q][2])
                           : sum + FN(near_s)(t, p, i + d[q][0], j + d[q][1], k + d[q][2]);
            ++cnt;
        }
        const R pgs = (sum - div[s] * dx2) / (R)cnt;
        const R pold = p[s];
        p[s] = pold + omega * (pgs - pold);
    }
}

void FN(hnso_rbgs_neumann)(const hnso_topo* t, const R* div, R* p, R dx, int iterations, R omega) {
    for (int it = 0; it < iterations; ++it) {
        FN(hnso_rbgs_sweep_neumann)(t, div, p, dx, 0, omega);
        FN(hnso_rbgs_sweep_neumann)(t, div, p, dx, 1, omega);
    }
}

/* r = div dx^2 - (sum of the in-domain neighbours - n p), accumulated in double. */
void FN(hnso_residual_neumann)(const hnso_topo* t, const R* div, const R* p, R dx, double* r2, double* b2) {
    const int64_t N = hnso_topo_num_voxels(t);
    const double h2 = (double)dx * (double)dx;
    double sr = 0.0, sb = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : sr, sb)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        const int32_t d[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        double lap = 0.0;
        int cnt = 0;
        for (int q = 0; q < 6; ++q)
            if (FN(inside)(t, i + d[q][0], j + d[q][1], k + d[q][2])) {
                lap += (double)FN(near_s)(t, p, i + d[q][0], j + d[q][1], k + d[q][2]);
                ++cnt;
            }
        lap -= (double)cnt * (double)p[s];
        const double b = (double)div[s] * h2;
        sr += (b - lap) * (b - lap);
        sb += b * b;
    }
    *r2 = sr;
    *b2 = sb;
}

/* Face-connected components of the leaves (two leaves sharing a face share voxel faces):
 * comp[leaf] in [0, ncomp), labelled in leaf order of first appearance. Returns ncomp. */
static int64_t FN(components)(const hnso_topo* t, int64_t* comp) {
    const int64_t L = t->num_leaves;
    for (int64_t l = 0; l < L; ++l) comp[l] = -1;
    int64_t* stack = (int64_t*)malloc(sizeof(int64_t) * (size_t)(L > 0 ? L : 1));
    int64_t nc = 0;
    for (int64_t l0 = 0; l0 < L; ++l0) {
        if (comp[l0] >= 0) continue;
        int64_t top = 0;
        stack[top++] = l0;
        comp[l0] = nc;
        while (top > 0) {
            const int64_t l = stack[--top];
            const int32_t* o = t->origins + 3 * l;
            const int32_t d[6][3] = {{8, 0, 0}, {-8, 0, 0}, {0, 8, 0}, {0, -8, 0}, {0, 0, 8}, {0, 0, -8}};
            for (int q = 0; q < 6; ++q) {
                const int64_t m = find_leaf(t, o[0] + d[q][0], o[1] + d[q][1], o[2] + d[q][2]);
                if (m >= 0 && comp[m] < 0) {
                    comp[m] = nc;
                    stack[top++] = m;
                }
            }
        }
        ++nc;
    }
    free(stack);
    return nc;
}

/* Removes the mean of div per component: sums in double, the mean subtracted in R. */
void FN(hnso_remove_mean)(const hnso_topo* t, R* div) {
    const int64_t L = t->num_leaves;
    int64_t* comp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(L > 0 ? L : 1));
    const int64_t nc = FN(components)(t, comp);
    double* sum = (double*)calloc((size_t)(nc > 0 ? nc : 1), sizeof(double));
    double* cnt = (double*)calloc((size_t)(nc > 0 ? nc : 1), sizeof(double));
    for (int64_t s = 0; s < 512 * L; ++s) {
        sum[comp[s >> 9]] += (double)div[s];
        cnt[comp[s >> 9]] += 1.0;
    }
    for (int64_t s = 0; s < 512 * L; ++s) div[s] = div[s] - (R)(sum[comp[s >> 9]] / cnt[comp[s >> 9]]);
    free(sum);
    free(cnt);
    free(comp);
}

/* u = u* - grad p with the wall's ghost pressure equal to the voxel's own. */
void FN(hnso_subtract_gradient_neumann)(const hnso_topo* t, const R* vel, const R* p, R* out, R inv_dx) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R h = (R)0.5 * inv_dx;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        const R c = p[s];
#define HNSO_NP(a, b, cc) (FN(inside)(t, a, b, cc) ? FN(near_s)(t, p, a, b, cc) : c)
        const R gx = (HNSO_NP(i + 1, j, k) - HNSO_NP(i - 1, j, k)) * h;
        const R gy = (HNSO_NP(i, j + 1, k) - HNSO_NP(i, j - 1, k)) * h;
        const R gz = (HNSO_NP(i, j, k + 1) - HNSO_NP(i, j, k - 1)) * h;
#undef HNSO_NP
        out[3 * s] = vel[3 * s] - gx;
        out[3 * s + 1] = vel[3 * s + 1] - gy;
        out[3 * s + 2] = vel[3 * s + 2] - gz;
    }
}

/* The projection with zero-gradient walls: divergence, its mean removed per component,
 * p = 0, iterations x (red, black), gradient subtraction. omega < 0: 2/(1+sin(3.14159 dx)). */
void FN(hnso_project_neumann)(const hnso_topo* t, R* vel, R* div, R* p, R dx, int iterations, R omega) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R inv_dx = (R)1 / dx;
    if (omega < (R)0) omega = (R)(2.0f / (1.0f + sin(3.14159 * (double)dx)));
    FN(hnso_divergence)(t, vel, div, inv_dx);
    FN(hnso_remove_mean)(t, div);
    for (int64_t s = 0; s < N; ++s) p[s] = 0;
    FN(hnso_rbgs_neumann)(t, div, p, dx, iterations, omega);
    R* tmp = (R*)malloc(sizeof(R) * 3 * (size_t)N);
    memcpy(tmp, vel, sizeof(R) * 3 * (size_t)N);
    FN(hnso_subtract_gradient_neumann)(t, tmp, p, vel, inv_dx);
    free(tmp);
}

/* subtractPressureGradient (src/Cuda/Kernel.cu:495-541), no collision: u = u* - grad p,
 * central differences, p = 0 outside. */
static void FN(subtract_gradient_impl)(const hnso_topo* t, const R* vel, const R* p, R* out, R inv_dx, const R* sdf) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R h = (R)0.5 * inv_dx;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        const R gx = (FN(near_s)(t, p, i + 1, j, k) - FN(near_s)(t, p, i - 1, j, k)) * h;
        const R gy = (FN(near_s)(t, p, i, j + 1, k) - FN(near_s)(t, p, i, j - 1, k)) * h;
        const R gz = (FN(near_s)(t, p, i, j, k + 1) - FN(near_s)(t, p, i, j, k - 1)) * h;
        R u[3] = {vel[3 * s] - gx, vel[3 * s + 1] - gy, vel[3 * s + 2] - gz};
        /* With a collision SDF: the collision treatment, margin 0.1, blend 1 - sdf / 0.1 (Kernel.cu:528-538). */
        if (sdf) FN(collide)(t, sdf, s, i, j, k, inv_dx, (R)0.1f, u);
        out[3 * s] = u[0];
        out[3 * s + 1] = u[1];
        out[3 * s + 2] = u[2];
    }
}

void FN(hnso_subtract_gradient)(const hnso_topo* t, const R* vel, const R* p, R* out, R inv_dx) {
    FN(subtract_gradient_impl)(t, vel, p, out, inv_dx, NULL);
}

/* computeVorticityMag (src/Cuda/Utils.cuh:226-243): |curl u| at a voxel. */
static R FN(vort_mag)(const hnso_topo* t, const R* vel, int32_t i, int32_t j, int32_t k, R factor) {
    R px[3], mx[3], py[3], my[3], pz[3], mz[3];
    FN(near_v)(t, vel, i + 1, j, k, px);
    FN(near_v)(t, vel, i - 1, j, k, mx);
    FN(near_v)(t, vel, i, j + 1, k, py);
    FN(near_v)(t, vel, i, j - 1, k, my);
    FN(near_v)(t, vel, i, j, k + 1, pz);
    FN(near_v)(t, vel, i, j, k - 1, mz);
    const R ox = ((py[2] - my[2]) - (pz[1] - mz[1])) * factor;
    const R oy = ((pz[0] - mz[0]) - (px[2] - mx[2])) * factor;
    const R oz = ((px[1] - mx[1]) - (py[0] - my[0])) * factor;
    return SQRT(ox * ox + oy * oy + oz * oz);
}

/* vorticityConfinement (src/Cuda/Kernel.cu:682-727), out of place. The |omega| gradient is
 * taken at offsets of int(factor_scale) voxels: the reference builds a Coord from the float
 * (Kernel.cu:707-712), which truncates toward zero, so 0.5 gives a zero force. */
void FN(hnso_vorticity_confinement)(const hnso_topo* t, const R* vel, R* out, R dt, R inv_dx, R scale, R factor_scale) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R factor = (R)0.5 * inv_dx;
    const int32_t fs = (int32_t)factor_scale;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < N; ++s) {
        int32_t i, j, k;
        FN(coord_of)(t, s, &i, &j, &k);
        R px[3], mx[3], py[3], my[3], pz[3], mz[3];
        FN(near_v)(t, vel, i + 1, j, k, px);
        FN(near_v)(t, vel, i - 1, j, k, mx);
        FN(near_v)(t, vel, i, j + 1, k, py);
        FN(near_v)(t, vel, i, j - 1, k, my);
        FN(near_v)(t, vel, i, j, k + 1, pz);
        FN(near_v)(t, vel, i, j, k - 1, mz);
        const R ox = ((py[2] - my[2]) - (pz[1] - mz[1])) * factor;
        const R oy = ((pz[0] - mz[0]) - (px[2] - mx[2])) * factor;
        const R oz = ((px[1] - mx[1]) - (py[0] - my[0])) * factor;
        const R mpx = FN(vort_mag)(t, vel, i + fs, j, k, factor), mmx = FN(vort_mag)(t, vel, i - fs, j, k, factor);
        const R mpy = FN(vort_mag)(t, vel, i, j + fs, k, factor), mmy = FN(vort_mag)(t, vel, i, j - fs, k, factor);
        const R mpz = FN(vort_mag)(t, vel, i, j, k + fs, factor), mmz = FN(vort_mag)(t, vel, i, j, k - fs, factor);
        const R gx = (mpx - mmx) * (R)0.5 * inv_dx;
        const R gy = (mpy - mmy) * (R)0.5 * inv_dx;
        const R gz = (mpz - mmz) * (R)0.5 * inv_dx;
        const R glen = SQRT(gx * gx + gy * gy + gz * gz) + (R)1e-5f;
        const R nx = gx / glen, ny = gy / glen, nz = gz / glen;
        const R fx = scale * (ny * oz - nz * oy), fy = scale * (nz * ox - nx * oz), fz = scale * (nx * oy - ny * ox);
        out[3 * s] = vel[3 * s] + fx * dt;
        out[3 * s + 1] = vel[3 * s + 1] + fy * dt;
        out[3 * s + 2] = vel[3 * s + 2] + fz * dt;
    }
}

/* temperature_buoyancy (src/Cuda/Kernel.cu:546-563): v.y += max(0,(T-Tamb)*beta)*dt where
 * T > Tamb; otherwise the velocity passes through. */
void FN(hnso_temperature_buoyancy)(int64_t n, const R* vel, const R* temp, R* out, R dt, R ambient, R strength) {
    for (int64_t s = 0; s < n; ++s) {
        const R T = temp[s];
        out[3 * s] = vel[3 * s];
        out[3 * s + 2] = vel[3 * s + 2];
        if (T <= ambient) {
            out[3 * s + 1] = vel[3 * s + 1];
        } else {
            const R f = FN(fmax_)((R)0, (T - ambient) * strength);
            out[3 * s] = vel[3 * s] + (R)0 * dt;
            out[3 * s + 1] = vel[3 * s + 1] + f * dt;
            out[3 * s + 2] = vel[3 * s + 2] + (R)0 * dt;
        }
    }
}

/* temperature_buoyancy with a density term, the extension the configurations' buoyancy needs
 * (the reference has no density term): v.y += (b_T - alpha * density) dt, with b_T the
 * reference's max(0, (T - Tamb) beta) where T > Tamb and 0 elsewhere. alpha = 0 is exactly
 * hnso_temperature_buoyancy. density may be NULL (taken as 0). */
void FN(hnso_buoyancy_density)(int64_t n, const R* vel, const R* temp, const R* density, R* out, R dt, R ambient,
                               R strength, R alpha) {
    if (alpha == (R)0) {
        FN(hnso_temperature_buoyancy)(n, vel, temp, out, dt, ambient, strength);
        return;
    }
    for (int64_t s = 0; s < n; ++s) {
        const R T = temp[s];
        const R bt = T > ambient ? FN(fmax_)((R)0, (T - ambient) * strength) : (R)0;
        const R f = bt - alpha * (density ? density[s] : (R)0);
        out[3 * s] = vel[3 * s];
        out[3 * s + 1] = vel[3 * s + 1] + f * dt;
        out[3 * s + 2] = vel[3 * s + 2];
    }
}

/* combustion (src/Cuda/Kernel.cu:568-588): burn min(fuel, rate*dt) where fuel > 0 and
 * T >= ignition; heat release raises T. */
void FN(hnso_combustion)(int64_t n, const R* fuel, const R* temp, R* out_fuel, R* out_temp, R dt, R ignition, R rate,
                         R heat) {
    for (int64_t s = 0; s < n; ++s) {
        R f = fuel[s], T = temp[s];
        if (f > (R)0 && T >= ignition) {
            const R burned = FN(fmin_)(f, rate * dt);
            f -= burned;
            T += burned * heat;
        }
        out_fuel[s] = f;
        out_temp[s] = T;
    }
}

/* combustion_oxygen (src/Cuda/Kernel.cu:641-677): oxygen = 1 - fuel - waste, burn =
 * min(oxygen, fuel); waste += 2 burn; flame = max(flame, min(1, 10 burn)); T += burn*gain;
 * div += burn*expansion. Fuel below 1e-3 counts as 0. */
void FN(hnso_combustion_oxygen)(int64_t n, const R* fuel, const R* waste, const R* temp, R* div, const R* flame,
                                R* o_fuel, R* o_waste, R* o_temp, R* o_flame, R gain, R expansion) {
    for (int64_t s = 0; s < n; ++s) {
        R f = fuel[s];
        const R w = waste[s], T = temp[s], fl = flame[s];
        if (f < (R)0.001f) f = 0;
        const R ox = (R)1 - f - w;
        if (ox < (R)0) {
            o_fuel[s] = f;
            o_waste[s] = w;
            o_temp[s] = T;
            o_flame[s] = fl;
            continue;
        }
        const R burn = FN(fmin_)(ox, f);
        o_fuel[s] = f - burn;
        o_waste[s] = w + burn * (R)2;
        o_temp[s] = T + burn * gain;
        div[s] += burn * expansion;
        o_flame[s] = FN(fmax_)(fl, FN(fmin_)((R)1, burn * (R)10));
    }
}

/* add_scalar_source / add_velocity_source(_xyz) / add_gravity
 * (src/Cuda/Kernel.cu:732-755, 834-838). */
void FN(hnso_add_scalar_source)(int64_t n, R* field, const R* src, R dt) {
    for (int64_t s = 0; s < n; ++s) field[s] += dt * src[s];
}

void FN(hnso_add_velocity_source)(int64_t n, R* vel, const R* src, R dt) {
    for (int64_t s = 0; s < 3 * n; ++s) vel[s] += src[s] * dt;
}

void FN(hnso_add_velocity_source_xyz)(int64_t n, R* vel, const R* sx, const R* sy, const R* sz, R dt) {
    for (int64_t s = 0; s < n; ++s) {
        vel[3 * s] += dt * sx[s];
        vel[3 * s + 1] += dt * sy[s];
        vel[3 * s + 2] += dt * sz[s];
    }
}

void FN(hnso_add_gravity)(int64_t n, R* vel, R g, R dt) {
    for (int64_t s = 0; s < n; ++s) vel[3 * s + 1] -= g * dt;
}

/* HNanoProjectNonDivergent (src/Cuda/PressureProjection.cu:9-78): divergence, p = 0,
 * iterations x (red, black), gradient subtraction back into the velocity. omega < 0 selects
 * that path's 2/(1+sin(3.14159*dx)) evaluated in double (PressureProjection.cu:53). */
void FN(hnso_project)(const hnso_topo* t, R* vel, R* div, R* p, R dx, int iterations, R omega) {
    const int64_t N = hnso_topo_num_voxels(t);
    const R inv_dx = (R)1 / dx;
    if (omega < (R)0) omega = (R)(2.0f / (1.0f + sin(3.14159 * (double)dx)));
    FN(hnso_divergence)(t, vel, div, inv_dx);
    for (int64_t s = 0; s < N; ++s) p[s] = 0;
    FN(hnso_rbgs)(t, div, p, dx, iterations, omega);
    R* tmp = (R*)malloc(sizeof(R) * 3 * (size_t)N);
    memcpy(tmp, vel, sizeof(R) * 3 * (size_t)N);
    FN(hnso_subtract_gradient)(t, tmp, p, vel, inv_dx);
    free(tmp);
}

/* ---- HNS_Advance with a force model ----------------------------------------------------
 * The kernel sequence of one HNS_Advance call (src/Cuda/HNanoSolver.cu:223-456): with a
 * collision SDF, enforceCollisionBoundaries on the velocity first (:241-244); per substep
 * advect velocity, confinement (run out of place; the reference's in-place launch at
 * :279-281 races), velocity and scalar sources, gravity, divergence, the combustion model,
 * buoyancy from the burned temperature, iteration x (red, black) from p = 0 with omega =
 * 2/(1+sin(3.14159 dx)), the disturbance re-solve (divergence again, p = 0,
 * max(2, iteration/2) sweeps) when enabled, gradient subtraction into the velocity (with the
 * SDF, then enforceCollisionBoundaries again, :411-414), then advection of the persistent
 * scalars with the projected velocity; the SDF also enters the velocity and scalar advection
 * and the gradient subtraction.
 * The model (NULL: the reference) chooses the combustion: combustion_oxygen (Kernel.cu:641-677,
 * the reference's step; adds expansion to the divergence), combustion (Kernel.cu:568-588,
 * rate/heat; no step of the reference calls it) or none; adds the density term of the
 * buoyancy (hnso_buoyancy_density); and may replace the SOR factor (FP64 solves run to
 * convergence). Fields the combustion model uses (oxygen: fuel, waste, temperature, flame;
 * rate: fuel, temperature; none: temperature) that are absent from F->scalars are created
 * zero-filled in F->created on first use and not advected during this call. */
static R* FN(find_scalar)(const FN(hnso_advance_fields)* f, const char* name) {
    for (int i = 0; i < f->nscalars; ++i)
        if (strcmp(f->names[i], name) == 0) return f->scalars[i];
    return NULL;
}

void FN(hnso_hns_advance_model)(const hnso_topo* t, const FN(hnso_advance_fields)* F, R dx, int iteration, R dt,
                                const hnso_combustion_params* P, const hnso_force_model* M) {
    const hnso_force_model reference_model = {0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (!M) M = &reference_model;
    const int64_t N = F->n;
    const R inv_dx = (R)1 / dx;
    const int SUBS = P->substeps > 1 ? P->substeps : 1;
    const R dt_sub = dt / (R)SUBS;
    static const char* special[4] = {"fuel", "waste", "temperature", "flame"};
    int uses[4] = {1, 1, 1, 1};
    if (M->combustion == 1) uses[1] = uses[3] = 0;
    if (M->combustion == 2) uses[0] = uses[1] = uses[3] = 0;
    int made[4] = {0, 0, 0, 0};
    R* adv = (R*)calloc((size_t)(3 * N), sizeof(R));
    R* adv2 = (R*)calloc((size_t)(3 * N), sizeof(R));
    R* div = (R*)calloc((size_t)N, sizeof(R));
    R* p = (R*)calloc((size_t)N, sizeof(R));
    R* o[4];
    for (int q = 0; q < 4; ++q) o[q] = (R*)calloc((size_t)N, sizeof(R));

    const R* sdf = F->collision_sdf;
    if (sdf) FN(hnso_enforce_collision)(t, F->velocity, sdf, inv_dx);
    for (int s = 0; s < SUBS; ++s) {
        FN(advect_vector_impl)(t, F->velocity, adv, dt_sub, inv_dx, sdf);
        FN(hnso_vorticity_confinement)(t, adv, adv2, dt_sub, inv_dx, P->vorticityScale, P->factorScale);
        R* sw = adv;
        adv = adv2;
        adv2 = sw;
        if (F->src_vel) {
            FN(hnso_add_velocity_source)(N, adv, F->src_vel, dt_sub);
        } else if (F->src_vel_x && F->src_vel_y && F->src_vel_z) {
            FN(hnso_add_velocity_source_xyz)(N, adv, F->src_vel_x, F->src_vel_y, F->src_vel_z, dt_sub);
        }
        const R* srcs[3] = {F->src_temperature, F->src_density, F->src_fuel};
        const char* dsts[3] = {"temperature", "density", "fuel"};
        for (int q = 0; q < 3; ++q) {
            R* dst = FN(find_scalar)(F, dsts[q]);
            if (!dst)
                for (int k = 0; k < 4; ++k)
                    if (made[k] && strcmp(special[k], dsts[q]) == 0) dst = F->created[k];
            if (srcs[q] && dst) FN(hnso_add_scalar_source)(N, dst, srcs[q], dt_sub);
        }
        if (P->gravity != 0.0f) FN(hnso_add_gravity)(N, adv, P->gravity, dt_sub);
        FN(hnso_divergence)(t, adv, div, inv_dx);

        R* fld[4] = {NULL, NULL, NULL, NULL};
        for (int k = 0; k < 4; ++k) {
            if (!uses[k]) continue;
            fld[k] = FN(find_scalar)(F, special[k]);
            if (!fld[k]) {
                fld[k] = F->created[k];
                if (!made[k]) {
                    memset(fld[k], 0, sizeof(R) * (size_t)N);
                    made[k] = 1;
                }
            }
        }
        if (M->combustion == 0) {
            for (int q = 0; q < 4; ++q) memset(o[q], 0, sizeof(R) * (size_t)N);
            FN(hnso_combustion_oxygen)(N, fld[0], fld[1], fld[2], div, fld[3], o[0], o[1], o[2], o[3],
                                       P->temperatureRelease, P->expansionRate);
            for (int k = 0; k < 4; ++k) memcpy(fld[k], o[k], sizeof(R) * (size_t)N);
        } else if (M->combustion == 1) {
            FN(hnso_combustion)(N, fld[0], fld[2], o[0], o[2], dt_sub, (R)M->ignition_temp, (R)M->burn_rate,
                                (R)M->heat_release);
            memcpy(fld[0], o[0], sizeof(R) * (size_t)N);
            memcpy(fld[2], o[2], sizeof(R) * (size_t)N);
        }
        FN(hnso_buoyancy_density)(N, adv, fld[2], FN(find_scalar)(F, "density"), adv, dt_sub, P->ambientTemp,
                                  P->buoyancyStrength, (R)M->density_buoyancy);

        memset(p, 0, sizeof(R) * (size_t)N);
        const R omega = M->omega > 0.0 ? (R)M->omega : OMEGA_OF_DX(dx);
        FN(hnso_rbgs)(t, div, p, dx, iteration, omega);
        if (P->disturbanceEnable > 0.0f) {
            FN(hnso_divergence)(t, adv, div, inv_dx);
            memset(p, 0, sizeof(R) * (size_t)N);
            FN(hnso_rbgs)(t, div, p, dx, iteration / 2 > 2 ? iteration / 2 : 2, omega);
        }
        FN(subtract_gradient_impl)(t, adv, p, F->velocity, inv_dx, sdf);
        if (sdf) FN(hnso_enforce_collision)(t, F->velocity, sdf, inv_dx);

        if (F->nscalars > 0) {
            R** outs = (R**)malloc(sizeof(R*) * (size_t)F->nscalars);
            for (int k = 0; k < F->nscalars; ++k) outs[k] = (R*)calloc((size_t)N, sizeof(R));
            FN(advect_scalars_impl)(t, F->velocity, (const R* const*)F->scalars, outs, F->nscalars, dt_sub, inv_dx, sdf);
            for (int k = 0; k < F->nscalars; ++k) {
                memcpy(F->scalars[k], outs[k], sizeof(R) * (size_t)N);
                free(outs[k]);
            }
            free(outs);
        }
    }
    free(adv);
    free(adv2);
    free(div);
    free(p);
    for (int q = 0; q < 4; ++q) free(o[q]);
}

#undef FN
#undef CAT
#undef CAT2
