/* hns.h -- C ABI of the B200 sparse smoke/fire solver (libhns.so).
 *
 * Plain C: opaque context, status codes, raw pointers and sizes. No exception crosses this
 * boundary and no C++ or torch type appears in it. The C++ surface that mirrors the
 * reference's own entry points (HNS_EnsureContext, AdvectIndexGrid, ...) is declared in
 * hns_legacy.hpp and is implemented on top of these functions.
 *
 * Data layout (the reference's "indexed" layout, src/Utils/GridBuilder.hpp:164-174,
 * 231-251): the domain is a set of 8^3 leaves; leaf i owns slots [512 i, 512 i + 512) and
 * slot 512 i + n holds the voxel at origin_i + ((n>>6)&7, (n>>3)&7, n&7). A voxel's
 * NanoVDB ValueOnIndex offset is 1 + slot, and 0 outside the domain
 * (externals/nanovdb/NanoVDB.h:4219-4227, 4598-4601). Scalar fields are float[N]; vec3
 * fields are float[3N] interleaved x,y,z per slot (the reference's nanovdb::Vec3f arrays).
 *
 * Unless a function says otherwise, field pointers are DEVICE pointers on the context's
 * device and work is enqueued on the context's stream; every entry point returns after
 * its work is enqueued (call hns_synchronize to wait). All functions are thread-safe for
 * distinct contexts; one context must not be used from two threads at once.
 */
#ifndef HNS_H
#define HNS_H

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define HNS_API __declspec(dllexport)
#else
#define HNS_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define HNS_ABI_VERSION 1

typedef enum hns_status {
    HNS_OK = 0,
    HNS_ERR_INVALID_ARG = 1,   /* null pointer, bad size, bad enum value */
    HNS_ERR_CUDA = 2,          /* a CUDA runtime call failed; see hns_last_error() */
    HNS_ERR_OUT_OF_MEMORY = 3, /* device allocation failed */
    HNS_ERR_NOT_FOUND = 4,     /* named field does not exist */
    HNS_ERR_LAYOUT = 5,        /* coordinates are not leaf-dense / leaves not 8-aligned or repeated */
    HNS_ERR_NOT_CONVERGED = 6, /* iterative solve hit its iteration cap above the tolerance */
    HNS_ERR_UNSUPPORTED = 7,   /* valid request this build does not support (see message) */
    HNS_ERR_TIMEOUT = 8        /* a bounded device-side wait gave up */
} hns_status;

typedef struct hns_ctx hns_ctx;

HNS_API int hns_abi_version(void);
HNS_API const char* hns_status_string(hns_status status);
/* Message of the last failing call on this thread ("" if none). */
HNS_API const char* hns_last_error(void);

/* ---- topology --------------------------------------------------------------------------
 * Replaces CreateIndexGrid (src/Cuda/HNanoSolver.cu:498-510, which builds a NanoVDB
 * ValueOnIndex grid with voxelsToGrid) and the per-context setup of HNS_EnsureContext
 * (src/Cuda/HNanoSolver.cu:58-156). The caller's slot order is authoritative: leaf i of
 * `leaf_origins` owns slots [512 i, 512 i + 512). When the leaves are in NanoVDB order
 * (hns_sort_leaves_nanovdb) every voxel's offset equals the reference grid's. */

/* leaf_origins: host int32[3 * num_leaves], each a multiple of 8, no repeats.
 * device: CUDA device ordinal. The context creates its own non-blocking stream. */
HNS_API hns_status hns_create(hns_ctx** out, const int32_t* leaf_origins, int64_t num_leaves, float voxel_size,
                              int device);
/* coords: host int32[3 * num_voxels] in the leaf-dense layout above (num_voxels a multiple
 * of 512); HNS_ERR_LAYOUT otherwise. This is the coordinate block of GridIndexedData. */
HNS_API hns_status hns_create_from_coords(hns_ctx** out, const int32_t* coords, int64_t num_voxels,
                                          float voxel_size, int device);
/* The domain set-up of the HNanoSolver SOP (src/SOP/HNanoSolver/SOP_HNanoSolver.cpp:280-285: the
 * velocity grid's active voxels dilated by `padding` voxels, face, edge and vertex neighbours)
 * with the grid built from the voxel list (CreateIndexGrid, src/Cuda/HNanoSolver.cu:498-510),
 * on the device: the context's leaves are every leaf that a dilated voxel touches, in NanoVDB
 * order. ijk: int32[3 * num_voxels], on the host, or on this context's device when
 * ijk_on_device is nonzero; repeats allowed; |coordinate| < 2^23 - 64; padding in [0, 8].
 * hns_leaf_origins returns the leaves. */
HNS_API hns_status hns_create_from_voxels(hns_ctx** out, const int32_t* ijk, int64_t num_voxels, int padding,
                                          int ijk_on_device, float voxel_size, int device);
HNS_API hns_status hns_destroy(hns_ctx* ctx);
/* Use a caller-owned cudaStream_t (NULL restores the context's own stream). */
HNS_API hns_status hns_set_stream(hns_ctx* ctx, void* cuda_stream);
HNS_API void* hns_get_stream(const hns_ctx* ctx);
HNS_API hns_status hns_synchronize(hns_ctx* ctx);
HNS_API int64_t hns_num_voxels(const hns_ctx* ctx);
HNS_API int64_t hns_num_leaves(const hns_ctx* ctx);
HNS_API float hns_voxel_size(const hns_ctx* ctx);
/* Host int32[3 * num_leaves]. */
HNS_API hns_status hns_leaf_origins(const hns_ctx* ctx, int32_t* out);
/* ValueOnIndex offsets (0 outside the domain, else 1 + slot) of host ijk[3n], computed on
 * the device; out is host uint64[n]. Synchronous. */
HNS_API hns_status hns_index_offsets(hns_ctx* ctx, const int32_t* ijk, int64_t n, uint64_t* out);
/* Sorts host leaf origins in place into NanoVDB leaf order. */
HNS_API hns_status hns_sort_leaves_nanovdb(int32_t* leaf_origins, int64_t num_leaves);
/* *out = 1 if the context's leaves are in NanoVDB order, else 0. */
HNS_API hns_status hns_is_nanovdb_order(const hns_ctx* ctx, int* out);

/* ---- operators on device arrays ---------------------------------------------------------
 * One call = one pass of the corresponding reference kernel over every slot, with the
 * context's voxel size. Inputs and outputs must not alias unless stated. */

/* MacCormack vec3 advection (advect_vector, src/Cuda/Kernel.cu:349-426): vel -> out. */
HNS_API hns_status hns_advect_vec3(hns_ctx* ctx, const float* vel, float* out, float dt);
/* Single-field MacCormack advection (advect_scalar, src/Cuda/Kernel.cu:294-344; the kernel
 * behind HNanoAdvect): samplers read 0 outside the domain. */
HNS_API hns_status hns_advect_scalar(hns_ctx* ctx, const float* vel, const float* in, float* out, float dt);
/* Multi-field advection of HNS_Advance (advect_scalars, src/Cuda/Kernel.cu:163-289): the
 * back-trace uses the voxel's own velocity and out-of-domain taps read slot 0.
 * in/out: HOST arrays of nfields device pointers. */
HNS_API hns_status hns_advect_scalars(hns_ctx* ctx, const float* vel, const float* const* in, float* const* out,
                                      int nfields, float dt);
/* Central divergence (divergence, src/Cuda/Kernel.cu:432-453). */
HNS_API hns_status hns_divergence(hns_ctx* ctx, const float* vel, float* div);

/* Flags of the pressure solve. */
#define HNS_SOLVE_ZERO_INIT 1u   /* start from p = 0 (p is not read; the reference's memset) */
#define HNS_SOLVE_NEUMANN 2u     /* zero-gradient walls instead of the reference's p = 0 outside: a
                                    voxel averages its in-domain face neighbours, (sum - div dx^2) / n,
                                    and the gradient takes a missing neighbour's pressure as the
                                    voxel's own. hns_project and hns_step_plain first remove the
                                    divergence's mean per face-connected component of leaves (FP64
                                    sums), which the singular system needs; hns_rbgs relaxes the div
                                    it is given. Plain red-black solves only (not with
                                    HNS_SOLVE_REFINE, the mixed step or hns_project_static). */

/* `iterations` red-black SOR iterations on div (redBlackGaussSeidelUpdate,
 * src/Cuda/Kernel.cu:459-489, looped as src/Cuda/HNanoSolver.cu:366-373): colour
 * (i+j+k)&1, p = 0 outside, fixed 1/6. p: device float[N], in/out. */
HNS_API hns_status hns_rbgs(hns_ctx* ctx, const float* div, float* p, int iterations, float omega, unsigned flags);
/* u = u* - grad p (subtractPressureGradient, src/Cuda/Kernel.cu:495-541). */
HNS_API hns_status hns_subtract_gradient(hns_ctx* ctx, const float* vel, const float* p, float* out);
/* Vorticity confinement (vorticityConfinement, src/Cuda/Kernel.cu:682-727), out of place.
 * The |omega| gradient is taken int(factor_scale) voxels away, as the reference's Coord
 * construction truncates the float. */
HNS_API hns_status hns_vorticity_confinement(hns_ctx* ctx, const float* vel, float* out, float dt, float scale,
                                             float factor_scale);

/* Result of a pressure solve. */
typedef struct hns_solve_info {
    int iterations;           /* red-black iterations run */
    double residual;          /* ||b - A p||_2 / ||b||_2 in FP64 after the solve (b = div dx^2) */
    double initial_residual;  /* same for the initial p */
} hns_solve_info;

/* HNanoProjectNonDivergent (src/Cuda/PressureProjection.cu:9-78): divergence of vel,
 * p = 0, `iterations` red-black iterations, vel -= grad p in place. omega <= 0 selects the
 * reference's 2/(1+sin(3.14159 dx)). `info` may be NULL; when given, the FP64 residuals
 * are computed (two extra reduction passes) and the call synchronizes. */
HNS_API hns_status hns_project(hns_ctx* ctx, float* vel, int iterations, float omega, unsigned flags,
                               hns_solve_info* info);

/* hns_project without any device allocation: same arguments and results, but the divergence,
 * pressure and ping-pong scratch live in one fixed 12 MiB device array inside the library
 * rather than in buffers the context allocates on first use. No counterpart in the reference.
 * For callers that must not allocate while they run a solve: cudaMalloc synchronizes the
 * device and fails once another allocator (a host application's memory pool, a caching
 * allocator) holds the free memory.
 * - At most 1,048,576 active voxels (2048 leaves); larger grids return HNS_ERR_UNSUPPORTED.
 * - The first call on each device looks the array's address up (cudaGetSymbolAddress, which
 *   also loads its module); make that first call before any stream capture begins. Calls made
 *   outside capture look it up again; calls made during capture use the address found by the
 *   last call outside it, so the device must not be reset between that call and the capture.
 * - vel must be 4-byte aligned (HNS_ERR_INVALID_ARG otherwise).
 * - The array is shared by every context on a device: calls that overlap in time on one
 *   device (different streams or threads) race on it. Serialise them.
 * - The pressure scratch is cleared to zero on every call. */
HNS_API hns_status hns_project_static(hns_ctx* ctx, float* vel, int iterations, float omega, unsigned flags,
                                      hns_solve_info* info);

/* ---- one solver step ------------------------------------------------------------------- */

#define HNS_SOLVE_REFINE 4u /* hns_step_plain: FP64 iterative refinement around FP32 red-black
                               inner solves (max_outer x inner_iterations) instead of one plain
                               FP32 solve; removes the FP32 rounding floor of the residual */
#define HNS_SOLVE_MULTIGRID 8u /* with refinement (HNS_SOLVE_REFINE in hns_step_desc.flags; always in
                                    hns_mixed_desc.flags): each outer step's inner solve is geometric
                                    multigrid (levels of 8, 4, 2 and 1 cells per leaf side) instead of
                                    inner_iterations red-black iterations. The FP16 colour-split inner
                                    solve (hns_mixed_desc, the default layout) runs inner_iterations
                                    V-cycles per outer step with the colour-split red-black half-sweep
                                    as the fine smoother and FP32 coarse levels whose operator is
                                    corrected at the walls; the FP32 and other FP16 inner solves run
                                    one FP32 V-cycle. The reference declares this preconditioner
                                    (src/Cuda/Kernels.cuh:52-60) but does not implement it. */

typedef struct hns_step_desc {
    float dt;
    int max_iterations; /* red-black iteration cap (rounded up to even when tolerance > 0) */
    float omega;        /* SOR factor; <= 0 selects 2/(1+sin(3.14159 dx)) */
    double tolerance;   /* target ||b - A p|| / ||b|| (FP64); 0 runs exactly max_iterations */
    int check_every;    /* iterations between residual checks (rounded up to even; 0 = 10) */
    unsigned flags;     /* HNS_SOLVE_* (HNS_SOLVE_ZERO_INIT is implied) */
    int max_outer;      /* HNS_SOLVE_REFINE: outer refinement cap */
    int inner_iterations; /* HNS_SOLVE_REFINE: red-black iterations per outer refinement */
} hns_step_desc;

/* One step of the SOP operator chain HNanoAdvect + HNanoAdvectVelocity +
 * HNanoProjectNonDivergent (src/SOP/Advection/SOP_VDBAdvect.hpp:66,
 * src/SOP/VelocityAdvection/SOP_VDBAdvectVelocity.hpp:60,
 * src/SOP/ProjectNonDivergent/SOP_VDBProjectNonDivergent.hpp:69): vel_in and every
 * scalars_in[i] are advected along the same MacCormack trace into vel_out / scalars_out[i]
 * (advect_vector and advect_scalar semantics), then vel_out is projected in place. The
 * solve starts from p = 0 and, with a tolerance, stops on the device once the residual
 * test passes. Device pointers; scalars_in/out are host arrays of device pointers.
 * info may be NULL (no synchronization); with info the call synchronizes, reports the
 * exact FP64 residual and returns HNS_ERR_NOT_CONVERGED if the tolerance was not met. */
HNS_API hns_status hns_step_plain(hns_ctx* ctx, const float* vel_in, float* vel_out, const float* const* scalars_in,
                                  float* const* scalars_out, int nscalars, const hns_step_desc* desc,
                                  hns_solve_info* info);
/* hns_step_plain on HOST buffers updated in place (uploads, step, downloads; synchronous):
 * the host-memory form of the SOP-facing operators. */
HNS_API hns_status hns_step_plain_host(hns_ctx* ctx, float* vel, float* const* scalars, int nscalars,
                                       const hns_step_desc* desc, hns_solve_info* info);
/* Iterations and last checked residual of the most recent convergence-checked solve
 * (synchronizes). residual is -1 when that solve ran without a tolerance. */
HNS_API hns_status hns_last_solve(hns_ctx* ctx, hns_solve_info* info);
/* Convergence log. Every convergence-checked solve (a tolerance > 0) and every refined solve
 * appends one entry on the device, in stream order and without a host wait: the iterations
 * its result took (red-black iterations; outer x inner for a refined solve; the cap when the
 * tolerance was not reached) and the relative FP64 residual of its last check. The context
 * keeps the last 4096 entries. hns_solve_log (synchronizes) sets *count to the entries
 * appended since the last reset, copies the most recent min(*count, 4096, capacity) of them
 * to out (oldest first; initial_residual 1) and, when reset is nonzero, starts a new count.
 * No counterpart in the reference, whose solves have no tolerance. */
HNS_API hns_status hns_solve_log(hns_ctx* ctx, hns_solve_info* out, int capacity, int* count, int reset);

/* ---- mixed precision -------------------------------------------------------------------
 * Fields stored as BF16 velocity (3 x bf16 interleaved per slot) and FP16 scalars, FP32
 * arithmetic, and the pressure solve wrapped in iterative refinement: FP64 outer residual
 * r = b - L p and FP64 accumulated pressure, each outer step solving L e = r / rms(r) with
 * inner_iterations red-black SOR iterations on FP16 storage from e = 0. */
#define HNS_DTYPE_F32 0
#define HNS_DTYPE_F16 1
#define HNS_DTYPE_BF16 2
#define HNS_DTYPE_F64 3

/* Elementwise conversion of `count` device values (round to nearest). Supported pairs:
 * F32<->BF16, F32<->F16, F32<->F64, and same-type copies. */
HNS_API hns_status hns_convert(hns_ctx* ctx, const void* src, int src_dtype, void* dst, int dst_dtype, int64_t count);

typedef struct hns_mixed_desc {
    float dt;
    float omega;          /* inner SOR factor; <= 0 selects 1.9 */
    double tolerance;     /* target ||b - L p|| / ||b|| in FP64 (> 0) */
    int max_outer;        /* outer refinement cap */
    int inner_iterations; /* red-black iterations per outer refinement (V-cycles with HNS_SOLVE_MULTIGRID) */
    unsigned flags;       /* 0, or HNS_SOLVE_MULTIGRID */
} hns_mixed_desc;

/* hns_step_plain on reduced-precision storage: vel_in/vel_out BF16 (3 per slot), scalars
 * FP16; same operator chain, refined solve. Device pointers; scalars_in/out are host arrays
 * of device pointers. With info the call synchronizes and reports inner iterations run
 * (outer x inner_iterations) and the exact FP64 residual of the returned pressure. */
HNS_API hns_status hns_step_mixed(hns_ctx* ctx, const void* vel_in, void* vel_out, const void* const* scalars_in,
                                  void* const* scalars_out, int nscalars, const hns_mixed_desc* desc,
                                  hns_solve_info* info);
/* hns_step_mixed from FP32 HOST buffers updated in place: uploads, converts to BF16/FP16 on
 * the device, steps, converts back and downloads (synchronous). */
HNS_API hns_status hns_step_mixed_host(hns_ctx* ctx, float* vel, float* const* scalars, int nscalars,
                                       const hns_mixed_desc* desc, hns_solve_info* info);
/* Result of the most recent refined solve (synchronizes). */
HNS_API hns_status hns_last_refine(hns_ctx* ctx, hns_solve_info* info);
/* The FP64 pressure of the most recent refined solve, copied to device p_out[num_voxels]. */
HNS_API hns_status hns_refine_pressure(hns_ctx* ctx, double* p_out, int* outer_iterations, double* residual);

/* ---- named fields and the all-in-one step -----------------------------------------------
 * The context keeps named device fields, as the reference's SimContext keeps d_state and
 * d_src (src/Cuda/HNanoSolver.cu:27-48): "velocity" (3 components), persistent scalars,
 * sources named "src_*" (src_vel or src_vel_x/y/z, src_temperature, src_density,
 * src_fuel). Fields live across calls; the simulation state stays on the device. */

/* Creates or overwrites a field from `data` (host, or device if on_device); data NULL
 * creates a zero field. components: 1 or 3. Host uploads complete before return. */
HNS_API hns_status hns_field_set(hns_ctx* ctx, const char* name, int components, const float* data, int on_device);
/* Copies a field to `out` (host, or device if on_device); host copies complete before return. */
HNS_API hns_status hns_field_get(hns_ctx* ctx, const char* name, float* out, int on_device);
/* Device pointer of a field (valid until the field is removed or the next hns_advance). */
HNS_API hns_status hns_field_ptr(hns_ctx* ctx, const char* name, float** dev_ptr, int* components);
HNS_API hns_status hns_field_remove(hns_ctx* ctx, const char* name);
HNS_API int hns_field_count(const hns_ctx* ctx);
/* Name (truncated to name_len-1 chars) and component count of field `index`. */
HNS_API hns_status hns_field_info(const hns_ctx* ctx, int index, char* name, size_t name_len, int* components);

/* Parameters of the all-in-one step; same layout as the reference's CombustionParams
 * (src/Cuda/Kernels.cuh:5-24). */
typedef struct hns_combustion_params {
    float expansionRate;
    float temperatureRelease;
    float buoyancyStrength;
    float ambientTemp;
    float vorticityScale;
    float factorScale;
    float disturbanceEnable;
    float disturbanceStrength;
    float disturbanceSwirl;
    float disturbanceThreshold;
    float disturbanceGain;
    float disturbanceFrequency;
    int substeps;
    float gravity;
    float maskDensityMin;
    float maskDensityMax;
    int downloadVel;
    int simReset;
} hns_combustion_params;

/* HNS_Advance (src/Cuda/HNanoSolver.cu:223-456) on the context's fields, without collision:
 * per substep advect the velocity, vorticity confinement (out of place), velocity and scalar
 * sources, gravity, divergence, oxygen combustion, buoyancy, `iterations` red-black
 * iterations from p = 0 with omega = 2/(1+sin(3.14159 dx)), the re-solve of the reference's
 * disturbance branch when disturbanceEnable > 0, gradient subtraction, and advection of the
 * scalars present at the call's start with the projected velocity. fuel, waste, temperature
 * and flame are created zero-filled when missing. */
HNS_API hns_status hns_advance(hns_ctx* ctx, int iterations, float dt, const hns_combustion_params* params);
/* Force models of the all-in-one step. The reference's HNS_Advance burns with
 * combustion_oxygen and has a temperature-only buoyancy; its `combustion` kernel (rate and heat,
 * src/Cuda/Kernel.cu:568-588) is called by no step. hns_force_model selects the burn and adds a
 * density term to the buoyancy; its zero value is the reference's step. */
#define HNS_COMBUSTION_OXYGEN 0 /* combustion_oxygen (Kernel.cu:641-677): fuel, waste, temperature, flame;
                                   adds expansionRate x burn to the divergence */
#define HNS_COMBUSTION_RATE 1   /* combustion (Kernel.cu:568-588): where fuel > 0 and T >= ignition_temp,
                                   burn min(fuel, burn_rate dt); T += burned x heat_release */
#define HNS_COMBUSTION_NONE 2   /* no burn */

typedef struct hns_force_model {
    int combustion;         /* HNS_COMBUSTION_* */
    float burn_rate;        /* HNS_COMBUSTION_RATE */
    float heat_release;     /* HNS_COMBUSTION_RATE */
    float ignition_temp;    /* HNS_COMBUSTION_RATE */
    float density_buoyancy; /* alpha: v.y += (b_T - alpha density) dt, b_T the reference's temperature
                               buoyancy (max(0, (T - ambientTemp) buoyancyStrength) where
                               T > ambientTemp, else 0); 0 is the reference's buoyancy */
} hns_force_model;

/* hns_advance with a force model (NULL: the reference's). The fields the combustion model uses
 * are created zero-filled when missing (oxygen: fuel, waste, temperature, flame; rate: fuel,
 * temperature; none: temperature), and "density" when density_buoyancy != 0. */
HNS_API hns_status hns_advance_model(hns_ctx* ctx, int iterations, float dt, const hns_combustion_params* params,
                                     const hns_force_model* model);
/* ---- the all-in-one step on reduced-precision storage --------------------------------------
 * HNS_Advance's sequence (hns_advance_model) on caller-owned device arrays stored as BF16
 * velocity (3 per slot, interleaved) and FP16 scalars, with FP32 arithmetic and each pressure
 * solve the FP64 iterative refinement of hns_step_mixed, run to solve->tolerance instead of a
 * fixed iteration count. A field is given in both `in` and `out` or in neither; in and out must
 * not alias. temperature is required; fuel unless the model burns nothing; waste and flame for
 * the oxygen burn; density for a density buoyancy. Every field given is advected (the
 * reference's advect_scalars, along the projected velocity); the step creates no field. */
typedef struct hns_fire_fields {
    void* velocity;    /* BF16 [3N] */
    void* density;     /* FP16 [N] or NULL */
    void* temperature; /* FP16 [N] */
    void* fuel;        /* FP16 [N] or NULL */
    void* waste;       /* FP16 [N] or NULL */
    void* flame;       /* FP16 [N] or NULL */
} hns_fire_fields;

/* Sources added each substep, f += dt src (add_velocity_source / add_scalar_source,
 * src/Cuda/Kernel.cu:732-745); NULL entries (or a NULL struct) add nothing. */
typedef struct hns_fire_sources {
    const void* velocity;    /* BF16 [3N] */
    const void* temperature; /* FP16 [N] */
    const void* density;     /* FP16 [N] */
    const void* fuel;        /* FP16 [N] */
} hns_fire_sources;

/* One HNS_Advance call from `in` to `out` (params->substeps substeps of dt / substeps; the
 * intermediate states live in solver-owned arrays). solve: omega (inner SOR factor, <= 0:
 * 1.9), tolerance, max_outer, inner_iterations and flags as in hns_step_mixed; its dt is
 * ignored. With the disturbance branch (params->disturbanceEnable > 0) the velocity is solved
 * again after the buoyancy, as HNS_Advance does. With info the call synchronizes, reports the
 * last solve's inner iterations (outer x inner) and FP64 residual, and returns
 * HNS_ERR_NOT_CONVERGED when it is above the tolerance; every solve is also appended to the
 * convergence log (hns_solve_log). */
HNS_API hns_status hns_advance_mixed(hns_ctx* ctx, const hns_fire_fields* in, const hns_fire_fields* out,
                                     const hns_fire_sources* sources, float dt, const hns_combustion_params* params,
                                     const hns_force_model* model, const hns_mixed_desc* solve, hns_solve_info* info);

/* hns_advance_model with each pressure solve run to a tolerance instead of a fixed iteration
 * count: solve->tolerance (> 0), and either plain red-black SOR checked every check_every
 * iterations up to max_iterations, or (flags HNS_SOLVE_REFINE) the FP64 iterative refinement
 * around FP32 red-black inner solves (max_outer x inner_iterations); omega <= 0 selects
 * 2/(1+sin(3.14159 dx)). The FP32 step the mixed-precision hns_advance_mixed is compared with
 * at an equal residual. A collider ("collision_sdf") is supported by the plain solve only.
 * With info the call synchronizes and reports the last solve (HNS_ERR_NOT_CONVERGED above
 * the tolerance); every solve is appended to the convergence log. */
HNS_API hns_status hns_advance_solve(hns_ctx* ctx, float dt, const hns_combustion_params* params,
                                     const hns_force_model* model, const hns_step_desc* solve, hns_solve_info* info);

/* The fire step's fields and sources as FP32 arrays (the reference's GridIndexedData blocks):
 * host arrays for hns_advance_mixed_host, device arrays for the adjoints below. */
typedef struct hns_fire_f32 {
    float* velocity;    /* [3N] */
    float* density;     /* [N] or NULL */
    float* temperature; /* [N] */
    float* fuel;        /* [N] or NULL */
    float* waste;       /* [N] or NULL */
    float* flame;       /* [N] or NULL */
} hns_fire_f32;

typedef struct hns_fire_sources_f32 {
    const float* velocity;    /* [3N] or NULL */
    const float* temperature; /* [N] or NULL */
    const float* density;     /* [N] or NULL */
    const float* fuel;        /* [N] or NULL */
} hns_fire_sources_f32;

/* hns_advance_mixed from FP32 HOST arrays updated in place: uploads the fields and sources,
 * converts them to BF16/FP16 on the device, steps, converts back and downloads (synchronous).
 * Pinned host memory makes the copies faster. */
HNS_API hns_status hns_advance_mixed_host(hns_ctx* ctx, const hns_fire_f32* fields, const hns_fire_sources_f32* sources,
                                          float dt, const hns_combustion_params* params, const hns_force_model* model,
                                          const hns_mixed_desc* solve, hns_solve_info* info);

/* host uint8[num_voxels]: the activity mask of the last step (the reference's
 * build_activity_mask marks every slot active, src/Cuda/Kernel.cu:75). */
HNS_API hns_status hns_active_mask(hns_ctx* ctx, unsigned char* out);

/* ---- adjoints ----------------------------------------------------------------------------
 * Reverse-mode derivatives of the step's operators, for gradient-based use of the solver
 * (inverse design, control, learned closures). The reference has no adjoint path; these
 * differentiate the forward operators declared above. Each takes the forward operator's
 * inputs and the adjoint of its output (device arrays, same layouts) and ADDS the transpose of
 * the forward derivative, taken at those inputs, into the adjoint arrays of the inputs, which
 * the caller zeroes before their first use. Scatters use FP32 atomics, so the last bits vary
 * from run to run. */

/* hns_advect_scalar: in_bar += (d out / d in)^T out_bar, vel_bar += (d out / d vel)^T out_bar. */
HNS_API hns_status hns_adjoint_advect_scalar(hns_ctx* ctx, const float* vel, const float* in, const float* out_bar,
                                             float* in_bar, float* vel_bar, float dt);
/* hns_advect_vec3 (self-advection): vel_bar += (d out / d vel)^T out_bar. */
HNS_API hns_status hns_adjoint_advect_vec3(hns_ctx* ctx, const float* vel, const float* out_bar, float* vel_bar, float dt);
/* hns_divergence: vel_bar += D^T div_bar. */
HNS_API hns_status hns_adjoint_divergence(hns_ctx* ctx, const float* div_bar, float* vel_bar);
/* hns_subtract_gradient: vel_bar += out_bar (may be NULL to skip), p_bar += (d out / d p)^T out_bar. */
HNS_API hns_status hns_adjoint_subtract_gradient(hns_ctx* ctx, const float* out_bar, float* vel_bar, float* p_bar);
/* hns_rbgs from p = 0 (HNS_SOLVE_ZERO_INIT), `iterations` iterations: div_bar += M^T p_bar,
 * where p = M div is the linear map of the iterations. omega is used as given, as hns_rbgs
 * uses it. */
HNS_API hns_status hns_adjoint_rbgs(hns_ctx* ctx, const float* p_bar, float* div_bar, int iterations, float omega);
/* hns_project (`iterations` iterations from p = 0): vel_bar, the adjoint of the projected
 * velocity, becomes the adjoint of the velocity before the projection (in place). */
HNS_API hns_status hns_adjoint_project(hns_ctx* ctx, float* vel_bar, int iterations, float omega);
/* hns_vorticity_confinement: vel_bar += (d out / d vel)^T out_bar. */
HNS_API hns_status hns_adjoint_vorticity_confinement(hns_ctx* ctx, const float* vel, const float* out_bar, float* vel_bar,
                                                     float dt, float scale, float factor_scale);
/* hns_step_plain with a fixed iteration count (tolerance 0): from the step's inputs and the
 * adjoints of its outputs, adds the adjoints of its inputs (velocity and each scalar).
 * scalars_in, scalars_out_bar, scalars_in_bar: host arrays of nscalars device pointers. */
HNS_API hns_status hns_adjoint_step_plain(hns_ctx* ctx, const float* vel_in, const float* const* scalars_in, int nscalars,
                                          const float* vel_out_bar, const float* const* scalars_out_bar, float* vel_in_bar,
                                          float* const* scalars_in_bar, float dt, int iterations, float omega);

/* Adjoint of the fire step: hns_advance_model's step (one substep, no disturbance re-solve, no
 * collider) on FP32 device arrays with `iterations` red-black iterations per solve from p = 0
 * at HNS_Advance's omega. `in` are the step's inputs and `sources` its sources (as for the
 * step; NULL entries add nothing); out_bar the adjoints of its outputs (NULL scalar entries:
 * zero); in_bar receives, added, the adjoints of its inputs (zeroed by the caller; an entry
 * for every field of `in`). The forward is recomputed inside the call. Branches (MacCormack
 * clamps, trace cells, the burn's thresholds and minimum, T > ambient) are taken at the
 * forward's values. The reference has no adjoint path. */
HNS_API hns_status hns_adjoint_advance(hns_ctx* ctx, const hns_fire_f32* in, const hns_fire_sources_f32* sources,
                                       const hns_fire_f32* out_bar, const hns_fire_f32* in_bar, float dt, int iterations,
                                       const hns_combustion_params* params, const hns_force_model* model);
/* The same for hns_advance_mixed's step: inputs and sources in BF16/FP16 as that step takes them,
 * adjoints in FP32. Its solves run to solve->tolerance and are taken as exact, so the projection's
 * transpose is one more refined solve (the Laplacian is symmetric). */
HNS_API hns_status hns_adjoint_advance_mixed(hns_ctx* ctx, const hns_fire_fields* in, const hns_fire_sources* sources,
                                             const hns_fire_f32* out_bar, const hns_fire_f32* in_bar, float dt,
                                             const hns_combustion_params* params, const hns_force_model* model,
                                             const hns_mixed_desc* solve);

/* ---- options ----------------------------------------------------------------------------- */
#define HNS_OPT_RBGS_KERNEL 1 /* which red-black kernel: */
#define HNS_RBGS_PLAIN 0      /*   plain loads into a padded halo tile (also the zero-gradient walls' kernel) */
#define HNS_RBGS_BULK 1       /*   bulk async copies of the contiguous leaf payload into a staged tile, both
                                   colours per launch (used when div and p are 16-byte aligned) */
#define HNS_RBGS_SPLIT 2      /*   the solve on colour-split leaves, one in-place launch per colour, no
                                   staging (default; a call that runs single iterations, such as
                                   hns_project_static, takes HNS_RBGS_BULK). The three give the same
                                   results to the bit. */
#define HNS_OPT_INNER_LAYOUT 2 /* layout of the FP16 inner solve of the mixed-precision refinement: */
#define HNS_INNER_ROWS 0       /*   the leaf-dense slot order, relaxed by the HNS_RBGS_BULK kernel */
#define HNS_INNER_PACKED 1     /*   colour-packed rows (z = 0,2,4,6 then 1,3,5,7) with face buffers,
                                    staged by TMA, both colours per launch */
#define HNS_INNER_SPLIT 2      /*   colour-split leaves (a leaf's red values, then its black ones),
                                    one in-place launch per colour (default). All three give the
                                    same results to the bit; the solver's own arrays, never the
                                    caller's */
#define HNS_OPT_WAIT_POLLS 3    /* test hook of the timeout paths (value >= 0; -1 restores the
                                    defaults). The HNS_RBGS_BULK kernel: the poll limit of its first
                                    bounded copy wait; 0 makes every CTA give up at its first leaf, wait
                                    for its copies in flight with the normal limit, raise the device
                                    error flag (hns_device_status) and return, leaving p_out
                                    unfinished. The persistent colour-split solves (HNS_SPLIT_PERSISTENT):
                                    every dependency wait behaves as if the neighbour never finished and
                                    gives up after `value` polls, raising the flag; every CTA then
                                    returns, leaving the solve unfinished. */
#define HNS_OPT_SPLIT_SOLVE 4   /* how the colour-split solves (HNS_RBGS_SPLIT, HNS_INNER_SPLIT) launch: */
#define HNS_SPLIT_PER_COLOUR 0  /*   one launch per half-sweep (programmatic dependent launches;
                                     default: the faster of the two on a B200) */
#define HNS_SPLIT_PERSISTENT 1  /*   one cooperative launch per inner solve, or per run of iterations
                                     between convergence checks, leaf groups ordered by per-group
                                     progress counters instead of launch boundaries. Both give the
                                     same results to the bit. */
#define HNS_OPT_COARSE_SOLVE 5  /* how the FP16 multigrid cycle (HNS_SOLVE_MULTIGRID) solves its coarsest
                                     level, one cell per leaf: */
#define HNS_COARSE_LAUNCHES 0   /*   two launches per SOR sweep */
#define HNS_COARSE_CLUSTER 1    /*   all sweeps in one launch of a 16-CTA thread-block cluster (8 where
                                     the device cannot schedule 16) that holds the level in shared
                                     memory (default; up to 5,810 leaves per CTA, 92,960 in all with 16;
                                     larger domains take HNS_COARSE_LAUNCHES). Both give the same
                                     results to the bit. */
#define HNS_OPT_L2_PERSIST 6    /* 1 (default): where the FP16 inner solve's correction array fits the
                                     device's persisting-L2 maximum (79 MB on a B200: grids up to about
                                     41M voxels), it is marked persisting in L2 while a refined solve
                                     runs (an access-policy window on the inner solve's launches; the
                                     process's persisting-L2 limit is raised to hold it, once per
                                     context); 0: ordinary caching. The results are the same to the bit. */
HNS_API hns_status hns_set_option(hns_ctx* ctx, int option, int value);
/* Device-side error flags raised since the last call (bounded waits that gave up): returns
 * HNS_ERR_TIMEOUT and clears them if any was raised, else HNS_OK. Synchronizes. */
HNS_API hns_status hns_device_status(hns_ctx* ctx);

/* ---- profiling --------------------------------------------------------------------------
 * While enabled, the step entry points record CUDA events on the context's stream around
 * each phase; hns_profile_read sums them (synchronizes) and resets. */
#define HNS_PHASE_ADVECT 0
#define HNS_PHASE_DIVERGENCE 1
#define HNS_PHASE_SOLVE 2
#define HNS_PHASE_GRADIENT 3
#define HNS_PHASE_FORCES 4
#define HNS_PHASE_INNER 5 /* refinement: the inner red-black iterations (also counted in SOLVE) */
#define HNS_NUM_PHASES 8

typedef struct hns_profile_data {
    double phase_ms[HNS_NUM_PHASES];        /* device time per phase since the last read */
    int phase_count[HNS_NUM_PHASES];        /* phase executions since the last read */
    unsigned long long solver_launches;     /* red-black sweeps that ran (not skipped): launches, and
                                               the half-sweeps inside a persistent inner solve */
    unsigned long long kernel_launches;     /* the library's kernel launches since the last read, of
                                               every context of the process (memsets not counted) */
} hns_profile_data;

HNS_API hns_status hns_profile_enable(hns_ctx* ctx, int enable);
HNS_API hns_status hns_profile_read(hns_ctx* ctx, hns_profile_data* out);

#ifdef __cplusplus
}
#endif

#endif /* HNS_H */
