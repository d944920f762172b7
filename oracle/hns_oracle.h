/* CPU oracle for the sparse smoke/fire step: a plain-C restatement of the reference's
 * kernels and step sequence.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product links or calls this library; only
 * tests/, bench.py's CPU-baseline leg and the smoke check load it, as the checker.
 *
 * Parity pins: the restatement is checked (tests/test_oracle.py) against
 *   - the reference's own kernels compiled from src/Cuda/Kernel.cu as host C++
 *     (oracle/ref_driver.cpp -> oracle/_ref/libhns_ref.so), on the same inputs;
 *   - golden vectors that build made with that library (tests/golden/), and the sampler
 *     and layout known answers of Tests/IndexGrid.cpp restated on the leaf-dense layout.
 *
 * Every function exists in two precisions, suffix _f32 (float, the reference's) and _f64
 * (the same arithmetic in double, for error statements against an FP64 oracle).
 * Layout: leaf-dense slots, slot = 512*leaf + ((x&7)<<6 | (y&7)<<3 | (z&7)); vec3 fields
 * are interleaved x,y,z per slot (the reference's nanovdb::Vec3f arrays).
 */
#ifndef HNS_ORACLE_H
#define HNS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hnso_topo hnso_topo;

/* Leaves in the caller's order: leaf i owns slots [512 i, 512 i + 512). */
hnso_topo* hnso_topo_create(const int32_t* leaf_origins, int64_t num_leaves);
void hnso_topo_destroy(hnso_topo* t);
int64_t hnso_topo_num_voxels(const hnso_topo* t);
/* NanoVDB ValueOnIndex offset of a voxel: 0 outside the domain, else 1 + slot. */
uint64_t hnso_offset(const hnso_topo* t, int32_t i, int32_t j, int32_t k);
void hnso_offsets(const hnso_topo* t, const int32_t* ijk, int64_t n, uint64_t* out);
/* Coordinates of every slot (3 int32 per slot). */
void hnso_slot_coords(const hnso_topo* t, int32_t* out);
/* Sort leaf origins in place into NanoVDB's leaf order (the order value offsets of a
 * ValueOnIndex grid are assigned in). */
void hnso_sort_leaves_nanovdb(int32_t* leaf_origins, int64_t num_leaves);

/* Parameters of the reference's step (src/Cuda/Kernels.cuh:5-24, same layout). */
typedef struct {
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
} hnso_combustion_params;

#define HNSO_DECLARE(R, S)                                                                                         \
    void hnso_sample_trilinear_scalar##S(const hnso_topo* t, const R* data, const R* xyz, int64_t n, R* out);       \
    void hnso_sample_trilinear_vec3##S(const hnso_topo* t, const R* data, const R* xyz, int64_t n, R* out);         \
    void hnso_advect_vector##S(const hnso_topo* t, const R* vel, R* out, R dt, R inv_dx);                          \
    void hnso_advect_scalars##S(const hnso_topo* t, const R* vel, const R* const* in, R* const* out, int nfields,   \
                                R dt, R inv_dx);                                                                   \
    void hnso_advect_scalar##S(const hnso_topo* t, const R* vel, const R* in, R* out, R dt, R inv_dx);             \
    void hnso_divergence##S(const hnso_topo* t, const R* vel, R* div, R inv_dx);                                   \
    void hnso_rbgs_sweep##S(const hnso_topo* t, const R* div, R* p, R dx, int color, R omega);                     \
    void hnso_rbgs##S(const hnso_topo* t, const R* div, R* p, R dx, int iterations, R omega);                      \
    void hnso_residual##S(const hnso_topo* t, const R* div, const R* p, R dx, double* r2, double* b2);             \
    void hnso_subtract_gradient##S(const hnso_topo* t, const R* vel, const R* p, R* out, R inv_dx);                \
    void hnso_vorticity_confinement##S(const hnso_topo* t, const R* vel, R* out, R dt, R inv_dx, R scale,          \
                                       R factor_scale);                                                            \
    void hnso_temperature_buoyancy##S(int64_t n, const R* vel, const R* temp, R* out, R dt, R ambient,             \
                                      R strength);                                                                 \
    void hnso_combustion##S(int64_t n, const R* fuel, const R* temp, R* out_fuel, R* out_temp, R dt, R ignition,   \
                            R rate, R heat);                                                                       \
    void hnso_buoyancy_density##S(int64_t n, const R* vel, const R* temp, const R* density, R* out, R dt,        \
                                  R ambient, R strength, R alpha);                                               \
    void hnso_combustion_oxygen##S(int64_t n, const R* fuel, const R* waste, const R* temp, R* div, const R* flame, \
                                   R* o_fuel, R* o_waste, R* o_temp, R* o_flame, R gain, R expansion);             \
    void hnso_add_scalar_source##S(int64_t n, R* field, const R* src, R dt);                                       \
    void hnso_add_velocity_source##S(int64_t n, R* vel, const R* src, R dt);                                       \
    void hnso_add_velocity_source_xyz##S(int64_t n, R* vel, const R* sx, const R* sy, const R* sz, R dt);          \
    void hnso_add_gravity##S(int64_t n, R* vel, R g, R dt);                                                        \
    void hnso_project##S(const hnso_topo* t, R* vel, R* div, R* p, R dx, int iterations, R omega);                \
    void hnso_rbgs_sweep_neumann##S(const hnso_topo* t, const R* div, R* p, R dx, int color, R omega);            \
    void hnso_rbgs_neumann##S(const hnso_topo* t, const R* div, R* p, R dx, int iterations, R omega);             \
    void hnso_residual_neumann##S(const hnso_topo* t, const R* div, const R* p, R dx, double* r2, double* b2);    \
    void hnso_remove_mean##S(const hnso_topo* t, R* div);                                                        \
    void hnso_subtract_gradient_neumann##S(const hnso_topo* t, const R* vel, const R* p, R* out, R inv_dx);       \
    void hnso_project_neumann##S(const hnso_topo* t, R* vel, R* div, R* p, R dx, int iterations, R omega);        \
    void hnso_enforce_collision##S(const hnso_topo* t, R* vel, const R* sdf, R inv_dx);

HNSO_DECLARE(float, _f32)
HNSO_DECLARE(double, _f64)

/* Fields of one HNS_Advance call (src/Cuda/HNanoSolver.cu:223-456), in float (_f32) or double
 * (_f64). `names`/`scalars` are the persistent scalar fields present when the call starts;
 * exactly these are advected. fuel/waste/temperature/flame absent from that list are created
 * zero-filled on first use in `created` (n values each, in that order) and are not advected
 * during this call. */
#define HNSO_ADVANCE_FIELDS(R, S)                                                                                  \
    typedef struct {                                                                                               \
        int64_t n;                                                                                                 \
        R* velocity;                                                                                               \
        int nscalars;                                                                                              \
        const char* const* names;                                                                                  \
        R* const* scalars;                                                                                         \
        R* created[4];                                                                                             \
        const R* src_vel;                                                                                          \
        const R* src_vel_x;                                                                                        \
        const R* src_vel_y;                                                                                        \
        const R* src_vel_z;                                                                                        \
        const R* src_temperature;                                                                                  \
        const R* src_density;                                                                                      \
        const R* src_fuel;                                                                                         \
        const R* collision_sdf; /* n, or NULL: no collider */                                                      \
    } hnso_advance_fields##S;
HNSO_ADVANCE_FIELDS(float, _f32)
HNSO_ADVANCE_FIELDS(double, _f64)
typedef hnso_advance_fields_f32 hnso_advance_fields;

/* Force model of the step. The zero value is the reference's HNS_Advance.
 * combustion: 0 combustion_oxygen (src/Cuda/Kernel.cu:641-677, the reference's step),
 *             1 combustion (Kernel.cu:568-588: burn min(fuel, burn_rate dt) where fuel > 0
 *               and T >= ignition_temp, T += burned heat_release), 2 none.
 * density_buoyancy: alpha of the buoyancy's density term v.y -= alpha density dt (an
 *             extension; the reference has none).
 * omega:      > 0 replaces the solves' SOR factor 2/(1+sin(3.14159 dx)). */
typedef struct {
    int combustion;
    double burn_rate;
    double heat_release;
    double ignition_temp;
    double density_buoyancy;
    double omega;
} hnso_force_model;

void hnso_hns_advance_f32(const hnso_topo* t, const hnso_advance_fields* f, float dx, int iteration, float dt,
                          const hnso_combustion_params* params);
void hnso_hns_advance_model_f32(const hnso_topo* t, const hnso_advance_fields_f32* f, float dx, int iteration, float dt,
                                const hnso_combustion_params* params, const hnso_force_model* model);
void hnso_hns_advance_model_f64(const hnso_topo* t, const hnso_advance_fields_f64* f, double dx, int iteration,
                                double dt, const hnso_combustion_params* params, const hnso_force_model* model);

#ifdef __cplusplus
}
#endif

#endif
