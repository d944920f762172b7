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
    void hnso_combustion_oxygen##S(int64_t n, const R* fuel, const R* waste, const R* temp, R* div, const R* flame, \
                                   R* o_fuel, R* o_waste, R* o_temp, R* o_flame, R gain, R expansion);             \
    void hnso_add_scalar_source##S(int64_t n, R* field, const R* src, R dt);                                       \
    void hnso_add_velocity_source##S(int64_t n, R* vel, const R* src, R dt);                                       \
    void hnso_add_velocity_source_xyz##S(int64_t n, R* vel, const R* sx, const R* sy, const R* sz, R dt);          \
    void hnso_add_gravity##S(int64_t n, R* vel, R g, R dt);                                                        \
    void hnso_project##S(const hnso_topo* t, R* vel, R* div, R* p, R dx, int iterations, R omega);                \
    void hnso_enforce_collision##S(const hnso_topo* t, R* vel, const R* sdf, R inv_dx);

HNSO_DECLARE(float, _f32)
HNSO_DECLARE(double, _f64)

/* Fields of one HNS_Advance call (src/Cuda/HNanoSolver.cu:223-456). `names`/`scalars` are
 * the persistent scalar fields present when the call starts; exactly these are advected.
 * fuel/waste/temperature/flame absent from that list are created zero-filled on first use
 * in `created` (n floats each) and are not advected during this call. */
typedef struct {
    int64_t n;
    float* velocity;
    int nscalars;
    const char* const* names;
    float* const* scalars;
    float* created[4];
    const float* src_vel;
    const float* src_vel_x;
    const float* src_vel_y;
    const float* src_vel_z;
    const float* src_temperature;
    const float* src_density;
    const float* src_fuel;
    const float* collision_sdf; /* n, or NULL: no collider */
} hnso_advance_fields;

void hnso_hns_advance_f32(const hnso_topo* t, const hnso_advance_fields* f, float dx, int iteration, float dt,
                          const hnso_combustion_params* params);

#ifdef __cplusplus
}
#endif

#endif
