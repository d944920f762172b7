// Internal declarations of libhns: the context, the device topology view and error
// plumbing. Not installed; the public surface is include/hns.h.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "hns.h"

namespace hns {

// ---- errors --------------------------------------------------------------------------------

struct Error : std::runtime_error {
    hns_status status;
    Error(hns_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

[[noreturn]] void fail(hns_status s, const std::string& msg);
void cuda_check(cudaError_t e, const char* what, const char* file, int line);
#define HNS_CUDA(call) ::hns::cuda_check((call), #call, __FILE__, __LINE__)
#define HNS_LAUNCHED() (::hns::note_launch(), ::hns::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__))
// Counts the library's kernel launches (process-wide; hns_profile_read reports and resets it).
void note_launch();
extern std::atomic<unsigned long long> g_kernel_launches;

hns_status record_error(hns_status s, const std::string& msg);
void clear_error();

// Runs `body` and turns any exception into a status (no exception crosses the C ABI).
template <typename F>
hns_status guarded(F&& body) {
    try {
        clear_error();
        body();
        return HNS_OK;
    } catch (const Error& e) {
        return record_error(e.status, e.what());
    } catch (const std::bad_alloc&) {
        return record_error(HNS_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return record_error(HNS_ERR_INVALID_ARG, e.what());
    }
}

// ---- device memory -------------------------------------------------------------------------

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t n) { alloc(n); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr, o.bytes = 0; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) {
            reset();
            ptr = o.ptr, bytes = o.bytes;
            o.ptr = nullptr, o.bytes = 0;
        }
        return *this;
    }
    ~DeviceBuffer() { reset(); }
    void alloc(size_t n);
    void reset() noexcept;
    template <typename T>
    T* as() const { return static_cast<T*>(ptr); }
};

// ---- topology ------------------------------------------------------------------------------

// Device view of the leaf table. A coordinate's leaf is found either through the 27-leaf
// neighbourhood of the leaf being processed (staged in shared memory by the kernels) or
// through `lookup`, a dense table over the leaves' bounding box in leaf units.
struct TopoView {
    int64_t num_leaves;
    const int4* origin;   // [L] leaf origins (w unused)
    const int* nbr27;     // [L][27] neighbour leaf indices, -1 = none; index (dx+1)*9+(dy+1)*3+(dz+1)
    const int* lookup;    // dense leaf table, -1 = none
    int lo_x, lo_y, lo_z; // table origin in leaf units (coordinate >> 3)
    int dim_x, dim_y, dim_z;
};

struct Topology {
    int64_t num_leaves = 0;
    std::vector<int32_t> origins;  // host copy, 3 per leaf
    DeviceBuffer d_origin, d_nbr27, d_lookup;
    TopoView view{};
    bool nanovdb_order = false;
    void build(const int32_t* leaf_origins, int64_t n, cudaStream_t stream);
    // The leaves that the active voxels ijk (int32 [3 n], host or device) touch after a
    // 26-neighbour dilation by `padding` voxels, in NanoVDB order, built on the device
    // (hns_topology.cu).
    void build_from_voxels(const int32_t* ijk, int64_t n, bool ijk_on_device, int padding, cudaStream_t stream);
};

bool leaves_in_nanovdb_order(const int32_t* origins, int64_t n);
void sort_leaves_nanovdb(int32_t* origins, int64_t n);

// ---- context ------------------------------------------------------------------------------

// A named device field of the context (the reference's SimContext d_state / d_src maps).
struct Field {
    std::string name;
    int components;  // 1 or 3 (vec3 interleaved)
    DeviceBuffer buf;
};

// Schedule of one iterative-refinement solve (hns_mixed.cu): slots holds 2 doubles per
// residual check (max_outer + 1 checks) followed by the per-outer FP32 scales.
struct RefinePlan {
    int max_outer = 0;
    int inner = 0;
    double tol = 0.0;
    bool inner_fp16 = true;
    double* slots = nullptr;
};

// Schedule of one convergence-checked pressure solve (see rbgs_solve_checked).
struct SolvePlan {
    int max_iterations = 0;
    int check_every = 0;
    int num_checks = 0;
    double tol = 0.0;
    double* slots = nullptr;
};

// FP64 accumulators per context: 8 scratch doubles + 2 per convergence check.
constexpr int kMaxChecks = 4096;
constexpr int kReduceSlots = 8 + 2 * kMaxChecks;

struct Context {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    // A second stream for copies that can overlap the step (the host-buffer forms), made on
    // first use, and the event that orders it after the main stream.
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t aux_ready = nullptr;
    void ensure_aux();
    // Two pinned staging buffers for host copies (hns_transfer.cpp), made on first use, and the
    // events that order their reuse.
    void* staging[2] = {nullptr, nullptr};
    cudaEvent_t staging_done[2] = {nullptr, nullptr};
    void ensure_staging();
    void release_staging();
    float dx = 0.f;
    Topology topo;
    // Scratch owned by the context, grown on demand and reused across calls.
    std::map<std::string, DeviceBuffer> scratch;
    DeviceBuffer d_reduce;  // FP64 reduction accumulators, allocated once (kReduceSlots doubles)
    // Convergence log (hns_solve_log): kSolveLogCap entries of (iterations, residual) written on
    // the device by every checked or refined solve, then the count of entries appended (as a
    // 64-bit integer in the last slot). Allocated with the context.
    static constexpr int kSolveLogCap = 4096;
    DeviceBuffer d_solve_log;
    // Face-connected components of the leaves (hns_neumann.cu), made on the first solve with
    // zero-gradient walls: the component of each leaf, the voxels of each, FP64 sums.
    int num_components = 0;
    int leaf_depth = -1;  // max_leaf_depth(), computed once (hns_neumann.cu)
    DeviceBuffer d_components, d_component_counts, d_component_sums;
    SolvePlan last_solve;   // schedule of the most recent checked solve (hns_last_solve)
    RefinePlan last_refine; // schedule of the most recent refined solve (hns_last_refine)
    // Profiling (hns_profile_*): device counters and per-phase events on the stream.
    DeviceBuffer d_counters;
    unsigned long long* counters = nullptr;  // [0] red-black sweeps that ran (not skipped), [1] device error flag
    bool profiling = false;
    int rbgs_kernel = HNS_RBGS_SPLIT;     // hns_set_option(HNS_OPT_RBGS_KERNEL)
    int inner_layout = HNS_INNER_SPLIT;  // hns_set_option(HNS_OPT_INNER_LAYOUT)
    int first_wait_polls = -1;           // hns_set_option(HNS_OPT_WAIT_POLLS); -1: the kernel's default
    int split_solve = HNS_SPLIT_PER_COLOUR;  // hns_set_option(HNS_OPT_SPLIT_SOLVE)
    int coarse_solve = HNS_COARSE_CLUSTER;   // hns_set_option(HNS_OPT_COARSE_SOLVE)
    int l2_persist = 1;                      // hns_set_option(HNS_OPT_L2_PERSIST)
    // The access-policy window of the inner solve's launches while a refined solve runs
    // (num_bytes 0: none); added to their launch attributes by add_inner_window().
    cudaAccessPolicyWindow inner_window = {};
    size_t l2_persist_limit = 0;  // the persisting-L2 limit this context has set
    unsigned add_inner_window(cudaLaunchAttribute* attr, unsigned n) const {
        if (inner_window.num_bytes == 0) return n;
        attr[n].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[n].val.accessPolicyWindow = inner_window;
        return n + 1;
    }
    int coarse_cluster_ok = -1;     // CTAs of the coarsest level's cluster, 0 if none fits (-1: not chosen)
    int64_t coarse_table_leaves = -1;  // leaves of the coarsest level's cluster records made so far
    // Graphs of the multigrid refinement's outer iterations past the forecast (hns_mixed.cu): a
    // device-side condition runs the iteration only while the solve has not converged. Made on
    // first use per set of arguments; 0 in spare_graph_ok after one could not be made (those
    // iterations then launch as the others do).
    struct SpareGraph {
        std::vector<uintptr_t> key;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
    };
    std::vector<SpareGraph> spare_graphs;
    int spare_graph_ok = -1;
    void release_spare_graphs();
    // Whether the context's stream is being captured into a graph (work enqueued now runs only
    // when the graph does: a table built under capture is not marked built).
    bool stream_capturing() const;
    struct PhaseEvent {
        int phase;
        cudaEvent_t start, stop;
    };
    std::vector<PhaseEvent> phase_events;
    std::vector<size_t> open_phases;  // indices into phase_events (phases nest)
    void phase_begin(int phase);
    void phase_end();
    // Named fields in insertion order.
    std::vector<Field> fields;
    Field* find_field(const std::string& name);
    Field& ensure_field(const std::string& name, int components, bool zero);

    // Forecast of the refinement's outer iterations (hns_mixed.cu): each refined solve copies its
    // residual checks to pinned memory behind an event; a later solve whose event has completed
    // reads the count of outer iterations it needed. Outer iterations past the forecast launch
    // their kernels on short grids, so that when they return at once they cost little.
    double* refine_echo = nullptr;  // pinned, kEchoSlots doubles
    cudaEvent_t refine_echo_done = nullptr;
    bool refine_echo_pending = false;
    int refine_echo_outer = 0;      // max_outer of the solve in refine_echo
    double refine_echo_tol = 0.0;   // its tolerance
    int refine_forecast = 0;        // outer iterations the last read-back solve needed; 0: unknown
    static constexpr int kEchoSlots = 2 * (64 + 1);
    // Colour-split solves: the face-table buffer whose table is built, and the e buffers whose
    // zero leaf (past the last leaf) is cleared: the FP16 inner solve's, the FP32 solve's, the FP32
    // inner solve's.
    const void* split_faces_built = nullptr;
    const void* split_zero_leaf[3] = {nullptr, nullptr, nullptr};
    // The face table (built once) and a colour-split e buffer of n + 512 elements of `bytes`
    // each whose zero leaf is cleared once (which: index into split_zero_leaf).
    int* split_faces();
    void* split_e(const char* name, size_t bytes, int which);
    mutable int sms = 0;
    int sm_count() const;  // multiprocessors of the device (queried once)

    int64_t num_voxels() const { return topo.num_leaves * 512; }
    float* scratch_f32(const std::string& name, size_t count);
    double* reduce_slots(int count);
};

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev);
    ~DeviceGuard();
};

Context* check_ctx(hns_ctx* ctx);
const Context* check_ctx(const hns_ctx* ctx);

// ---- kernels (hns_kernels.cu) --------------------------------------------------------------

constexpr int kMaxAdvectFields = 16;

struct FieldSet {
    const float* in[kMaxAdvectFields];
    float* out[kMaxAdvectFields];
    int count;
};

// Velocity (vel_out, may be null) and HNanoAdvect scalars (f) along one shared trace.
// sdf (or null): the collision SDF of HNS_Advance's step.
void launch_advect_fused(const Context& c, const float* vel, float* vel_out, const FieldSet& f, float dt,
                         const float* sdf = nullptr);
void launch_advect_scalars(const Context& c, const float* vel, const FieldSet& f, float dt, const float* sdf = nullptr);
void launch_collision_enforce(const Context& c, float* vel, const float* sdf);
void launch_divergence(const Context& c, const float* vel, float* div);
// One fused red+black iteration: p_in -> p_out (ping-pong). p_in == nullptr means p = 0.
// check/tol2: skip when check[0] <= tol2 * check[1]; resid_out: accumulate the residual of
// p_in (FP64 {sum r^2, sum b^2}).
void launch_rbgs_iteration(const Context& c, const float* div, const float* p_in, float* p_out, float omega,
                           unsigned flags, const double* check = nullptr, double tol2 = 0.0,
                           double* resid_out = nullptr);
// The bulk-copy form of the iteration (hns_rbgs.cu); needs 16-byte aligned arrays.
bool rbgs_bulk_eligible(const float* div, const float* p_in, const float* p_out);
void launch_rbgs_bulk(const Context& c, const float* div, const float* p_in, float* p_out, float omega,
                      const double* check, double tol2, double* resid_out);
// The same iteration on FP16 storage (FP32 arithmetic) with unit dx^2: the inner solve of the
// mixed-precision refinement, L e = rhs. e_in null means e = 0.
void launch_rbgs_bulk_half(const Context& c, const void* rhs, const void* e_in, void* e_out, float omega,
                           const double* check, double tol2);
// flags: HNS_SOLVE_NEUMANN takes a missing neighbour's pressure as the voxel's own.
void launch_subtract_gradient(const Context& c, const float* vel, const float* p, float* out, const float* sdf = nullptr,
                              unsigned flags = 0);
// Zero-gradient walls (hns_neumann.cu): removes the mean of div (n values) per face-connected
// component of the leaves, the sums in FP64.
void remove_divergence_mean(Context& c, float* div);
void launch_vorticity(const Context& c, const float* vel, float* out, float dt, float scale, float factor_scale);
// acc[0] += sum (b - A p)^2, acc[1] += sum b^2 with b = div dx^2 (FP64).
void launch_residual(const Context& c, const float* div, const float* p, double* acc, unsigned flags);
void launch_index_offsets(const Context& c, const int32_t* ijk, int64_t n, uint64_t* out);

// The FP16 iteration on colour-packed rows (hns_rbgs_packed.cu): slot 8 r + z of a row r
// holds z at position (z & 1) * 4 + (z >> 1). rhs, e_in, e_out in that layout; faces_in/out the
// face buffers of e_in/e_out (kPackedFaceBytes per leaf; the kernel writes faces_out); halo the
// rhs halo records (kPackedHaloBytes per leaf, from launch_rhs_halo_pack). e_in null: e = 0.
constexpr int kPackedFaceBytes = 1024;
constexpr int kPackedHaloBytes = 640;
void launch_rhs_halo_pack(const Context& c, const void* rhs, void* halo, const double* check, double tol2);
// Host <-> device copies of `bytes` through pinned staging, overlapping the host-side copy with
// the DMA (hns_transfer.cpp). Both return when the data has arrived.
void copy_h2d(Context& c, void* dev, const void* host, size_t bytes);
void copy_d2h(Context& c, void* host, const void* dev, size_t bytes);
// One multigrid V-cycle (hns_multigrid.cu): u0 (n FP32) ~ A^-1 b0 for the unit-spacing system.
void mg_vcycle(Context& c, const float* b0, float* u0, const double* check, double tol2);
// How many leaves deep the domain is: the largest face-step distance from a leaf to one with a
// missing face neighbour (host, once per context).
int max_leaf_depth(Context& c);
// Process-wide settings of a device that several contexts share, only ever raised so that no
// context lowers another's: `which` 0 is the coarsest-level cluster kernel's dynamic shared
// memory limit, 1 the persisting-L2 limit. Returns the value now in force (>= value).
size_t raise_device_setting(int device, int which, size_t value);
// One V-cycle of the FP16 inner solve on the colour-split layout (e in place; e_zero: e = 0 before).
void mg16_vcycle(Context& c, const int* nb8, const void* rhat, void* e, bool e_zero, const double* check, double tol2);
// The FP16 inner solve on colour-split leaves (hns_rbgs_split.cu): the face-neighbour table
// (8 ints per leaf, missing neighbours = the zero leaf L) and one in-place half-sweep (colour 0
// red, 1 black). e holds L + 1 leaves, the last all zeros. e_zero: e = 0 before this red
// half-sweep (the first of a solve); a launch with e_zero false is a programmatic dependent
// launch, so the preceding kernel on the stream must be a half-sweep, and rhs, nb8 and check
// must have been written by kernels that finished before that one started.
void launch_split_face_table(const Context& c, int* nb8);
// short_grid: one wave of CTAs looping over the leaves, for a launch expected to find the
// refinement converged and return at once.
void launch_rbgs_split_half(const Context& c, const int* nb8, const void* rhs, void* e, int colour, bool e_zero,
                            float omega, const double* check, double tol2, bool short_grid = false);
// A whole FP16 inner solve on colour-split leaves in one cooperative launch: half_sweeps
// half-sweeps (red first), the values of as many launch_rbgs_split_half calls to the bit. e_zero:
// e = 0 before it. Follows any kernel (no programmatic dependency).
void launch_rbgs_split_solve(Context& c, const int* nb8, const void* rhs, void* e, int half_sweeps, bool e_zero,
                             float omega, const double* check, double tol2);
// The same for the FP32 solve (the half-sweeps of launch_rbgs_split_half_f32).
void launch_rbgs_split_solve_f32(Context& c, const int* nb8, const float* rhs, float* e, int half_sweeps, bool e_zero,
                                 float omega, float dx2, const double* check, double tol2);
// The FP32 half-sweep on colour-split leaves (the reference's update and precision): rhs the
// divergence in the split layout, scaled by dx2 in each update; e in place with the zero leaf.
// Launches with e_zero false are programmatic dependent launches: pdl false for one that follows
// a kernel other than a half-sweep.
void launch_rbgs_split_half_f32(const Context& c, const int* nb8, const float* rhs, float* e, int colour, bool e_zero,
                                float omega, float dx2, const double* check, double tol2, bool short_grid = false,
                                bool pdl = true);
// FP32 slot order <-> colour-split order (n values).
void convert_split_f32(const Context& c, const float* src, float* dst, bool to_split);
// acc += {sum r^2, sum b^2} of the FP32 split iterate e (FP64), unless check has passed.
void launch_split_residual_f32(const Context& c, const int* nb8, const float* rhs, const float* e, double h2,
                               const double* check, double tol2, double* acc);
void launch_rbgs_packed_half(const Context& c, const void* rhs, const void* halo, const void* e_in, const void* faces_in,
                             void* e_out, void* faces_out, float omega, const double* check, double tol2);

// Same iteration in FP32 with unit dx^2 (the FP32-inner refinement): L e = rhs.
void launch_rbgs_bulk_unit(const Context& c, const float* rhs, const float* e_in, float* e_out, float omega,
                           const double* check, double tol2);

// ---- adjoints (hns_adjoint.cu): each adds its transpose into the adjoint arrays ----
void launch_adj_advect_scalar(const Context& c, const float* vel, const float* in, const float* out_bar, float* in_bar,
                              float* vel_bar, float dt);
void launch_adj_advect_vec3(const Context& c, const float* vel, const float* out_bar, float* vel_bar, float dt);
void launch_adj_divergence(const Context& c, const float* div_bar, float* vel_bar);
void launch_adj_gradient(const Context& c, const float* out_bar, float* p_bar);
void launch_adj_rbgs_colour(const Context& c, float* lam, float* div_bar, int colour, float keep, float nbr, float dmul);
void launch_adj_confinement(const Context& c, const float* vel, const float* out_bar, float* vel_bar, float dt,
                            float scale, float factor_scale);
void launch_adj_accumulate(const Context& c, const float* src, float* dst, int64_t n);
// div_bar += M^T p_bar for `iterations` red-black iterations from p = 0 (p = M div).
void adj_rbgs(Context& c, const float* p_bar, float* div_bar, int iterations, float omega);

// ---- mixed precision and refinement (hns_mixed.cu) ----
void convert_array(const Context& c, const void* src, int src_dt, void* dst, int dst_dt, int64_t n);
template <typename TI>
// flags: HNS_SOLVE_MULTIGRID selects a multigrid V-cycle as the inner solve.
RefinePlan refine_solve(Context& c, const float* div, double* p, int max_outer, int inner, float omega, double tol,
                        unsigned flags = 0);
void refine_result(Context& c, const RefinePlan& plan, int* outer, double* residual);
void launch_advect_mixed(Context& c, const void* vel, void* vel_out, const void* const* sin, void* const* sout, int ns,
                         float dt);
void launch_divergence_mixed(const Context& c, const void* vel, float* div);
void launch_gradient_mixed(const Context& c, void* vel, const double* p);
// u -= grad p for an FP32 velocity and an FP64 pressure, in place.
void launch_gradient_f64(const Context& c, float* vel, const double* p);

// HNS_Advance over the context's fields with a force model (hns_advance.cu).
// solve: null runs `iterations` red-black iterations per solve (the reference); otherwise each
// solve runs to solve->tolerance (checked SOR, or the FP32 refinement with HNS_SOLVE_REFINE) and,
// with info, the last solve's result is reported (synchronizes).
void run_advance(Context& c, int iterations, float dt, const hns_combustion_params& params, const hns_force_model& model,
                 const hns_step_desc* solve, hns_solve_info* info);
void check_force_model(const hns_force_model& m);
// The step's force kernels (hns_advance.cu): confinement + velocity source + gravity, vel -> out;
// divergence + burn (in place on its fields) + buoyancy, vel -> vel_out.
void launch_confine_sources(const Context& c, const float* vel, float* out, float dt, float scale, float factor_scale,
                            const float* src_v3, float gravity);
void launch_div_combust_buoy(const Context& c, const float* vel, float* vel_out, float* div, float* fuel, float* waste,
                             float* temp, float* flame, const float* density, const hns_combustion_params& P,
                             const hns_force_model& M, float dt);

// Runs `iterations` fused RBGS iterations from `p` (or zero) and leaves the result in `p`.
void rbgs_solve(Context& c, const float* div, float* p, int iterations, float omega, unsigned flags);
// The FP32 solve on colour-split leaves (hns_step.cu): whether a solve with these flags takes it,
// and the solve (plan: the convergence checks of rbgs_solve_checked, or null).
bool use_split32(const Context& c, unsigned flags, const float* div, const float* p);
void split32_solve(Context& c, const float* div, float* p, int K, float omega, unsigned flags, const SolvePlan* plan);

// Convergence-checked solve: at most `max_iterations` (rounded up to even) iterations; the
// FP64 residual of the iterate is evaluated inside the sweep every `check_every` iterations
// and the remaining launches return at once when ||r|| <= tol ||b||. Enqueues only; the
// check slots (2 doubles per check, from c.reduce_slots) are read by solve_result().

SolvePlan rbgs_solve_checked(Context& c, const float* div, float* p, int max_iterations, float omega, unsigned flags,
                             double tol, int check_every);
// Host readback (synchronizes): iterations run and the last evaluated relative residual.
void solve_result(Context& c, const SolvePlan& plan, int* iterations, double* residual);
// Appends a solve's result to the context's convergence log on the device (no host wait). The
// solve's checks are nchecks pairs {sum r^2, sum b^2}; the first passing check q (r^2 <= tol^2
// b^2) stands for (q + offset) * per iterations; when none passes, the entry has cap_iterations
// and the last check's residual.
void log_solve(Context& c, const double* checks, int nchecks, double tol, int per, int offset, int cap_iterations);

}  // namespace hns

struct hns_ctx {
    hns::Context impl;
};
