// The device-resident force/operator object behind fx_force (exec::InternalForce's role,
// src/exec/internal_force.hpp:80-213): every device buffer of one mesh, the execution plans
// and the work vectors, allocated at creation; applies and solves allocate nothing.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "brick_gp.cuh"
#include "common.cuh"
#include "pimy_element.cuh"

namespace fx {

// equations whose slot sum runs a warp each (k_gather_heavy) instead of a thread
constexpr int32_t kHeavySlots = 64;

// Coefficients of the exact modal element operator of one parameter set on the box grid, for
// the current operator coefficients (box.cu builds them). Scaled by 1/64 where the two
// Walsh-Hadamard transforms (unnormalised) would otherwise multiply the result by 64.
//
// The 24 modal unknowns (component c, mode m) fall into 8 groups by s = m ^ 2^c, and the
// operator couples unknowns of one group only: groups 1..6 hold one coupling (between two
// components), groups 0 and 7 three. So the table is group-major: grp[s][c] is the diagonal of
// (c, s ^ 2^c) (stiffness + mass, consistent or lumped: H^T H = 8 I), grp[s][3] the group's first
// coupling, more[0..1] the second and third couplings of group 0 and more[2..3] those of group 7.
struct BoxCoef {
  double grp[8][4];
  double more[4];
  double body[3];  // force mode: body force per corner (b J), on mode 0
  double pad_;
};
static_assert(sizeof(BoxCoef) == 40 * 8, "BoxCoef layout");

struct BoxCoef32 {  // the same in FP32 for the mixed-precision operator
  float grp[8][4];
  float more[4];
  float body[3];
  float pad_;
};

// The table of a grid whose parameter sets differ only in E (a per-element modulus, the
// heterogeneous cube): the element operator is E_e / E_ref times the stiffness of the reference
// set plus the common mass, so one table serves every element with a per-element scale. grp and
// more as in BoxCoef for the stiffness alone (E_ref), dmm[m] the mass diagonal of mode m (the same
// for the three components).
struct BoxScaled {
  double grp[8][4];
  double more[4];
  double dmm[8];
  double body[3];
  double pad_;
};
static_assert(sizeof(BoxScaled) == 48 * 8, "BoxScaled layout");
struct BoxScaled32 {
  float grp[8][4];
  float more[4];
  float dmm[8];
  float body[3];
  float pad_;
};

// The coefficient tables of a layered grid (one parameter set per element plane, at most
// kTableParams sets and kTableLayers planes), passed to the box kernel as a kernel parameter: the
// set of a plane is then the same for every thread, and its coefficients are read through the
// constant cache instead of the shared-memory pipe that the node values already load.
constexpr int kTableParams = 16, kTableLayers = 1024;
template <class CT>
struct BoxTable {
  CT c[kTableParams];
  uint8_t layer[kTableLayers];  // parameter set of element plane k
};

// A structured grid of axis-aligned boxes with equal spacing: (nx, ny, nz) elements.
struct BoxPlan {
  bool qualifies = false;
  std::string why_not;
  int nx = 0, ny = 0, nz = 0;
  double h[3] = {0, 0, 0};
  // The force (explicit) form runs here when every parameter set has one stiffness-proportional
  // damping factor beta and either the lumped mass or no mass-proportional damping (then
  // f = K (u + beta v) - body + la v, la the lumped alphaM masses, zero without alphaM);
  // otherwise the general path evaluates the force.
  bool force_ok = false;
  double beta = 0.0;
  DeviceArray<double> la;  // [neq] lumped alphaM masses (element and nodal), force form
  DeviceArray<int32_t> node_eq;     // [(nz+1)(ny+1)(nx+1)]: first free equation | free-DOF mask << 29
  DeviceArray<int32_t> elem_param;  // [nz ny nx]: parameter set of each element
  DeviceArray<int32_t> node_of;     // host-side check only: grid node -> internal node
  std::vector<int32_t> grid_node_h; // grid node -> internal node
  // Launch shape per precision (0: FP64, 1: FP32) and kernel mode (0: operator apply, 1: internal
  // force), chosen by the autotuner: variant (block of element columns, CTAs per SM), kz node
  // planes per tile, and the persistent form (one wave of CTAs taking tiles from `queue`) or one
  // CTA per tile.
  struct Shape {
    int variant = 2, kz = 8;
    bool persistent = false;
  } shape[2][2];
  DeviceArray<int> queue;    // [next tile, CTAs done], zero between launches
  bool tuned = false;
  bool layered = false;  // one parameter set per element plane (kernel-parameter tables)
  bool scaled = false;   // the sets differ only in E: one table and a per-element scale
  bool full = false;     // every grid node has all three DOFs free or none
  DeviceArray<double> escale;   // [nz ny nx]: E_e / E_ref
  DeviceArray<float> escale32;
  // The coefficient tables of one use (0: the operator for the last operator coefficients k, 1: the
  // internal force, 2: the mass product M x), each kept until its coefficients change, so that a
  // solve that alternates forces, mass products and operator applies builds them once.
  struct CoefSet {
    DeviceArray<BoxCoef> coef;  // per parameter set (neither layered nor scaled)
    DeviceArray<BoxCoef32> coef32;
    BoxTable<BoxCoef> tab{};    // layered
    BoxTable<BoxCoef32> tab32{};
    DeviceArray<BoxScaled> scoef;  // scaled
    DeviceArray<BoxScaled32> scoef32;
    double k[3] = {0, 0, 0};
    bool built = false;
  } cset[3];
  std::vector<int32_t> node_eq_h;  // node_eq on the host (the host apply's tile ranges)
  // The host-buffer apply in pieces (box_apply_host): x arrives in `chunks` equation ranges on
  // one stream, the tiles that read only arrived equations run as each range lands (tiles sorted
  // by the last equation they read), and after the tiles of range c have run, y leaves up to
  // ready[c], the longest prefix of equations whose owners have all run, on a third stream: the
  // two copy directions overlap each other and the kernel. Built for the FP64 operator's launch
  // shape (variant, kz).
  struct HostPipe {
    int variant = -1, kz = 0, chunks = 0;
    std::vector<int64_t> edge;   // [chunks + 1] equation boundaries of the ranges
    std::vector<int> seg;        // [chunks + 1]: the tiles of range c are tiles[seg[c] .. seg[c+1])
    std::vector<int64_t> ready;  // [chunks]: y[0 .. ready[c]) is final after the tiles of range c
    DeviceArray<int> tiles;     // tile ids (x fastest), by the last equation each reads
    cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
    std::vector<cudaEvent_t> ev_in, ev_comp;
    cudaEvent_t ev_start = nullptr, ev_done = nullptr;
    HostPipe() = default;
    HostPipe(const HostPipe&) = delete;
    HostPipe& operator=(const HostPipe&) = delete;
    ~HostPipe();
  } pipe;
};

// Buffers of the explicit step loop (ground motion, step counter, force, recorded history),
// grown on the first run that needs them.
struct ExplicitWork {
  DeviceArray<double> ag;
  DeviceArray<int> step;
  DeviceArray<double> f64;
  DeviceArray<float> f32;
  DeviceArray<double> hist;
  int32_t record_eq = -1;
  // explicit stages: the half-step velocity (ExplicitDifference) or the previous displacement
  // (CentralDifference) carried between calls, the element velocity, the stage time
  DeviceArray<double> carry, v_elem, time;
  DeviceArray<double> w64;  // w = u + beta v of the next force evaluation (box path)
  DeviceArray<float> w32;
  int carry_scheme = -1;
  // the stage's checks (exec::RunOptions nan_check_interval and stable_step_check_interval, the
  // stage's allow_unstable_dt; 0 turns a periodic check off) and their progress: steps taken in
  // the stage so far (resumed calls continue it), the start's stable step, whether the re-check
  // runs and whether an allowed unstable step was met
  int32_t nan_interval = 100, stable_interval = 100;
  bool allow_unstable = false;
  int64_t stage_step = 0;
  double stage_dt_crit = 0.0;
  bool recheck = false, warned = false;
  DeviceArray<int> bad;  // non-finite count
};

struct ForceState {
  int device = 0;
  int32_t N = 0, neq = 0, count = 0, P = 0, nparams = 0;
  std::vector<ParamGP> params_h;
  std::vector<int32_t> node_h, eq_h, param_h;
  std::vector<double> coords_h, lumped_h, nodal_mass_h, nodal_alpha_h;
  std::vector<int8_t> eq_dof_h;
  DeviceArray<double> coords;
  DeviceArray<int32_t> node, eq, param;
  DeviceArray<ParamGP> params;
  DeviceArray<int32_t> gstart, glist;  // per-equation slot lists in (element, DOF) order
  DeviceArray<int32_t> gheavy;          // the equations with more than kHeavySlots slots (tied DOFs), a warp each
  int32_t nheavy = 0;
  DeviceArray<double> slots;           // [24 * P]
  DeviceArray<float> geom32, nshape32, slots32;  // FP32 operator: point geometry, shape values, slots
  DeviceArray<double> nodal_mass, nodal_alpha_mass, lumped_mass;
  DeviceArray<int8_t> eq_dof;
  bool has_nodal_mass = false, has_nodal_alpha = false;
  int path = FX_PATH_AUTO;  // requested
  BoxPlan box;
  // work vectors (host-buffer apply, solvers)
  DeviceArray<double> wx, wy;
  DeviceArray<double> scratch;  // reduction partials and solver scalars
  int64_t plastic_points = 0;
  // J2 sets (general path): per element and Gauss point, component c of point gp of element e at
  // [(c * 8 + gp) * P + e]: committed state, trial state of the last force evaluation, and that
  // evaluation's compact consistent tangent (elastic until the first force evaluation)
  bool has_j2 = false;
  bool initial = false;  // the operator's stiffness term takes the initial (elastic) matrix
  DeviceArray<double> j2_committed, j2_trial, j2_tan;
  DeviceArray<int> plastic_dev;  // plastic points of the last force evaluation
  // PressureIndependMultiYield sets (general path): the materials bound to parameter sets (table,
  // with their stages), and per Gauss point value k of the state at [(k * 8 + gp) * P + e] (as many
  // values as the largest material holds), value c of the compact tangent likewise
  bool has_pimy = false;
  std::vector<PimySet> pimy_h;
  DeviceArray<PimySet> pimy_dev;
  DeviceArray<double> pimy_committed, pimy_trial, pimy_tan;
  DeviceArray<double> pimy_sig;  // the points' stresses of the last force evaluation, [(c * 8 + gp) * P + e]
  DeviceArray<int> pimy_failed;  // points whose update met a state OpenSees stops for (cumulative)
  int pimy_nstate = 0;
  // PressureDependMultiYield sets, laid out the same way (their trial state is written in full)
  bool has_pdmy = false;
  std::vector<PdmySet> pdmy_h;
  DeviceArray<PdmySet> pdmy_dev;
  DeviceArray<double> pdmy_committed, pdmy_trial, pdmy_tan, pdmy_sig;
  int pdmy_nstate = 0;
  // the soil points' stiffness-proportional damping stresses (sets with betaK or betaKcomm),
  // [(c * 8 + gp) * P + e];
  // unallocated (NULL) when no soil set is damped
  DeviceArray<double> soil_sd;
  // the compacted plastic corrector (compact_soil): per point the strain and strain rate of the
  // predictor, its flag, the list of flagged points, block counts and their total
  bool compact_soil = false;
  DeviceArray<double> soil_eps, soil_rate;
  DeviceArray<int> soil_flag, soil_list, soil_counts, soil_total;
  ExplicitWork xw;
  // SSPbrick sets: per element the geometry record and the stabilization constants,
  // value k of element e at [k * P + e] (ssp_brick.cuh: kGeo, kCon values)
  bool has_ssp = false;
  // the Gauss-point path's form: exact (false: the reference's arithmetic order, bit for bit) or
  // fast (true: eight threads per element, fused multiply-adds; elastic stdBrick sets only)
  bool fast_general = false;
  DeviceArray<double> ssp_geo, ssp_con;
  // stable time step: the minimum's key (general.cu) and, for the periodic re-check, each
  // element's omega^2 with its reference stability tangent (prepare_stability_bounds)
  DeviceArray<unsigned long long> dt_key;
  DeviceArray<double> w2_ref;
  bool bounds_ready = false;
  bool use_box() const { return box.qualifies && path != FX_PATH_GENERAL; }
  bool use_box_force() const { return use_box() && box.force_ok; }
  int64_t device_bytes() const;
};

// general.cu (Gauss-point path, built without fused multiply-adds)
// the Gauss-point operator in FP32 (FP32 geometric factors built at the first call)
void general_apply_f32(ForceState& s, const double k[3], const float* x, float* y, cudaStream_t st,
                       const int* skip = nullptr);
void general_apply(ForceState& s, const double k[3], const double* x, double* y, cudaStream_t st,
                   const int* skip = nullptr);
void general_diagonal(ForceState& s, const double k[3], double* d, cudaStream_t st);
void general_force(ForceState& s, const double* u, const double* v, double* f, cudaStream_t st);
void general_mass_times_ground(ForceState& s, int dir, double* y, cudaStream_t st);
// SSPbrick sets: every element's geometry record and stabilization constants on the device
void ssp_setup(ForceState& s);
// the slot gathers of the operator (with the nodal-mass terms) and of the internal force
void general_gather(ForceState& s, const double k[3], const double* x, double* y, cudaStream_t st, const int* skip);
void general_force_gather(ForceState& s, const double* v, double* f, cudaStream_t st);
// general_fast.cu: the fast form, where it applies (fast_general set, every set elastic stdBrick)
bool general_fast_applies(const ForceState& s);
void general_apply_fast(ForceState& s, const double k[3], const double* x, double* y, cudaStream_t st,
                        const int* skip);
void general_force_fast(ForceState& s, const double* u, const double* v, double* f, cudaStream_t st);
// Stable explicit step on the device (one warp per element, the reference's eigen-solve bit for
// bit): the minimum over the elements of `list` (all elements when NULL, n of them), each
// element's step into dt_out when given (device, n values). scheme 0 CentralDifference, 1
// ExplicitDifference.
double general_min_critical_dt(ForceState& s, int scheme, const int32_t* list, int32_t n, double* dt_out,
                               cudaStream_t st);
// the periodic re-check: whether a set's stable step can change during a stage (the multi-yield
// soils), each element's reference omega^2 (once per stage), and the bound from the points' factors
bool stability_may_change(const ForceState& s);
void prepare_stability_bounds(ForceState& s, cudaStream_t st);
double min_critical_dt_bound(ForceState& s, int scheme, cudaStream_t st);
// commitState of the multi-yield soil points (PressureIndependMultiYield: copy-on-write surfaces;
// PressureDependMultiYield: the whole trial state)
void pimy_commit(ForceState& s, cudaStream_t st);

// stepping.cu: the Newmark form-D kernels (implicit_stage.cpp:29-68)
void newmark_predict(int64_t n, double* u, double* v, double* a, double* ut, double* vt, double* at, double a1,
                     double a2, double a3, double a4, cudaStream_t st);
void newmark_update(int64_t n, const double* du, double* u, double* v, double* a, double c2, double c3,
                    cudaStream_t st);

// box.cu (modal node-owner path)
void box_build_plan(ForceState& s);
void box_apply(ForceState& s, const double k[3], const double* x, double* y, cudaStream_t st,
               const int* skip = nullptr);
void box_apply_f32(ForceState& s, const double k[3], const float* x, float* y, cudaStream_t st,
                   const int* skip = nullptr);
// Build the box coefficient tables for operator coefficients k now (outside any graph capture).
void box_prepare(ForceState& s, const double k[3]);
void box_force(ForceState& s, const double* u, const double* v, double* f, cudaStream_t st);
void box_force_f32(ForceState& s, const float* u, const float* v, float* f, cudaStream_t st);
// y = M x (element masses, consistent or lumped, and nodal masses) on the box path
void box_mass_apply(ForceState& s, const double* x, double* y, cudaStream_t st);
// the box force from w = u + beta v formed by the caller with fma(beta, v, u), as the force kernel
// forms it (the same values), v for the lumped alphaM term: one staged vector instead of two
void box_force_w(ForceState& s, const double* w, const double* v, double* f, cudaStream_t st);
void box_force_w_f32(ForceState& s, const float* w, const float* v, float* f, cudaStream_t st);
int box_num_variants();
void box_set_launch(ForceState& s, int variant, int kz);
void box_autotune(ForceState& s, cudaStream_t st);
// y = K_eff x from and to host buffers on the box path, copies and kernel overlapped in equation
// ranges (BoxPlan::HostPipe) when both buffers are page-locked and the mesh is large enough;
// returns false, having done nothing, otherwise (the caller then copies, applies and copies back)
bool box_apply_host(ForceState& s, const double k[3], const double* xh, double* yh, cudaStream_t st);
// Batches of box grids in one launch: the per-grid descriptor (box_args_bytes bytes, written by
// box_fill_args for y = K_eff x with operator coefficients k, FP64 or FP32 vectors x, y and a
// skip flag), the grid's tile counts, and the launch over a work list of
// (grid, tile x, tile y, tile z) items.
size_t box_args_bytes(bool f32);
void box_fill_args(ForceState& s, const double k[3], bool f32, const void* x, void* y, const int* skip, void* dst);
void box_batch_tiles(const ForceState& s, int& gx, int& gy, int& gz);
// queue: a device int[2], zero between launches, for the persistent form (NULL: one CTA per item)
void box_batch_apply(bool f32, const void* inst, const int4* work, int nwork, int* queue, cudaStream_t st);

}  // namespace fx

struct fx_force {
  fx::ForceState s;
};
