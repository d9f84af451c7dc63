/* femorax_b200: B200-native matrix-free hex8 (stdBrick, 2x2x2 Gauss) hot path behind a C ABI.
 *
 * Plain C types only: pointers, sizes, status codes. Device vectors are FP64 (or FP32 for the
 * *_f32 twins), in the compile step's equation numbering, resident in the memory of the device
 * the handle was created on. Calls on one handle are stream-ordered on the stream the caller
 * passes (cudaStream_t as void*; NULL is the legacy default stream). Nothing here allocates
 * device memory after the create calls, except where a function says so.
 *
 * Each entry point names the reference interface it replaces (amnp95/FemoraX, paths relative to
 * its repository root).
 */
#ifndef FEMORAX_B200_H
#define FEMORAX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes
 * Replace the reference's exceptions (io::ModelError, io::UnsupportedComponent,
 * std::runtime_error from solvers/jacobi.cpp:22) and Kokkos::abort calls
 * (src/exec/internal_force.cpp:359,541,562): no exception crosses this ABI. */
#define FX_OK 0
#define FX_E_INVALID 1     /* bad argument or model (io::ModelError) */
#define FX_E_UNSUPPORTED 2 /* valid but not supported here (io::UnsupportedComponent) */
#define FX_E_NOMEM 3       /* device or host allocation failed */
#define FX_E_NOT_SPD 4     /* CG met p.Ap <= 0 (SolveResult::indefinite) */
#define FX_E_DIVERGED 5    /* non-finite values or no convergence */
#define FX_E_TIMEOUT 6     /* a bounded device wait gave up (reserved: no entry point waits on the device) */
#define FX_E_CUDA 7        /* a CUDA runtime error (message in fx_last_error) */
#define FX_E_UNSTABLE 8    /* an explicit step above the stable step (the stage's io::ModelError) */

/* Message of the last failed call on this host thread. */
const char* fx_last_error(void);
/* Library version string. */
const char* fx_version(void);
/* Free and total bytes of device memory on `device` (cudaMemGetInfo with that device current; the
 * caller's current device is restored): native::cuda_free_memory_bytes
 * (src/native/device_memory_cuda.cpp:7-11), what the serving loop sizes its admissions against. */
int fx_device_memory(int32_t device, int64_t* free_bytes, int64_t* total_bytes);

/* ------------------------------------------------------------------ model description
 * The fields of io::Model the hot path reads (src/io/model.hpp:34-172), as flat arrays.
 * Replaces the HDF5 model file for this path: the host side builds the model in memory. */
typedef struct fx_model fx_model;

/* Material kinds of a parameter set. */
#define FX_MAT_ELASTIC 0 /* ElasticIsotropic (src/physics/materials/elastic_isotropic.hpp) */
#define FX_MAT_J2 1      /* J2 plasticity, linear hardening (no counterpart in the reference) */

/* One material: kind and its constants. J2 uses E, nu, rho, sigma_y, H (hardening modulus) and
 * hk (kinematic share of H, 0 = isotropic, 1 = kinematic). */
/* element types of a group (io::ElementType, src/io/model.hpp:93) */
#define FX_ELEM_STDBRICK 0
#define FX_ELEM_SSPBRICK 1 /* SSPbrick: one point, physical stabilization; elastic material; lumped mass */

typedef struct fx_material {
  int32_t kind;
  int32_t element; /* FX_ELEM_*: the group's element type */
  double E, nu, rho;
  double sigma_y, H, hk;
} fx_material;

/* N nodes: tags and coordinates (row-major, 3 per node); 3 DOFs per node. */
int fx_model_create(int32_t num_nodes, const int32_t* tags, const double* coords, fx_model** out);
void fx_model_destroy(fx_model* m);
/* One stdBrick element group (io::ElementGroup, model.hpp:100-126) with its own material:
 * body force b[3], -lumped flag, element tags, 8 node tags per element in stdBrick order. */
int fx_model_add_group(fx_model* m, const fx_material* mat, const double* b, int32_t lumped, int32_t count,
                       const int32_t* element_tags, const int32_t* connectivity);
/* One SSPbrick element's per-element data as the device path caches it, computed on the host:
 * xl[3][8] its corner coordinates (x of the 8 corners, then y, then z), E and nu its elastic
 * material; geo[33] = dNmod (8 x 3, node-major: the rows of Bnot), the volume and each node's
 * volume weight; con[110] = the hourglass vectors gamma_st, gamma_ut, gamma_us, gamma_stu (8 each,
 * Mben's rows) and the upper triangle of the stabilization's 12 x 12 interior matrix, row by row
 * (SSPbrick::point_store_geometry and element_constants, src/physics/elements/ssp_brick.hpp). */
int fx_ssp_element_constants(const double* xl, double E, double nu, double* geo, double* con);
/* fix rows (node tag, 1-based DOF), model.hpp:134-137. */
int fx_model_add_fix(fx_model* m, int32_t n, const int32_t* node, const int32_t* dof);
/* equalDOF rows (retained, constrained, 1-based DOF), model.hpp:157-162. */
int fx_model_add_equal_dof(fx_model* m, int32_t n, const int32_t* retained, const int32_t* constrained,
                           const int32_t* dof);
/* A Rayleigh region (model.hpp:164-170); the last region naming an element wins. */
int fx_model_add_rayleigh(fx_model* m, double alphaM, double betaK, double betaKinit, double betaKcomm, int32_t n,
                          const int32_t* element_tags);
/* Nodal masses (node tag, 1-based DOF, value), model.hpp:129-132. */
int fx_model_add_mass(fx_model* m, int32_t n, const int32_t* node, const int32_t* dof, const double* value);

/* ------------------------------------------------------------------ compile step
 * compile::compile_model (src/compile/batches.cpp:54-393) for stdBrick groups: RCM node order
 * (src/compile/renumber.cpp:98-183), element order, DOF numbering with equalDOF groups and
 * fixes (src/compile/dof_numbering.cpp:269-485), one batch padded to simd_width, parameter
 * sets per (group, Rayleigh region), lumped masses, optional greedy coloring (:23-50). The
 * arrays are bit-identical to the reference's. */
typedef struct fx_compiled fx_compiled;
#define FX_RENUMBER_OFF 0
#define FX_RENUMBER_RCM 1
int fx_compile(const fx_model* m, int32_t renumbering, int32_t simd_width, int32_t coloring, fx_compiled** out);
void fx_compiled_destroy(fx_compiled* c);
/* sizes[8] = num_nodes, num_equations, num_slots, num_batches, count, padded, num_params,
 * num_colors (batch 0). */
int fx_compiled_sizes(const fx_compiled* c, int64_t* sizes);
/* Named arrays, as the reference's Compiled holds them (batches.hpp:80-116); returns the
 * length, or -1 for an unknown name; out may be NULL to ask the length. int32 names:
 * node_tag, node_order, element_order, eq, dof_offset, node_model_index, b_node, b_eq,
 * b_param, b_tag, color_start, color_elements, eq_dof. double names: coords, lumped_mass,
 * lumped_alpha_mass, nodal_mass, nodal_alpha_mass. */
int64_t fx_compiled_array_i32(const fx_compiled* c, const char* name, int32_t* out);
int64_t fx_compiled_array_f64(const fx_compiled* c, const char* name, double* out);

/* ------------------------------------------------------------------ mesh arrays
 * What the device path consumes: the compile step's arrays as plain host pointers
 * (compile::Compiled, batches.hpp:80-116, one stdBrick batch), from fx_compile or from the
 * reference's own compile_model. */
typedef struct fx_param_set {
  int32_t kind;      /* FX_MAT_* */
  int32_t mass_type; /* 0 consistent, 1 lumped (StdBrick::Params::massType) */
  double E, nu, rho;
  double b[3];                                /* body force per unit volume */
  double alphaM, betaK, betaKinit, betaKcomm; /* Rayleigh (physics/contracts.hpp:69-75) */
  double sigma_y, H, hk;                      /* J2 only */
  int32_t element;                            /* FX_ELEM_* */
  int32_t pad_;
} fx_param_set;

typedef struct fx_mesh {
  int32_t num_nodes, num_equations;
  const double* coords; /* [3 * num_nodes] structure of arrays x[N] y[N] z[N] */
  int32_t count, padded;
  const int32_t* node;  /* [8 * padded]: internal node of corner a of element e at a*padded+e */
  const int32_t* eq;    /* [24 * padded]: equation of local DOF k at k*padded+e, -1 fixed */
  const int32_t* param; /* [padded] */
  int32_t num_params;
  int32_t pad_;
  const fx_param_set* params;      /* [num_params] */
  const double* lumped_mass;       /* [num_equations] or NULL */
  const double* nodal_mass;        /* [num_equations] or NULL */
  const double* nodal_alpha_mass;  /* [num_equations] or NULL */
  const int8_t* eq_dof;            /* [num_equations] or NULL: the nodal DOF of each equation */
} fx_mesh;

/* Fills *mesh with pointers into c (valid while c lives); params[] must hold num_params. */
int fx_compiled_mesh(const fx_compiled* c, fx_param_set* params, fx_mesh* mesh);

/* ------------------------------------------------------------------ internal force / operator
 * exec::InternalForce (src/exec/internal_force.hpp:80-213): owns every device buffer of one
 * mesh (maps, parameters, state, plans, work vectors); compute/apply allocate nothing. */
typedef struct fx_force fx_force;

/* Execution paths (set by fx_force_set_path; default FX_PATH_AUTO).
 *   FX_PATH_GENERAL     Gauss-point element kernel in the reference's arithmetic order, element
 *                       values into slots, per-equation slot gather in (element, DOF) order:
 *                       any hexahedra.
 *   FX_PATH_BOX         node-owner kernel over structured grids of axis-aligned boxes, exact
 *                       modal (Walsh-Hadamard) form of the 2x2x2-Gauss element operator.
 *   FX_PATH_AUTO        BOX when the mesh qualifies, else GENERAL. */
#define FX_PATH_AUTO 0
#define FX_PATH_GENERAL 1
#define FX_PATH_BOX 2

int fx_force_create(const fx_mesh* mesh, int32_t device, fx_force** out);
void fx_force_destroy(fx_force* f);
int fx_force_set_path(fx_force* f, int32_t path);
/* The Gauss-point path's form (meshes off the box path): FX_GENERAL_EXACT (default) evaluates every
 * element in the reference's arithmetic order, bit for bit its results; FX_GENERAL_FAST evaluates
 * elastic stdBrick elements with eight threads each (one per Gauss point) and fused multiply-adds,
 * within 1e-12 of the largest entry of the exact form, for the operator and the internal force.
 * Meshes with J2, multi-yield soil or SSPbrick sets keep the exact form. */
/* The multi-yield soil points' update: FX_SOIL_FUSED (default) updates every point in one pass;
 * FX_SOIL_COMPACTED runs the compacted plastic corrector (src/exec/compacted_kernels.hpp): a
 * predictor pass that finishes the points that stay elastic and flags the others, a compaction
 * that lists the flagged points in order, and the corrector on the listed points only. Both give
 * every point the same bits. */
#define FX_SOIL_FUSED 0
#define FX_SOIL_COMPACTED 1
int fx_force_set_soil_corrector(fx_force* f, int32_t mode);
#define FX_GENERAL_EXACT 0
#define FX_GENERAL_FAST 1
int fx_force_set_general_mode(fx_force* f, int32_t mode);
/* info[9] = num_equations, num_elements, path of the operator, box qualifies (0/1), grid nx, ny,
 * nz, device bytes held, force form on the box path (0/1: lumped masses and one beta). */
int fx_force_info(const fx_force* f, int64_t* info);
/* Box path launch shape: variant (block of element columns, CTAs per SM) and kz (node planes
 * per CTA); fx_force_tune times the candidates on the device, for the FP64 and the FP32 operator
 * and internal force separately, and keeps the fastest of each (the autotuner fx_force_create
 * runs on meshes of 262,144 elements or more; exec::choose_force_settings' role,
 * src/exec/force_settings.cpp:71-205). fx_force_set_launch pins every precision and kernel to
 * one shape; launch[2] of fx_force_get_launch receives the FP64 operator's shape (variant, kz).
 * A negative kz selects (or reports) the persistent form of that shape: one wave of CTAs taking
 * tiles of |kz| planes from a queue. The environment variable FEMORAX_B200_BOX_LAUNCH="variant,kz"
 * makes fx_force_create pin that shape instead of timing the candidates (the role of the
 * reference's FEMORAX_FORCE_SETTINGS, src/exec/force_settings.cpp:186-190). */
int fx_force_set_launch(fx_force* f, int32_t variant, int32_t kz);
int fx_force_get_launch(const fx_force* f, int32_t* launch);
/* Every tuned shape: launch[8] = (variant, kz) of the FP64 operator, FP64 internal force, FP32
 * operator, FP32 internal force (no counterpart in the reference). */
int fx_force_get_launches(const fx_force* f, int32_t* launch);
int fx_force_tune(fx_force* f, void* stream);

/* Operator coefficients K_eff = stiffness K_t + damping C + mass M (OperatorCoefficients,
 * src/physics/operators/element_operator.hpp:33-40). */
typedef struct fx_coeffs {
  double stiffness, damping, mass;
  int32_t initial; /* K_0 in the stiffness term (ModifiedNewton -initial) */
  int32_t pad_;
} fx_coeffs;

/* y = K_eff x (InternalForce::apply_operator, internal_force.cpp:545-573; x, y device FP64,
 * never aliasing). */
int fx_apply_operator(fx_force* f, fx_coeffs k, const double* x, double* y, void* stream);
/* FP32 twin: x, y device FP32, parameters rounded to FP32 (the mixed-precision inner operator):
 * on box grids the box kernel in FP32; on other meshes (J2 sets included, with their stored
 * point tangents) the Gauss-point operator in FP32 with FP32 geometric factors of the points,
 * computed once in FP64 and rounded. */
int fx_apply_operator_f32(fx_force* f, fx_coeffs k, const float* x, float* y, void* stream);
/* The same apply from HOST vectors (pinned or pageable): copies in, applies, copies out. */
int fx_apply_operator_host(fx_force* f, fx_coeffs k, const double* x_host, double* y_host, void* stream);
/* d = diag(K_eff) (InternalForce::operator_diagonal, internal_force.cpp:575-599). */
int fx_operator_diagonal(fx_force* f, fx_coeffs k, double* d, void* stream);
/* The same diagonal into a HOST vector (Jacobi::setup of a solver whose vectors live on the host,
 * jacobi.cpp:10-26): computed on the device, copied out; returns after the copy. */
int fx_operator_diagonal_host(fx_force* f, fx_coeffs k, double* d_host, void* stream);
/* f = f_int(u) + Rayleigh damping forces at v + nodal alphaM M v (InternalForce::compute,
 * internal_force.cpp:354-377). u, v, f device FP64. */
int fx_force_compute(fx_force* f, const double* u, const double* v, double* out, void* stream);
int fx_force_compute_f32(fx_force* f, const float* u, const float* v, float* out, void* stream);
/* y = M r_dir, the UniformExcitation load shape (InternalForce::mass_times_ground,
 * internal_force.cpp:601-626). */
int fx_mass_times_ground(fx_force* f, int32_t dir, double* y, void* stream);
/* Smallest stable step of the elements (InternalForce::min_critical_dt,
 * internal_force.hpp:201): scheme 0 CentralDifference, 1 ExplicitDifference. Host result. Each
 * element's largest omega^2 with the lumped mass and the material's stability tangent (the elastic
 * moduli at the committed state for the multi-yield soils, contracts.hpp:355-365) by the
 * reference's cyclic Jacobi rotations (sym_eigen.hpp), one warp per element on the device, bit for
 * bit the reference's; on box grids of elastic or J2 sets one element per parameter set. */
int fx_min_critical_dt(fx_force* f, int32_t scheme, double* dt);
/* Every element's stable step into dt_dev[count] (device, batch order):
 * InternalForce::element_critical_dts (internal_force.hpp:202-204). */
int fx_element_critical_dts(fx_force* f, int32_t scheme, double* dt_dev, void* stream);
/* The periodic stable-step re-check (InternalForce::stability_may_change, prepare_stability_bounds,
 * min_critical_dt_bound; internal_force.hpp:205-210): whether a set's stable step can change in a
 * stage (the multi-yield soils), each element's omega^2 with the reference tangent (once per stage),
 * and the smallest step from the bound: the soil points' largest stability factor times that
 * omega^2, never above the exact omega^2 (so the bound never overstates the step). */
int fx_stability_may_change(const fx_force* f, int32_t* out);
int fx_stability_prepare(fx_force* f, void* stream);
int fx_min_critical_dt_bound(fx_force* f, int32_t scheme, double* dt, void* stream);
/* Material state: commit the trial state (InternalForce::commit_state, internal_force.cpp:507). */
int fx_force_commit(fx_force* f, void* stream);
/* Number of Gauss points that were plastic at the last force evaluation (J2). */
int fx_force_plastic_points(fx_force* f, int64_t* count);
/* The J2 material state of the Gauss points (the state InternalForce keeps per point and swaps
 * in commit_state, internal_force.cpp:507-509; for checkpoints and tests). which = 0 committed
 * and 1 trial state (13 components per point: plastic strain with engineering shear [6],
 * equivalent plastic strain, back stress [6]), 2 the compact consistent tangent of the last force
 * evaluation (8: theta, thetab, n[6]); component c of point gp of element e at
 * [(c * 8 + gp) * padded + e]. `count` is the host buffer's length in doubles (get: at least the
 * array's; set: exactly it; set takes which 0 or 1). FX_E_UNSUPPORTED without J2 sets. */
int fx_force_state(fx_force* f, int32_t which, double* host, int64_t count);
int fx_force_set_state(fx_force* f, int32_t which, const double* host, int64_t count);

/* ------------------------------------------------------------------ vector kernels
 * solvers::VectorOps (src/solvers/vector_ops.hpp:17-57): deterministic reductions in the
 * documented order (chunks of 2048 entries; lane l of `lanes` sums entries l, l+lanes, ... of a
 * chunk; the lane sums are added in lane order; levels of chunk sums until one value is left).
 * lanes = 32 is the order of the reference's CUDA build, lanes = 1 that of its host build.
 * Products are fused multiply-adds. Like VectorOps(n, lanes), the handle owns the partial sums
 * for vectors of up to `capacity` entries, allocated at creation. */
typedef struct fx_vops fx_vops;
int fx_vops_create(int64_t capacity, int32_t lanes, int32_t device, fx_vops** out);
void fx_vops_destroy(fx_vops* v);
/* x.y of n entries (VectorOps::dot, vector_ops.cpp:54-73): written to *result_dev (device) when
 * given, and to *result_host (after a stream synchronisation) when given. */
int fx_vops_dot(fx_vops* v, const double* x, const double* y, int64_t n, double* result_dev, double* result_host,
                void* stream);
/* x.y of n entries on the current device (x and y must be that device's memory, or managed
 * memory; others are rejected with FX_E_INVALID, and `stream` must belong to that device), in the
 * same order and with the same bits as
 * fx_vops_dot with the same lanes, but allocating nothing: no cudaMalloc, no cudaFree and no
 * allocating library routine. It has no counterpart in the reference. It is for callers that
 * must not allocate device memory: an application that hands all of the GPU's memory to its own
 * pool at start-up and forbids other allocations, or a latency-bound loop that cannot afford
 * cudaMalloc's implicit device synchronisation. The partial sums live in one fixed device array
 * of this library, so n is limited to 2^27 (134,217,728) entries; larger n is rejected with
 * FX_E_INVALID. The first call on a device looks up that array's address there (once per
 * device), so make the first call on each device before any stream capture. Every call in the
 * process shares the array and it keeps the last call's partials (each call writes every partial
 * it reads, so none has to start at zero); calls whose kernels overlap on the GPU, from two
 * streams or two host threads, race on it and must be ordered by the caller. The result goes to
 * *result_dev (device) and/or *result_host (after a stream synchronisation); at least one must be
 * given. lanes is 1..32 as in fx_vops_create. */
int fx_dot_noalloc(const double* x, const double* y, int64_t n, int32_t lanes, double* result_dev,
                   double* result_host, void* stream);
/* Element-wise kernels (vector_ops.cpp:77-103): y += a x; y = x + a y; y = d .* x. */
int fx_axpy(double a, const double* x, double* y, int64_t n, void* stream);
int fx_xpay(const double* x, double a, double* y, int64_t n, void* stream);
int fx_multiply(const double* d, const double* x, double* y, int64_t n, void* stream);

/* ------------------------------------------------------------------ solvers
 * solvers::SolveOptions / SolveResult (src/solvers/linear_solver.hpp:79-94). */
typedef struct fx_solve_opts {
  double rtol, atol;
  int32_t max_iterations;
  int32_t lanes;   /* dot order; 32 = the reference's CUDA order */
  int32_t restart; /* GMRES */
  int32_t pad_;
} fx_solve_opts;
typedef struct fx_solve_result {
  int32_t converged, iterations;
  double rhs_norm, initial_residual, final_residual;
  int32_t indefinite, status;
  int32_t refinements; /* fx_ir_solve: outer FP64 corrections */
  int32_t pad_;
} fx_solve_result;

/* A linear solver on the matrix-free operator K_eff of one fx_force (solvers::LinearSolver,
 * src/solvers/linear_solver.hpp:96-105, with the Jacobi preconditioner of jacobi.cpp:10-26).
 * fx_solver_create allocates the work vectors (LinearSolver::setup's allocation);
 * fx_solver_setup takes the operator coefficients and builds the Jacobi diagonal (call it when
 * the coefficients change); fx_solver_solve solves K_eff x = b with x holding the initial guess.
 * Methods:
 *   FX_SOLVER_CG      Jacobi-PCG (ConjugateGradient::solve, src/solvers/cg.cpp:24-71),
 *                     device-resident: scalars stay on the device, the iterations run as one
 *                     CUDA graph that loops on the device until the solve is done (kept for the
 *                     next solve on the same vectors); the host reads the result once.
 *   FX_SOLVER_GMRES   FGMRES(restart) with CGS2 (Gmres::solve, src/solvers/gmres.cpp:32-123).
 *   FX_SOLVER_KRYLOV  CG, then GMRES from the initial guess if CG meets p.Ap <= 0
 *                     (KrylovSolver::solve, src/solvers/krylov.cpp:25-41).
 *   FX_SOLVER_IR      CG in FP32 (FP32 operator and vectors) inside FP64 iterative refinement:
 *                     r = b - K x in FP64, K d = r by FP32 PCG to inner_rtol, x += d in FP64,
 *                     until ||b - K x|| <= rtol ||b|| in FP64 (converged), or until a round
 *                     leaves ||b - K x|| above half the previous round's (the FP64 residual's
 *                     floor for this operator: not converged, x kept), or 50 rounds. The FP32
 *                     operator is fx_apply_operator_f32's (box kernel, or the FP32 Gauss-point
 *                     form). */
#define FX_SOLVER_CG 0
#define FX_SOLVER_GMRES 1
#define FX_SOLVER_KRYLOV 2
#define FX_SOLVER_IR 3
typedef struct fx_solver fx_solver;
int fx_solver_create(fx_force* f, int32_t method, fx_solve_opts o, fx_solver** out);
void fx_solver_destroy(fx_solver* s);
int fx_solver_setup(fx_solver* s, fx_coeffs k, void* stream);
/* FX_SOLVER_IR: the relative tolerance of each inner FP32 solve (default 1e-4). */
int fx_solver_set_inner_tolerance(fx_solver* s, double inner_rtol);
int fx_solver_solve(fx_solver* s, const double* b, double* x, fx_solve_result* r, void* stream);
/* Newton iterations of one quasi-static load step (ImplicitStage's Newton loop without inertia,
 * src/exec/implicit_stage.cpp:118-437): r = f_ext - f_int(u) with every point's material update
 * (J2: the return map, which also stores the points' consistent tangents), the Jacobi diagonal
 * of that tangent, K_t du = r by this CG solver from du = 0, u += du; until the stage's test
 * (implicit_stage.cpp:199, 241-242, 342) holds, absolute: FX_TEST_NORM_UNBALANCE ||r|| <= tol,
 * FX_TEST_NORM_DISP_INCR ||du|| <= tol (then the force is evaluated once more at the final u);
 * or max_newton solves. u (device) holds the start and receives the result; the trial material
 * state is u's, left for fx_force_commit. r: converged, iterations (CG iterations in all),
 * rhs_norm = ||f_ext||, initial/final_residual = ||r|| at the first and last evaluation.
 * FX_SOLVER_CG, or FX_SOLVER_IR (FP32 CG on the tangent inside FP64 refinement: the FP32
 * operator uses the points' stored tangents, the return map stays FP64); set up with the
 * stiffness coefficient 1. */
#define FX_TEST_NORM_UNBALANCE 0
#define FX_TEST_NORM_DISP_INCR 1
int fx_solver_newton(fx_solver* s, const double* fext, double* u, int32_t test, double tol, int32_t max_newton,
                     int32_t* newton_iterations, fx_solve_result* r, void* stream);
/* One Newmark time step of size dt (Newmark::newStep with displ == 1 and ImplicitStage's Newton
 * loop with inertia, src/exec/implicit_stage.cpp:29-68, 118-437): predict v and a from the last
 * step (u kept), then Newton iterations r = f_ext - f_int(u, v) - M a, K_eff du = r by this
 * solver (FX_SOLVER_CG: plain FP64; FX_SOLVER_IR: FP32 CG inside FP64 refinement), u += du,
 * v += c2 du, a += c3 du, with the test of fx_solver_newton. The solver must be set up with the
 * coefficients (1, c2 = gamma/(beta dt), c3 = 1/(beta dt^2)). u, v, a (device) hold the last
 * step's state and receive the new one; the trial material state is left for fx_force_commit. */
int fx_solver_newmark(fx_solver* s, const double* fext, double* u, double* v, double* a, double dt, double beta,
                      double gamma, int32_t test, double tol, int32_t max_newton, int32_t* newton_iterations,
                      fx_solve_result* r, void* stream);
/* Femora's retry and substep recovery around one Newmark step (ImplicitStage,
 * implicit_stage.cpp:261-402): an attempt whose Newton iterations do not converge goes back to the
 * committed u, v, a and is retried at the same size up to max_retries times; then, below
 * num_sublevels levels, the step is split into num_substeps steps one level down, each with the
 * same recovery. Every converged attempt commits the material state (Domain::commit); the caller
 * need not commit again. The load of an attempt that ends at the fraction theta of the step is
 * fext0 + theta (fext1 - fext0) (device vectors; fext0 NULL: fext1 throughout). The solver is set
 * up for each attempt's size (1, gamma/(beta h_s), 1/(beta h_s^2)) and back to dt's at the end.
 * stats[5] = attempts, failed attempts, retries, substeppings, Newton iterations. Returns FX_OK
 * with r->status FX_E_DIVERGED when every attempt failed (the state is then the committed one). */
int fx_solver_newmark_recover(fx_solver* h, const double* fext0, const double* fext1, double* u, double* v, double* a,
                              double dt, double beta, double gamma, int32_t test, double tol, int32_t max_newton,
                              int32_t max_retries, int32_t num_sublevels, int32_t num_substeps, int32_t* stats,
                              fx_solve_result* r, void* stream);
/* The same for a quasi-static load step (fx_solver_newton): retries only, as the reference's static
 * stages; a converged step commits the material state. stats as above (no substeppings). */
int fx_solver_newton_recover(fx_solver* h, const double* fext, double* u, int32_t test, double tol, int32_t max_newton,
                             int32_t max_retries, int32_t* stats, fx_solve_result* r, void* stream);

/* ------------------------------------------------------------------ time stepping
 * ExplicitDifference steps (src/exec/explicit_analysis.cpp:62-84, 687-705): per step
 * predict (vh += dt a; u += dt vh), force at (u, vh), correct (a = (-f - m ag)/m,
 * v = vh + dt/8 (3a + a_old)). ag(t) of the UniformExcitation in direction dir is given per
 * step in ag_host[steps] (NULL: none). State vectors u, vh, a, v device FP64 (FP32 for _f32). */
int fx_explicit_run(fx_force* f, const double* mass, int32_t dir, const double* ag_host, int32_t steps, double dt,
                    double* u, double* vh, double* a, double* v, void* stream);
int fx_explicit_run_f32(fx_force* f, const float* mass, int32_t dir, const double* ag_host, int32_t steps, double dt,
                        float* u, float* vh, float* a, float* v, void* stream);
/* Acceleration history of one equation. With hist_dev NULL: record equation eq (-1: none) in the
 * following fx_explicit_run calls. Otherwise copy the last run's first `count` recorded values
 * (hist_dev[step] = a[eq] after step `step`) to hist_dev (device, at least `count` doubles). */
int fx_explicit_record(fx_force* f, int32_t eq, double* hist_dev, int32_t count);

/* Ground motions on the device (exec::GroundMotions, src/exec/ground_motion.hpp:22-70,
 * ground_motion.cpp:64-175): UniformExcitation patterns, each with its own Path series.
 * fx_motions_add: pattern acting in DOF dof (0-based) with factor fact; the series has n values
 * and either a uniform spacing dt (times NULL; OpenSees PathSeries, prepend_zero puts a zero
 * first, use_last holds the last value after the end) or times[n] (PathTimeSeries); factor is
 * the series' cFactor. fx_motions_evaluate: accel_host[p] = fact_p * series_p(t) for every
 * pattern, evaluated on the device (a time series keeps its interval between calls, as the
 * reference's does). */
typedef struct fx_motions fx_motions;
int fx_motions_create(fx_motions** out);
int fx_motions_destroy(fx_motions* m);
int fx_motions_add(fx_motions* m, int32_t dof, double fact, const double* values, const double* times, int32_t n,
                   double dt, double factor, int32_t use_last, int32_t prepend_zero);
int fx_motions_evaluate(fx_motions* m, double t, double* accel_host);

/* An explicit analysis stage (src/exec/explicit_analysis.cpp:665-725; no local time stepping,
 * exact constraints, DRM or recorders): `steps` steps of dt from *time with scheme 1
 * ExplicitDifference (ed_predict / ed_correct, :62-84) or 0 CentralDifference
 * (cd_garbage_velocity / cd_solve, :86-117, alpha_mass = Compiled::lumped_alpha_mass), the
 * ground accelerations of `motions` (NULL: none) evaluated on the device at each step's load
 * time, the material state committed after every step. u, v, a (device FP64) hold the
 * committed displacement, velocity and acceleration and receive the stage's end state; *time
 * (host) receives the end time. resume = 0 starts a stage (ED: half-step velocity = v; CD:
 * previous displacement = u); resume = 1 continues the previous call of the same scheme, so that
 * a stage run in pieces equals one call. fx_explicit_record's equation is recorded (the
 * acceleration after each step). The stage's checks (explicit_analysis.cpp:582-653, 732-771): a
 * starting call compares dt with the stable step (FX_E_UNSTABLE above it, unless allowed);
 * every stable_step_check_interval steps of the stage (sets whose stable step can change) the
 * bound, then the exact step where the bound falls below dt, stops the stage with FX_E_UNSTABLE;
 * every nan_check_interval steps, and at the end of every call, non-finite displacements stop
 * it with FX_E_DIVERGED (the state then is that of the failing step). */
int fx_explicit_stage(fx_force* f, int32_t scheme, const double* mass, const double* alpha_mass, fx_motions* motions,
                      int32_t steps, double dt, double* time, double* u, double* v, double* a, int32_t resume,
                      void* stream);
/* The checks of later fx_explicit_stage calls on this force: exec::RunOptions nan_check_interval
 * and stable_step_check_interval (0 turns that periodic check off; defaults 100 and 100) and the
 * stage's allow_unstable_dt (default 0: an unstable step stops the stage). */
int fx_explicit_checks(fx_force* f, int32_t nan_check_interval, int32_t stable_step_check_interval,
                       int32_t allow_unstable_dt);

/* Newmark form D kernels (src/exec/implicit_stage.cpp:29-68). */
int fx_newmark_predict(int64_t n, double* u, double* v, double* a, double* ut, double* vt, double* at, double a1,
                       double a2, double a3, double a4, void* stream);
int fx_newmark_update(int64_t n, const double* du, double* u, double* v, double* a, double c2, double c3,
                      void* stream);

/* ------------------------------------------------------------------ batched Newton
 * Quasi-static load steps of many independent meshes at once (the batched J2 configuration): the
 * instances are concatenated into one mesh (instance s's equations at [offset_s, offset_s + n_s),
 * offsets multiples of 2048, the gaps unused), whose element kernels and gather run every
 * instance in one launch each, while each instance keeps its own Newton test and its own
 * Jacobi-PCG recurrence on the device (per-instance scalars and stopping flags, CG iterations as
 * CUDA graphs). Per instance the iterates and material states are bit for bit those of
 * fx_solver_newton with FX_TEST_NORM_UNBALANCE on that mesh alone. No counterpart in the
 * reference (one mesh per process; per instance its ImplicitStage Newton loop,
 * src/exec/implicit_stage.cpp:118-437, with ConjugateGradient, cg.cpp:24-71).
 *   fx_nbatch_create   the instances' mesh arrays (as fx_compiled_mesh gives them), CG options
 *   fx_nbatch_layout   offsets[count + 1] (offsets[count] = combined length) and the instances'
 *                      equation counts (may be NULL)
 *   fx_nbatch_step     one load step of every instance: f_ext and u (device, combined layout; u
 *                      holds the start and receives the result), NormUnbalance ||r|| <= tol,
 *                      at most max_newton solves; per instance the Newton solves and a result
 *                      (converged, CG iterations in all, final ||r||)
 *   fx_nbatch_force    the combined fx_force (owned by the batch): fx_force_commit commits every
 *                      instance's material state, fx_force_state reads it */
typedef struct fx_nbatch fx_nbatch;
int fx_nbatch_create(const fx_mesh* meshes, int32_t count, int32_t device, fx_solve_opts o, fx_nbatch** out);
/* The linear solves of the Newton iterations: FX_SOLVER_CG (plain FP64 Jacobi-PCG, the default)
 * or FX_SOLVER_IR (per instance FP32 Jacobi-PCG to inner_rtol inside FP64 refinement to the
 * options' tolerance, as fx_solver_newton with an FX_SOLVER_IR solver: FP32 operator on the
 * stored point tangents, FP64 return map and residuals; per instance the same bits). */
int fx_nbatch_set_inner(fx_nbatch* b, int32_t method, double inner_rtol);
void fx_nbatch_destroy(fx_nbatch* b);
int fx_nbatch_layout(const fx_nbatch* b, int64_t* offsets, int64_t* equations);
fx_force* fx_nbatch_force(fx_nbatch* b);
int fx_nbatch_step(fx_nbatch* b, const double* fext, double* u, double tol, int32_t max_newton,
                   int32_t* newton_iterations, fx_solve_result* results, void* stream);

/* ------------------------------------------------------------------ elementary functions
 * The exp, log, pow and cos of the PressureDependMultiYield device update (fx_math.h: built from
 * IEEE-exact operations, so a host and a device evaluation give the same bits; within 0.51 ulp and
 * one ulp of the host C library's). fx_math_eval runs them on device arrays (x, y, out on the
 * current device; y only for pow) on `stream`; fx_math_eval_host on host arrays. For checking the
 * device update against the reference's material linked to the same functions. No counterpart in
 * the reference, which calls its host C library (src/physics/materials/pressure_depend_multi_yield.hpp). */
#define FX_MATH_EXP 0
#define FX_MATH_LOG 1
#define FX_MATH_POW 2
#define FX_MATH_COS 3
int fx_math_eval(int32_t fn, const double* x, const double* y, double* out, int64_t n, void* stream);
int fx_math_eval_host(int32_t fn, const double* x, const double* y, double* out, int64_t n);

/* ------------------------------------------------------------------ batched and served solves
 * An engine holds many independent meshes ("slots", each one fx_force on the box path, a
 * structured grid of equal boxes) resident on one device and solves K_eff x = b for all of them
 * together by FP32 Jacobi-PCG inside FP64 iterative refinement, per slot exactly as
 * FX_SOLVER_IR (the same bits): one launch per operator apply over the element tiles of every
 * running slot, per-slot CG scalars and stopping on the device, inner iterations as CUDA graphs.
 * No counterpart in the reference, which solves one mesh per process
 * (ConjugateGradient::solve, src/solvers/cg.cpp:24-71, is the per-slot algorithm).
 *   fx_engine_create   vectors for `capacity` equations in all (rounded to 2048-entry chunks,
 *                      each slot a whole number of chunks) and `max_slots` slots; operator
 *                      coefficients k; rtol / atol / max_iterations / lanes as fx_solve_opts;
 *                      inner_rtol the inner FP32 solve's relative tolerance.
 *   fx_engine_admit    takes a mesh (the engine uses f until the slot is retired) and its
 *                      right-hand side (host, num_equations doubles) into a free slot: copies
 *                      b, builds the Jacobi diagonal, x = 0. FX_E_NOMEM when no slot or no
 *                      contiguous range of chunks is free (admit again after a retire).
 *   fx_engine_round    one tick: the slots whose inner solve has ended get their FP64
 *                      correction, those due get their outer step (FP64 residual and test, the
 *                      inner solve's start), then every running inner solve 8 iterations; each
 *                      slot in its own phase (no slot waits for another's inner solve);
 *                      *running = the unfinished slots it advanced.
 *   fx_engine_finished whether a slot's solve has ended (converged or given up).
 *   fx_engine_retire   copies x (host, may be NULL) and the result out and frees the slot.
 *   fx_engine_info     info[6] = capacity (equations), equations in use, max slots, slots in
 *                      use, rounds run, device bytes of the engine's vectors.
 *   fx_engine_set_precision  the inner solves' precision while no slot is in use:
 *                      FX_ENGINE_INNER_FP32 (the default, above) or FX_ENGINE_INNER_FP64 (FP64
 *                      Jacobi-PCG with the FP64 operator inside the same refinement rounds: the
 *                      batched engine without reduced precision, with inner_rtol at or below the
 *                      outer rtol a slot converges in its first round). */
#define FX_ENGINE_INNER_FP32 0
#define FX_ENGINE_INNER_FP64 1
typedef struct fx_engine fx_engine;
int fx_engine_create(int32_t device, int64_t capacity, int32_t max_slots, fx_coeffs k, fx_solve_opts o,
                     double inner_rtol, fx_engine** out);
void fx_engine_destroy(fx_engine* e);
int fx_engine_set_precision(fx_engine* e, int32_t inner);
/* The batched apply as one CTA per (slot, tile) work item (on = 0, the default) or as a persistent
 * wave of CTAs taking the items from a counter (on = 1); the same bits either way. */
int fx_engine_set_persistent(fx_engine* e, int32_t on);
int fx_engine_admit(fx_engine* e, fx_force* f, const double* b_host, int32_t* slot);
int fx_engine_round(fx_engine* e, int32_t* running);
int fx_engine_finished(fx_engine* e, int32_t slot, int32_t* finished);
int fx_engine_retire(fx_engine* e, int32_t slot, double* x_host, fx_solve_result* r);
int fx_engine_info(const fx_engine* e, int64_t* info);

/* ------------------------------------------------------------------ the serving loop
 * Requests arriving over time, served on one device with continuous batching (serve.cu): static
 * solves K x = b on resident fx_force meshes (several requests may share one) through an engine
 * (fx_engine_*), and quasi-static J2 load paths on compiled meshes in cohorts (fx_nbatch_*) beside
 * the engine. Prepared requests are added with their arrival time (seconds from the start);
 * fx_server_run serves them once: in arrival order (in real time, or all visible at once), static
 * solves admitted while the footprint of the admitted requests (mesh device bytes; a J2 instance's
 * estimate) fits hbm_budget and the engine has room; one engine tick per pass of the calling
 * thread's loop, each J2 cohort stepped through its path by a thread of its own on its own stream
 * (the cohorts' work overlaps the engine's on the device).
 *   fx_server_add_j2   mesh (fx_compiled_mesh; its arrays must live until the run ends), the load at
 *                      factor 1 (host, num_equations), the monitored equation, the load path (cycles
 *                      of steps_per_cycle steps, 0 -> 1 -> -1 -> 0), Newton ||r|| <= tol in at most
 *                      max_newton solves, CG (Jacobi) to cg_rtol in at most cg_max_iterations;
 *                      requests with the same path and settings share a cohort (up to max_cohort);
 *                      up to max_lanes cohorts run at once (a thread each), so J2 requests
 *                      arriving while a cohort runs start the next one.
 *   fx_server_result   x (num_equations), the result, times[3] = arrival, admitted, done (seconds
 *                      from the start of the run, steady clock); J2: the monitored displacement and
 *                      the Newton solves after each step (cycles * steps_per_cycle each).
 * A result is bit for bit the request's alone (the engine's solve of its mesh; the batched Newton
 * path of its mesh). No counterpart in the reference, which runs one analysis per process. */
typedef struct fx_server fx_server;
int fx_server_create(fx_engine* engine, int32_t device, int64_t hbm_budget, int32_t max_cohort, int32_t max_lanes,
                     fx_server** out);
void fx_server_destroy(fx_server* s);
int fx_server_add_static(fx_server* s, int64_t id, fx_force* f, const double* b_host, double arrival);
int fx_server_add_j2(fx_server* s, int64_t id, const fx_mesh* mesh, const double* unit_load, int64_t monitor,
                     int32_t cycles, int32_t steps_per_cycle, double tol, int32_t max_newton, double cg_rtol,
                     int32_t cg_max_iterations, double arrival);
int fx_server_run(fx_server* s, int32_t realtime, double* wall_seconds);
int fx_server_result(const fx_server* s, int64_t id, double* x_host, fx_solve_result* r, double* times,
                     double* monitor, int32_t* newton);

/* ------------------------------------------------------------------ PressureIndependMultiYield
 * Material points of the multi-yield-surface von Mises soil model (OpenSees nDMaterial
 * PressureIndependMultiYield, 3D; the reference's PressureIndependMultiYield<NS>,
 * src/physics/materials/pressure_independ_multi_yield.hpp: setup :102-139, initial_state :141-149,
 * update :218-224, the material stage of updateMaterialStage as `stage`). At most 40 surfaces.
 *   fx_pimy_create       in9 = rho, refShearModul, refBulkModul, cohesi, peakShearStra,
 *                        frictionAng, refPress, pressDependCoe, noYieldSurf; pairs = noYieldSurf
 *                        (gamma, G/Gmax) pairs of a user backbone, or NULL (hyperbolic backbone).
 *                        FX_E_INVALID for inputs OpenSees rejects, FX_E_UNSUPPORTED above 40
 *                        surfaces.
 *   fx_pimy_info         state values per point (31 + 8 surfaces) and the surfaces.
 *   fx_pimy_setup_values out[83] = residual pressure, friction angle, cohesion after setup, the 40
 *                        surface sizes, the 40 plastic moduli (surfaces past noYieldSurf 0).
 *   fx_pimy_init         the state of npoints new points (device; value k of point i at
 *                        state[k npoints + i]).
 *   fx_pimy_update       per point i: total strain strain[c npoints + i] (11 22 33 12 23 31,
 *                        engineering shear) from the committed state to the trial state (both
 *                        laid out as in fx_pimy_init; the trial state is written in full, so a
 *                        commit is a swap of the two buffers), stress[c npoints + i], the tangent
 *                        tangent[(6 r + c) npoints + i] (NULL: not stored), and *failed (device,
 *                        may be NULL) += the points that met a state OpenSees stops the program
 *                        for (their stress is NaN).
 *   fx_pimy_*_host       the same arithmetic on host arrays (failed: a host counter). */
typedef struct fx_pimy fx_pimy;
int fx_pimy_create(const double* in9, const double* pairs, fx_pimy** out);
void fx_pimy_destroy(fx_pimy* m);
int fx_pimy_info(const fx_pimy* m, int32_t* nstate, int32_t* surfaces);
int fx_pimy_setup_values(const fx_pimy* m, double* out);
int fx_pimy_init(fx_pimy* m, int64_t npoints, double* state, void* stream);
int fx_pimy_update(fx_pimy* m, int32_t stage, int64_t npoints, const double* committed, double* trial,
                   const double* strain, double* stress, double* tangent, int32_t* failed, void* stream);
/* Binds material m to parameter set `set` of a mesh (stdBrick with PressureIndependMultiYield
 * points: the reference's StdBrick<PressureIndependMultiYield<NS>>, std_brick.hpp:398-540, a
 * model material of that type). The set's elements run on the Gauss-point path (the box path is
 * taken out for the mesh); their points start from the material's state, elastic stage. The set's
 * density must equal the material's (the masses come from the set); betaK and betaKcomm Rayleigh
 * damping act through each point's current and committed tangents (the reference's damping stress,
 * std_brick.hpp:419-434, and effective_tangent, element_operator.hpp:58-75); betaKinit on the set
 * is FX_E_UNSUPPORTED (the reference refuses it too). Bind before creating solvers or running stages on the
 * mesh. fx_force_compute then updates every point (the trial state; fx_force_commit commits it),
 * the operator and its diagonal use each point's tangent of the last fx_force_compute (the
 * reference's stored tangents at that displacement; `initial` in fx_coeffs: the material's
 * reference elastic tangent), fx_force_plastic_points counts points with an active surface.
 *   fx_force_set_material_stage  updateMaterialStage for the set, PressureIndependMultiYield or
 *                                PressureDependMultiYield (InternalForce::set_material_stage,
 *                                src/exec/internal_force.cpp:511-515): 0 elastic, 1 plastic.
 *   fx_force_pimy_failed         points whose update met a state OpenSees stops for (stress NaN),
 *                                counted over all evaluations. */
int fx_force_set_pimy(fx_force* f, int32_t set, const fx_pimy* m);
int fx_force_set_material_stage(fx_force* f, int32_t set, int32_t stage);
int fx_force_pimy_failed(const fx_force* f, int64_t* count);
int fx_pimy_init_host(const fx_pimy* m, int64_t npoints, double* state);
int fx_pimy_update_host(const fx_pimy* m, int32_t stage, int64_t npoints, const double* committed, double* trial,
                        const double* strain, double* stress, double* tangent, int32_t* failed);

/* ------------------------------------------------------------------ PressureDependMultiYield
 * Material points of the pressure-dependent multi-yield-surface soil model with dilatancy and the
 * phase-transformation zone (OpenSees nDMaterial PressureDependMultiYield, 3D; the reference's
 * PressureDependMultiYield<NS>, src/physics/materials/pressure_depend_multi_yield.hpp: setup
 * :122-170, initial_state :173-177, update :248-262; `stage` is updateMaterialStage's 0 or 1; the
 * reference has no stage 2). At most 40 surfaces. The same calls as fx_pimy_*:
 *   fx_pdmy_create       in23 = rho, refShearModul, refBulkModul, frictionAng, peakShearStra,
 *                        refPress, pressDependCoe, PTAng, contrac, dilat1, dilat2, liquefac1,
 *                        liquefac2, liquefac3, noYieldSurf, e, cs1, cs2, cs3, pa, c, hv, pv (OpenSees'
 *                        order; hv = 0, pv = 1 for no volumetric plasticity); pairs or NULL.
 *   fx_pdmy_info         state values per point (89 + 6 surfaces) and the surfaces.
 *   fx_pdmy_setup_values out[85] = residual pressure, friction angle, phase-transformation angle,
 *                        its stress ratio, its octahedral strain, then 40 sizes, 40 plastic moduli.
 *   fx_pdmy_init / fx_pdmy_update / fx_pdmy_*_host as fx_pimy_* (value-major arrays; the trial
 *                        state is written in full, so a commit is a swap). */
typedef struct fx_pdmy fx_pdmy;
int fx_pdmy_create(const double* in23, const double* pairs, fx_pdmy** out);
void fx_pdmy_destroy(fx_pdmy* m);
int fx_pdmy_info(const fx_pdmy* m, int32_t* nstate, int32_t* surfaces);
int fx_pdmy_setup_values(const fx_pdmy* m, double* out);
int fx_pdmy_init(fx_pdmy* m, int64_t npoints, double* state, void* stream);
int fx_pdmy_update(fx_pdmy* m, int32_t stage, int64_t npoints, const double* committed, double* trial,
                   const double* strain, double* stress, double* tangent, int32_t* failed, void* stream);
/* Binds material m to parameter set `set` of a mesh, as fx_force_set_pimy (the reference's
 * StdBrick<PressureDependMultiYield<NS>>): Gauss-point path, elastic stage at first, the set's
 * density equal to the material's, betaK damping only; fx_force_set_material_stage,
 * fx_force_compute / commit, the operator (each point's stored tangent of the last compute, upper
 * triangle mirrored) and fx_force_pimy_failed work on it as on PressureIndependMultiYield sets. */
int fx_force_set_pdmy(fx_force* f, int32_t set, const fx_pdmy* m);
int fx_pdmy_init_host(const fx_pdmy* m, int64_t npoints, double* state);
int fx_pdmy_update_host(const fx_pdmy* m, int32_t stage, int64_t npoints, const double* committed, double* trial,
                        const double* strain, double* stress, double* tangent, int32_t* failed);

#ifdef __cplusplus
}
#endif
#endif
