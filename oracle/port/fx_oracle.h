/* Oracle (test infrastructure only): a plain-C restatement of the reference's hot path, used by
 * tests/, the smoke check and bench.py's CPU-baseline leg as the checker. It is never linked
 * into, called by or shipped with the product library.
 *
 * Every function follows the reference's operation order (file:line cited at each definition),
 * so that, compiled without fused multiply-adds (-ffp-contract=off), its results are the
 * reference's own bits; the tests pin that against oracle/_ref/libfxref.so (the reference built
 * here) and against the stored OpenSees golden vectors (tests/golden/).
 */
#ifndef FX_ORACLE_H
#define FX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One stdBrick parameter set (src/compile/batches.hpp:28-39 with StdBrick::Params,
 * src/physics/elements/std_brick.hpp:181-185) and its Rayleigh factors. */
typedef struct fxo_param {
  double E, nu, rho;
  double b[3];
  int32_t mass_type; /* 0 consistent, 1 lumped */
  int32_t pad_;
  double alphaM, betaK, betaKinit, betaKcomm;
} fxo_param;

/* One batch of stdBrick elements with ElasticIsotropic, as compile_model lays it out
 * (src/compile/batches.hpp:41-72): value[k * padded + e]. */
typedef struct fxo_mesh {
  int32_t num_nodes, num_equations, count, padded, num_params, pad_;
  const double* coords;           /* [3 * num_nodes], x[N] y[N] z[N] */
  const int32_t* node;            /* [8 * padded] */
  const int32_t* eq;              /* [24 * padded], -1 fixed */
  const int32_t* param;           /* [padded] */
  const fxo_param* params;        /* [num_params] */
  const double* nodal_mass;       /* [num_equations] or NULL */
  const double* nodal_alpha_mass; /* [num_equations] or NULL */
} fxo_mesh;

/* Element level (std_brick.hpp, element_operator.hpp). xe[8][3] node coordinates. */
void fxo_brick_compute(const fxo_param* p, const double* xe, const double* ue, const double* ve, double* fe,
                       double* Ke);
void fxo_brick_operator(const fxo_param* p, const double* k, const double* xe, const double* ve, double* ye);
void fxo_brick_diagonal(const fxo_param* p, const double* k, const double* xe, const int32_t* eq, double* de);
void fxo_brick_mass(const fxo_param* p, const double* xe, double* Me);
void fxo_brick_lumped_mass(const fxo_param* p, const double* xe, double* m);

/* System level (src/exec/internal_force.cpp). k = {stiffness, damping, mass}. */
void fxo_apply_operator(const fxo_mesh* m, const double* k, const double* x, double* y);
void fxo_operator_diagonal(const fxo_mesh* m, const double* k, double* d);
void fxo_force(const fxo_mesh* m, const double* u, const double* v, double* f);
void fxo_mass_times_ground(const fxo_mesh* m, int dir, double* y);

/* Vector kernels (src/solvers/vector_ops.cpp): the documented reduction order with `lanes`
 * lanes; fused = 1 forms each product-sum with fma() (the order a GPU build with contraction
 * follows), fused = 0 without (a host build). */
double fxo_dot(const double* x, const double* y, int64_t n, int lanes, int fused);

/* Jacobi-preconditioned CG (src/solvers/cg.cpp:24-71) on the mesh operator with
 * coefficients k; result = [converged, iterations, rhs_norm, initial_residual, final_residual,
 * indefinite]. */
void fxo_cg(const fxo_mesh* m, const double* k, const double* b, double* x, double rtol, double atol, int max_it,
            int lanes, double* result);
/* Jacobi-preconditioned FGMRES(restart) with CGS2 (src/solvers/gmres.cpp:32-123). */
void fxo_gmres(const fxo_mesh* m, const double* k, const double* b, double* x, double rtol, double atol, int max_it,
               int lanes, int restart, double* result);

/* ExplicitDifference step (src/exec/explicit_analysis.cpp:62-84, 687-705): predict, force,
 * correct with ground acceleration ag[3] acting along the equations' DOFs (eq_dof). */
void fxo_ed_step(const fxo_mesh* m, const double* mass, const int8_t* eq_dof, const double* ag, double dt, double* u,
                 double* vh, double* a, double* v_rec, double* f_work);

/* Ground motions (src/exec/ground_motion.cpp:21-77, 150-175): PathSeries::getFactor with a
 * uniform spacing (values[n], dt, cFactor, startTime, useLast) and PathTimeSeries::getFactor
 * with a time array (values[n], times[n], cFactor, *loc kept between calls). */
double fxo_path_uniform(const double* values, int64_t n, double dt, double factor, double start, int use_last,
                        double t);
double fxo_path_time(const double* values, const double* times, int64_t n, double factor, int* loc, double t);

/* One explicit step of a stage with npat UniformExcitation patterns whose ground accelerations
 * at the step's load time are accel[p] acting in DOF gdof[p] (explicit_analysis.cpp:51-58).
 * ExplicitDifference (:62-84, 700-711): predict, force at (u, vh), correct. CentralDifference
 * (:86-117, 712-721): v_elem = -c2 um, force at (u, v_elem), the diagonal solve with the lumped
 * alphaM masses cm; um, u, v_rec, a updated. f_work: neq doubles. */
void fxo_ed_stage_step(const fxo_mesh* m, const double* mass, const int8_t* eq_dof, const double* accel,
                       const int32_t* gdof, int npat, double dt, double* u, double* vh, double* a, double* v_rec,
                       double* f_work);
void fxo_cd_stage_step(const fxo_mesh* m, const double* mass, const double* cm, const int8_t* eq_dof,
                       const double* accel, const int32_t* gdof, int npat, double dt, double* u, double* um,
                       double* v_elem, double* a, double* v_rec, double* f_work);

/* Newmark form-D kernels (src/exec/implicit_stage.cpp:29-68). */
void fxo_newmark_predict(int64_t n, double* u, double* v, double* a, double* ut, double* vt, double* at, double a1,
                         double a2, double a3, double a4);
void fxo_newmark_update(int64_t n, const double* du, double* u, double* v, double* a, double c2, double c3);

/* J2 plasticity with linear isotropic/kinematic hardening, radial return (Simo and Hughes,
 * Computational Inelasticity, Box 3.2). No counterpart in the reference. state = [eps_p(6),
 * alpha, back(6)] in the reference's strain order 11 22 33 12 23 31 (engineering shear).
 * hk = kinematic share of H in [0, 1]. Writes sigma, D (6x6) and the trial state. Returns 1 if
 * the step was plastic. */
int fxo_j2_update(double E, double nu, double sigma_y, double H, double hk, const double* committed,
                  double* trial, const double* eps, double* sigma, double* D);

/* J2 system level (no counterpart in the reference): j2[4 * s] = {kind (0 elastic, 1 J2),
 * sigma_y, H, hk} per parameter set; per element and Gauss point, component c of point gp of
 * element e at [(c * 8 + gp) * padded + e]: state (13), consistent tangent (36, row-major).
 * fxo_force_j2: internal force at u, v from the committed state; writes the trial state, the
 * points' tangents and the number of plastic points. fxo_apply_j2 / fxo_diagonal_j2: the
 * operator and its diagonal with those tangents (initial: the elastic matrix instead). */
void fxo_force_j2(const fxo_mesh* m, const double* j2, const double* committed, double* trial, double* Dpts,
                  const double* u, const double* v, double* f, int* plastic);
void fxo_apply_j2(const fxo_mesh* m, const double* j2, const double* Dpts, const double* k, int initial,
                  const double* x, double* y);
void fxo_diagonal_j2(const fxo_mesh* m, const double* j2, const double* Dpts, const double* k, int initial,
                     double* d);

/* The host C library's exp (fn 0), log (1), pow (2, of x and y) and cos (3), element by element:
   the functions the reference calls, beside which the device update's own (fx_math_eval_host of
   the product library) are measured. */
void fxo_libm_eval(int fn, const double* x, const double* y, double* out, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
