// Time stepping: the ExplicitDifference step loop and the Newmark form-D kernels
// (src/exec/explicit_analysis.cpp:62-84, 687-705; src/exec/implicit_stage.cpp:29-68), and the
// stable time step (StdBrick::critical_dt, std_brick.hpp:629-694; stable_dt,
// src/physics/explicit_stability.hpp:16-32).
//
// One ExplicitDifference step is two launches: the force at (u, vh), then one fused pass that
// does the correction of this step and the prediction of the next (a = (-f + g)/m,
// v = vh + dt/8 (3a + a_old), vh += dt a, u += dt vh). The prediction only needs the corrected
// acceleration, so moving it into the correction pass changes no value. The steps run as a
// CUDA graph of a block of steps; the ground acceleration of each step is read from a device
// array indexed by a device step counter, so one captured graph serves every block.
#include <algorithm>
#include <cmath>
#include <vector>

#include "force.hpp"

namespace fx {
namespace {

// w (when set): u + beta vh of the force evaluation that follows, fma(beta, vh, u) as the box force
// kernel forms it
template <class T>
__global__ void k_ed_predict(T* __restrict__ u, T* __restrict__ vh, const T* __restrict__ a, T dt, int64_t n,
                             T* __restrict__ w, T beta) {
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const T v = vh[q] + a[q] * dt;
    vh[q] = v;
    const T un = u[q] + v * dt;
    u[q] = un;
    if (w) w[q] = fma(beta, v, un);
  }
}

// correction of step `step` and prediction of step `step + 1`; the full-step velocity v is written by
// the call's last step only (predict == 0): the steps between read the half-step velocity vh
template <class T>
__global__ void k_ed_correct_predict(const T* __restrict__ f, const T* __restrict__ m, const int8_t* __restrict__ dof,
                                     const double* __restrict__ ag, int* __restrict__ step, int dir, T dt,
                                     T* __restrict__ u, T* __restrict__ vh, T* __restrict__ a, T* __restrict__ v,
                                     int64_t n, int32_t record_eq, double* __restrict__ hist, int predict,
                                     T* __restrict__ w, T beta) {
  const int s = *step;
  const T g = ag ? static_cast<T>(ag[s]) : T(0);
  const T halfT = dt * T(0.125);
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const T mq = m[q];
    T gl = T(0);
    if (ag && dof[q] == dir) gl = -(mq * g);
    const T R = -f[q] + gl;
    const T an = R / mq;
    const T t = T(3) * an + a[q];
    const T vhq = vh[q];
    if (!predict) v[q] = vhq + t * halfT;  // (read only after the call's last step, which does not predict)
    a[q] = an;
    if (q == record_eq && hist) hist[s] = static_cast<double>(an);
    if (predict) {
      const T vn = vhq + an * dt;
      vh[q] = vn;
      const T un = u[q] + vn * dt;
      u[q] = un;
      if (w) w[q] = fma(beta, vn, un);
    }
  }
}

__global__ void k_step_advance(int* step) { ++*step; }

// ---- explicit stages with device ground motions
// Every operation of these kernels is an explicitly rounded IEEE operation (no contraction into
// fused multiply-adds), in the reference's order, so a stage on the bit-exact general path gives
// the reference's host bits.
struct MotionPattern {
  int32_t dof, uniform, use_last, pad_;
  int64_t n, off;  // samples, offset into the values (and times) arrays
  double fact, dt, factor;
};

// PathSeries::getFactor with a uniform spacing (src/exec/ground_motion.cpp:21-39), start 0
__device__ double path_uniform(const double* v, int64_t n, double dt, double factor, int use_last, double t) {
  if (t < 0.0) return 0.0;
  const double incr = __ddiv_rn(t, dt);
  // floor(incr) + 1 >= n, tested before the conversion (which could overflow for huge t / dt)
  if (!(incr < static_cast<double>(n - 1))) return use_last ? __dmul_rn(factor, v[n - 1]) : 0.0;
  const long long i1 = static_cast<long long>(floor(incr));
  const double v1 = v[i1], v2 = v[i1 + 1];
  return __dmul_rn(factor, __dadd_rn(v1, __dmul_rn(__dsub_rn(v2, v1), __dsub_rn(incr, static_cast<double>(i1)))));
}

// PathTimeSeries::getFactor (ground_motion.cpp:41-77): the interval walk from *loc, kept
__device__ double path_time(const double* v, const double* tm, int64_t n, double factor, int* loc, double t) {
  int l = *loc;
  double t1 = tm[l];
  if (t < t1 && l == 0) return 0.0;
  if (t == t1) return __dmul_rn(factor, v[l]);
  const int last = static_cast<int>(n) - 1;
  if (t > t1 && l == last) return 0.0;
  double t2 = tm[l + 1];
  if (t > t2) {
    while (t > t2 && l < last - 1) {
      ++l;
      t1 = t2;
      t2 = tm[l + 1];
    }
    *loc = l;
    if (t > t2) return 0.0;
  } else if (t < t1) {
    while (t < t1 && l > 0) {
      --l;
      t2 = t1;
      t1 = tm[l];
    }
    *loc = l;
    if (t < t1) return 0.0;
  }
  const double v1 = v[l], v2 = v[l + 1];
  return __dmul_rn(factor, __dadd_rn(v1, __ddiv_rn(__dmul_rn(__dsub_rn(v2, v1), __dsub_rn(t, t1)), __dsub_rn(t2, t1))));
}

// One thread: the stage's step counter and time, and every pattern's ground acceleration at the
// step's load time (GroundMotions::evaluate, ground_motion.cpp:150-175). ExplicitDifference
// evaluates after time += dt, CentralDifference before it (explicit_analysis.cpp:700-721).
// dt == 0: evaluate at *time only (no step).
__global__ void k_motions(const MotionPattern* __restrict__ pats, int npat, const double* __restrict__ values,
                          const double* __restrict__ times, int* __restrict__ loc, double* __restrict__ accel,
                          double* __restrict__ time, int* __restrict__ step, double dt, int advance_first) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (step) ++*step;
  if (advance_first) *time = __dadd_rn(*time, dt);
  const double t = *time;
  for (int p = 0; p < npat; ++p) {
    const MotionPattern& m = pats[p];
    double g = 0.0;  // GroundMotion::getAccel: 0 for t < 0
    if (t >= 0.0) {
      if (m.uniform) g = path_uniform(values + m.off, m.n, m.dt, m.factor, m.use_last, t);
      else g = path_time(values + m.off, times + m.off, m.n, m.factor, &loc[p], t);
    }
    accel[p] = __dmul_rn(m.fact, g);  // UniformExcitation: R = fact in its DOF
  }
  if (!advance_first && dt != 0.0) *time = __dadd_rn(*time, dt);
}

// ground_load (explicit_analysis.cpp:51-58)
__device__ __forceinline__ double ground_load(double mq, int dof_q, const double* accel, const int* gdof, int npat) {
  double r = 0.0;
  for (int p = 0; p < npat; ++p)
    if (gdof[p] == dof_q) r = __dsub_rn(r, __dmul_rn(mq, accel[p]));
  return r;
}

// ed_predict (explicit_analysis.cpp:62-69); w (box path): u + beta vh for the force, as the box
// force kernel forms it
__global__ void k_stage_ed_predict(double* __restrict__ u, double* __restrict__ vh, const double* __restrict__ a,
                                   double dt, int64_t n, double* __restrict__ w, double beta) {
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = __dadd_rn(vh[q], __dmul_rn(a[q], dt));
    vh[q] = v;
    const double un = __dadd_rn(u[q], __dmul_rn(v, dt));
    u[q] = un;
    if (w) w[q] = __fma_rn(beta, v, un);
  }
}

// ed_correct (explicit_analysis.cpp:71-84), then the next step's ed_predict when `predict`
__global__ void k_stage_ed_correct(const double* __restrict__ f, const double* __restrict__ m,
                                   const int8_t* __restrict__ dof, const double* __restrict__ accel,
                                   const int* __restrict__ gdof, int npat, double dt, double* __restrict__ u,
                                   double* __restrict__ vh, double* __restrict__ a, double* __restrict__ v,
                                   int64_t n, const int* __restrict__ step, int32_t record_eq,
                                   double* __restrict__ hist, int predict, double* __restrict__ w, double beta) {
  const double halfT = __dmul_rn(dt, 0.125);
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double mq = m[q];
    const double R = __dadd_rn(-f[q], ground_load(mq, dof[q], accel, gdof, npat));
    const double an = __ddiv_rn(R, mq);
    const double t = __dadd_rn(__dmul_rn(3.0, an), a[q]);
    const double vhq = vh[q];
    v[q] = __dadd_rn(vhq, __dmul_rn(t, halfT));
    a[q] = an;
    if (q == record_eq && hist) hist[*step] = an;
    if (predict) {
      const double vn = __dadd_rn(vhq, __dmul_rn(an, dt));
      vh[q] = vn;
      const double un = __dadd_rn(u[q], __dmul_rn(vn, dt));
      u[q] = un;
      if (w) w[q] = __fma_rn(beta, vn, un);
    }
  }
}

// cd_garbage_velocity (explicit_analysis.cpp:86-92)
__global__ void k_stage_cd_garbage(double* __restrict__ ve, const double* __restrict__ um, double c2, int64_t n,
                                   double* __restrict__ w, const double* __restrict__ u, double beta) {
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = __dmul_rn(um[q], -c2);
    ve[q] = v;
    if (w) w[q] = __fma_rn(beta, v, u[q]);
  }
}

// cd_solve (explicit_analysis.cpp:94-117), then the next step's garbage velocity -c2 um
__global__ void k_stage_cd_solve(const double* __restrict__ f, const double* __restrict__ m,
                                 const double* __restrict__ cm, const int8_t* __restrict__ dof,
                                 const double* __restrict__ accel, const int* __restrict__ gdof, int npat, double c2,
                                 double c3, double dt, double* __restrict__ u, double* __restrict__ um,
                                 double* __restrict__ v, double* __restrict__ a, double* __restrict__ ve, int64_t n,
                                 const int* __restrict__ step, int32_t record_eq, double* __restrict__ hist,
                                 int next, double* __restrict__ w, double beta) {
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double uq = u[q], umq = um[q], mq = m[q];
    const double ag = __dadd_rn(__dmul_rn(uq, __dmul_rn(-2.0, c3)), __dmul_rn(umq, c3));
    const double R = __dadd_rn(__dsub_rn(-f[q], __dmul_rn(mq, ag)), ground_load(mq, dof[q], accel, gdof, npat));
    const double A = __dadd_rn(__dmul_rn(mq, c3), __dmul_rn(cm ? cm[q] : 0.0, c2));
    const double U = __ddiv_rn(R, A);
    double Ud = __dmul_rn(U, 3.0);
    Ud = __dadd_rn(Ud, __dmul_rn(uq, -4.0));
    Ud = __dadd_rn(Ud, umq);
    Ud = __dmul_rn(Ud, c2);
    const double Udd = __ddiv_rn(__dsub_rn(Ud, v[q]), dt);
    um[q] = uq;
    u[q] = U;
    v[q] = Ud;
    a[q] = Udd;
    if (q == record_eq && hist) hist[*step] = Udd;
    if (next) {
      const double vn = __dmul_rn(uq, -c2);
      ve[q] = vn;
      if (w) w[q] = __fma_rn(beta, vn, U);
    }
  }
}

// Non-finite displacements (explicit_analysis.cpp:369-378, all_finite): a count, exact in any order.
__global__ void k_count_nonfinite(const double* __restrict__ u, int64_t n, int* __restrict__ bad) {
  int local = 0;
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x)
    local += isfinite(u[q]) ? 0 : 1;
  local = __reduce_add_sync(0xffffffffu, local);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(bad, local);
}

__global__ void k_newmark_predict(double* __restrict__ u, double* __restrict__ v, double* __restrict__ a,
                                  double* __restrict__ ut, double* __restrict__ vt, double* __restrict__ at, double a1,
                                  double a2, double a3, double a4, int64_t n) {
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    ut[q] = u[q];
    vt[q] = v[q];
    at[q] = a[q];
    v[q] = v[q] * a1 + at[q] * a2;
    a[q] = a[q] * a4 + vt[q] * a3;
  }
}

__global__ void k_newmark_update(const double* __restrict__ du, double* __restrict__ u, double* __restrict__ v,
                                 double* __restrict__ a, double c2, double c3, int64_t n) {
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    u[q] += du[q];
    v[q] += du[q] * c2;
    a[q] += du[q] * c3;
  }
}

unsigned ew(int64_t n) {
  const int64_t blocks = (n + 255) / 256;
  const int64_t cap = static_cast<int64_t>(num_sms()) * 8;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min(blocks, cap)));
}

// Cyclic Jacobi largest eigenvalue of a symmetric 24 x 24 matrix (Golub and Van Loan, Algorithm
// 8.4.1, the rotation the reference's sym_eigen.hpp uses).
double max_eig24(double A[24][24]) {
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, dg = 0.0;
    for (int i = 0; i < 24; ++i) {
      dg += A[i][i] * A[i][i];
      for (int j = i + 1; j < 24; ++j) off += A[i][j] * A[i][j];
    }
    if (off <= 1e-30 * dg || off == 0.0) break;
    for (int p = 0; p < 23; ++p)
      for (int q = p + 1; q < 24; ++q) {
        const double apq = A[p][q];
        if (apq == 0.0) continue;
        const double th = (A[q][q] - A[p][p]) / (2.0 * apq);
        const double t = (th >= 0.0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 24; ++k) {
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 24; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        A[p][q] = A[q][p] = 0.0;
      }
  }
  double l = A[0][0];
  for (int i = 1; i < 24; ++i) l = std::max(l, A[i][i]);
  return l;
}

// omega^2 of one element: K with the elastic tangent, lumped mass (std_brick.hpp:658-688).
double element_omega_sq(const ParamGP& p, const double xl[3][8]) {
  double m[8];
  lumped_mass(p, xl, m);
  double D[6][6];
  elastic_D(p, D);
  double A[24][24];
  for (int a = 0; a < 24; ++a)
    for (int c = 0; c < 24; ++c) A[a][c] = 0.0;
  for (int gp = 0; gp < 8; ++gp) {
    PointShape s;
    point_shape(xl, gp, s);
    for (int j = 0; j < 8; ++j)
      for (int k = 0; k < 8; ++k) {
        double blk[3][3];
        block_tangent(s, D, j, k, blk);
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) A[3 * j + a][3 * k + c] += blk[a][c];
      }
  }
  double ism[8];
  for (int j = 0; j < 8; ++j) {
    if (!(m[j] > 0.0)) return 0.0;
    ism[j] = 1.0 / std::sqrt(m[j]);
  }
  for (int a = 0; a < 24; ++a)
    for (int c = 0; c < 24; ++c) A[a][c] *= ism[a / 3] * ism[c / 3];
  return max_eig24(A);
}

double stable_dt(int scheme, const ParamGP& p, double w2) {
  if (!(w2 > 0.0)) return INFINITY;
  const double w = std::sqrt(w2);
  if (scheme == 0) return 2.0 / w;
  const double beta = p.betaK + p.betaKinit + p.betaKcomm;
  const double c = p.alphaM + beta * w2;
  return 4.0 / (std::sqrt(c * c + 4.0 * w2) + c);
}

}  // namespace

void newmark_predict(int64_t n, double* u, double* v, double* a, double* ut, double* vt, double* at, double a1,
                     double a2, double a3, double a4, cudaStream_t st) {
  if (n <= 0) return;
  k_newmark_predict<<<ew(n), 256, 0, st>>>(u, v, a, ut, vt, at, a1, a2, a3, a4, n);
  FX_LAUNCH_CHECK("newmark_predict");
}
void newmark_update(int64_t n, const double* du, double* u, double* v, double* a, double c2, double c3,
                    cudaStream_t st) {
  if (n <= 0) return;
  k_newmark_update<<<ew(n), 256, 0, st>>>(du, u, v, a, c2, c3, n);
  FX_LAUNCH_CHECK("newmark_update");
}

}  // namespace fx

namespace {
template <class F>
int guard(F&& f) {
  try {
    f();
    return FX_OK;
  } catch (const fx::Error& e) {
    fx::set_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    fx::set_error(e.what());
    return FX_E_INVALID;
  }
}

fx::ExplicitWork& work_of(fx_force* f) { return f->s.xw; }

template <class T>
void explicit_run(fx_force* f, const T* mass, int32_t dir, const double* ag_host, int32_t steps, double dt, T* u,
                  T* vh, T* a, T* v, cudaStream_t st) {
  using namespace fx;
  ForceState& s = f->s;
  if (steps < 0 || !(dt > 0.0)) throw Error(FX_E_INVALID, "fx_explicit_run: steps >= 0 and dt > 0 required");
  if (ag_host && (dir < 0 || dir > 2)) throw Error(FX_E_INVALID, "fx_explicit_run: dir must be 0, 1 or 2");
  if (sizeof(T) == 4 && !s.use_box_force()) throw Error(FX_E_UNSUPPORTED, "the FP32 explicit step runs on the box path only");
  ExplicitWork& w = work_of(f);
  const int64_t n = s.neq;
  if (w.step.n == 0) w.step.alloc(1);
  if (ag_host) {
    if (w.ag.n < static_cast<size_t>(steps) + 1) w.ag.alloc(static_cast<size_t>(steps) + 1);
    FX_CUDA(cudaMemcpyAsync(w.ag.ptr, ag_host, sizeof(double) * steps, cudaMemcpyHostToDevice, st));
  }
  if (w.record_eq >= 0 && w.hist.n < static_cast<size_t>(steps) + 1) w.hist.alloc(static_cast<size_t>(steps) + 1);
  T* fbuf;
  if constexpr (sizeof(T) == 8) {
    if (w.f64.n < static_cast<size_t>(n)) w.f64.alloc(static_cast<size_t>(std::max<int64_t>(n, 1)));
    fbuf = w.f64.ptr;
  } else {
    if (w.f32.n < static_cast<size_t>(n)) w.f32.alloc(static_cast<size_t>(std::max<int64_t>(n, 1)));
    fbuf = w.f32.ptr;
  }
  // on the box path the update passes also form w = u + beta vh, so the force stages one vector
  T* wbuf = nullptr;
  if (s.use_box_force()) {
    if constexpr (sizeof(T) == 8) {
      if (w.w64.n < static_cast<size_t>(n)) w.w64.alloc(static_cast<size_t>(std::max<int64_t>(n, 1)));
      wbuf = w.w64.ptr;
    } else {
      if (w.w32.n < static_cast<size_t>(n)) w.w32.alloc(static_cast<size_t>(std::max<int64_t>(n, 1)));
      wbuf = w.w32.ptr;
    }
  }
  const T tbeta = static_cast<T>(s.box.beta);
  FX_CUDA(cudaMemsetAsync(w.step.ptr, 0, sizeof(int), st));
  if (steps == 0) return;
  const T tdt = static_cast<T>(dt);
  k_ed_predict<T><<<ew(n), 256, 0, st>>>(u, vh, a, tdt, n, wbuf, tbeta);
  FX_LAUNCH_CHECK("ed_predict");
  const double* agp = ag_host ? w.ag.ptr : nullptr;
  auto one_step = [&](int predict) {
    if constexpr (sizeof(T) == 8) {
      if (wbuf) box_force_w(s, wbuf, vh, fbuf, st);
      else general_force(s, u, vh, fbuf, st);
    } else {
      box_force_w_f32(s, wbuf, vh, fbuf, st);
    }
    k_ed_correct_predict<T><<<ew(n), 256, 0, st>>>(fbuf, mass, s.eq_dof.ptr, agp, w.step.ptr, dir, tdt, u, vh, a, v, n,
                                                   w.record_eq, w.hist.ptr, predict, wbuf, tbeta);
    k_step_advance<<<1, 1, 0, st>>>(w.step.ptr);
    FX_LAUNCH_CHECK("ed_step");
  };
  // first step eagerly (coefficient tables, attributes), then graphs of `block` steps
  const int block = 16;
  int done = 0;
  one_step(steps > 1);
  ++done;
  cudaStream_t cs = st;
  bool own_stream = false;
  if (cs == nullptr) {  // the legacy stream cannot be captured: run the graph on a private stream
    FX_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    own_stream = true;
    cudaEvent_t e;
    FX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    FX_CUDA(cudaEventRecord(e, st));
    FX_CUDA(cudaStreamWaitEvent(cs, e, 0));
    cudaEventDestroy(e);
  }
  st = cs;
  cudaGraphExec_t exec = nullptr;
  while (done < steps) {
    const int left = steps - done;
    if (left > block) {
      if (!exec) {
        cudaGraph_t g = nullptr;
        FX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < block; ++i) one_step(1);
        FX_CUDA(cudaStreamEndCapture(st, &g));
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        FX_CUDA(e);
      }
      FX_CUDA(cudaGraphLaunch(exec, st));
      done += block;
    } else {
      one_step(left > 1);
      ++done;
    }
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (own_stream) {
    FX_CUDA(cudaStreamSynchronize(cs));
    cudaStreamDestroy(cs);
  }
}
}  // namespace

// UniformExcitation patterns with their series, on the device (exec::GroundMotions).
struct fx_motions {
  int device = 0;
  std::vector<fx::MotionPattern> pats;
  std::vector<double> values, times;
  fx::DeviceArray<fx::MotionPattern> d_pats;
  fx::DeviceArray<double> d_values, d_times, d_accel, d_time;
  fx::DeviceArray<int> d_dof, d_loc;
  bool uploaded = false;

  void upload() {
    if (uploaded) return;
    d_pats.upload(pats);
    d_values.upload(values.empty() ? std::vector<double>(1, 0.0) : values);
    d_times.upload(times.empty() ? std::vector<double>(1, 0.0) : times);
    std::vector<int> dof;
    for (const auto& p : pats) dof.push_back(p.dof);
    d_dof.upload(dof.empty() ? std::vector<int>(1, -1) : dof);
    d_loc.upload(std::vector<int>(std::max<size_t>(pats.size(), 1), 0));
    d_accel.upload(std::vector<double>(std::max<size_t>(pats.size(), 1), 0.0));
    d_time.upload(std::vector<double>(1, 0.0));
    uploaded = true;
  }
};

namespace {

// Smallest stable step of the elements (InternalForce::min_critical_dt): on a box grid of elastic
// or J2 sets, whose elements of one parameter set are congruent, one eigenproblem per set on the
// host; otherwise every element's on the device (general_min_critical_dt).
double exact_min_dt(fx::ForceState& s, int scheme, cudaStream_t st) {
  using namespace fx;
  if (!s.box.qualifies || s.has_pimy || s.has_pdmy) return general_min_critical_dt(s, scheme, nullptr, s.count, nullptr, st);
  double best = 1e300;
  std::vector<char> seen(static_cast<size_t>(s.nparams), 0);
  for (int32_t e = 0; e < s.count; ++e) {
    const int32_t pi = s.param_h[e];
    if (seen[pi]) continue;
    seen[pi] = 1;
    double xl[3][8];
    for (int a = 0; a < 8; ++a) {
      const int32_t nd = s.node_h[static_cast<size_t>(a) * s.P + e];
      for (int d = 0; d < 3; ++d) xl[d][a] = s.coords_h[static_cast<size_t>(d) * s.N + nd];
    }
    const ParamGP& p = s.params_h[pi];
    best = std::min(best, stable_dt(scheme, p, element_omega_sq(p, xl)));
  }
  return best;
}

int count_nonfinite(fx::ExplicitWork& w, const double* u, int64_t n, cudaStream_t st) {
  if (w.bad.n == 0) w.bad.alloc(1);
  FX_CUDA(cudaMemsetAsync(w.bad.ptr, 0, sizeof(int), st));
  if (n > 0) fx::k_count_nonfinite<<<fx::ew(n), 256, 0, st>>>(u, n, w.bad.ptr);
  FX_LAUNCH_CHECK("nan_check");
  int bad = 0;
  FX_CUDA(cudaMemcpyAsync(&bad, w.bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  FX_CUDA(cudaStreamSynchronize(st));
  return bad;
}

// An explicit stage (src/exec/explicit_analysis.cpp:665-725 without local time stepping, exact
// constraints, DRM or recorders). Per ExplicitDifference step: [motions: time += dt, ag(time)]
// [force at (u, vh)] [ed_correct + the next ed_predict] [commit]; per CentralDifference step:
// [motions: ag(time), time += dt] [force at (u, -c2 um)] [cd_solve + the next garbage velocity]
// [commit]. The steps after the first run as CUDA graphs of 16.
void explicit_stage(fx_force* f, int scheme, const double* mass, const double* cm, fx_motions* mo, int32_t steps,
                    double dt, double* time, double* u, double* v, double* a, int resume, cudaStream_t st) {
  using namespace fx;
  ForceState& s = f->s;
  if (scheme != 0 && scheme != 1) throw Error(FX_E_INVALID, "fx_explicit_stage: scheme must be 0 (CD) or 1 (ED)");
  if (steps < 0 || !(dt > 0.0) || !time) throw Error(FX_E_INVALID, "fx_explicit_stage: steps >= 0, dt > 0 and time required");
  ExplicitWork& w = work_of(f);
  if (resume && w.carry_scheme != scheme) throw Error(FX_E_INVALID, "fx_explicit_stage: nothing to resume for this scheme");
  const int64_t n = s.neq;
  const size_t nn = static_cast<size_t>(std::max<int64_t>(n, 1));
  if (w.carry.n < nn) w.carry.alloc(nn);
  if (w.v_elem.n < nn) w.v_elem.alloc(nn);
  if (w.f64.n < nn) w.f64.alloc(nn);
  if (w.step.n == 0) w.step.alloc(1);
  if (w.time.n == 0) w.time.alloc(1);
  if (w.record_eq >= 0 && w.hist.n < static_cast<size_t>(steps) + 1) w.hist.alloc(static_cast<size_t>(steps) + 1);
  fx_motions none;
  fx_motions* m = mo ? mo : &none;
  m->upload();
  const int npat = static_cast<int>(m->pats.size());
  const double c2 = 0.5 / dt, c3 = 1.0 / (dt * dt);
  double* carry = w.carry.ptr;  // ED: the half-step velocity; CD: the previous displacement
  double* ve = scheme == 1 ? carry : w.v_elem.ptr;
  FX_CUDA(cudaMemcpyAsync(w.time.ptr, time, sizeof(double), cudaMemcpyHostToDevice, st));
  const int minus_one = -1;
  FX_CUDA(cudaMemcpyAsync(w.step.ptr, &minus_one, sizeof(int), cudaMemcpyHostToDevice, st));
  if (!resume && n > 0) {  // domainChanged: ED starts vh from the committed velocity, CD takes Utm1 = Ut
    FX_CUDA(cudaMemcpyAsync(carry, scheme == 1 ? v : u, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  }
  w.carry_scheme = scheme;
  if (!resume) {  // the stage's stable step against dt (explicit_analysis.cpp:582-653)
    w.stage_step = 0;
    w.warned = false;
    w.stage_dt_crit = exact_min_dt(s, scheme, st);
    if (dt > w.stage_dt_crit) {
      if (!w.allow_unstable)
        throw Error(FX_E_UNSTABLE, "fx_explicit_stage: dt = " + std::to_string(dt) + " is above the stable step " +
                                       std::to_string(w.stage_dt_crit) + " (reduce dt, or allow an unstable dt)");
      w.warned = true;
    }
    w.recheck = w.stable_interval > 0 && stability_may_change(s);
    if (w.recheck) prepare_stability_bounds(s, st);
  }
  if (steps == 0) {
    FX_CUDA(cudaStreamSynchronize(st));
    return;
  }
  // on the box path the update passes also form w = u + beta v_elem: the force stages one vector
  double* wbuf = nullptr;
  if (s.use_box_force()) {
    if (w.w64.n < nn) w.w64.alloc(nn);
    wbuf = w.w64.ptr;
  }
  const double beta = s.box.beta;
  if (n > 0) {
    if (scheme == 1) k_stage_ed_predict<<<ew(n), 256, 0, st>>>(u, carry, a, dt, n, wbuf, beta);
    else k_stage_cd_garbage<<<ew(n), 256, 0, st>>>(ve, carry, c2, n, wbuf, u, beta);
    FX_LAUNCH_CHECK("explicit_stage_begin");
  }
  double* fbuf = w.f64.ptr;
  auto one_step = [&](int more) {
    k_motions<<<1, 32, 0, st>>>(m->d_pats.ptr, npat, m->d_values.ptr, m->d_times.ptr, m->d_loc.ptr, m->d_accel.ptr,
                                w.time.ptr, w.step.ptr, dt, scheme == 1);
    if (n > 0) {
      if (wbuf) box_force_w(s, wbuf, ve, fbuf, st);
      else general_force(s, u, ve, fbuf, st);
      if (scheme == 1)
        k_stage_ed_correct<<<ew(n), 256, 0, st>>>(fbuf, mass, s.eq_dof.ptr, m->d_accel.ptr, m->d_dof.ptr, npat, dt, u,
                                                  carry, a, v, n, w.step.ptr, w.record_eq, w.hist.ptr, more, wbuf,
                                                  beta);
      else
        k_stage_cd_solve<<<ew(n), 256, 0, st>>>(fbuf, mass, cm, s.eq_dof.ptr, m->d_accel.ptr, m->d_dof.ptr, npat, c2,
                                                c3, dt, u, carry, v, a, ve, n, w.step.ptr, w.record_eq, w.hist.ptr,
                                                more, wbuf, beta);
    }
    FX_LAUNCH_CHECK("explicit_stage_step");
    if (s.has_j2)  // Domain::commit after every step
      FX_CUDA(cudaMemcpyAsync(s.j2_committed.ptr, s.j2_trial.ptr, s.j2_committed.bytes(), cudaMemcpyDeviceToDevice, st));
    pimy_commit(s, st);
  };
  // The last step does no prediction: u, v, a are the stage's end state; a resumed call
  // starts with the prediction (ED) or the garbage velocity (CD) from the carried vector.
  const int block = 16;
  int done = 0;
  one_step(steps > 1);
  ++done;
  cudaStream_t cs = st;
  bool own_stream = false;
  if (cs == nullptr) {  // the legacy stream cannot be captured: run the graph on a private stream
    FX_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    own_stream = true;
    cudaEvent_t e;
    FX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    FX_CUDA(cudaEventRecord(e, st));
    FX_CUDA(cudaStreamWaitEvent(cs, e, 0));
    cudaEventDestroy(e);
  }
  st = cs;
  cudaGraphExec_t exec = nullptr;
  // the periodic checks (explicit_analysis.cpp:732-765) after the steps whose stage index is a
  // multiple of their interval: the steps run in pieces that end there
  auto to_next = [&](int32_t interval, int64_t k) -> int64_t {
    return interval > 0 ? interval - k % interval : INT64_MAX;
  };
  auto finish = [&]() {  // the stage time back to the host; the private stream released
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    FX_CUDA(cudaMemcpyAsync(time, w.time.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
    FX_CUDA(cudaStreamSynchronize(st));
    if (own_stream) cudaStreamDestroy(cs);
    own_stream = false;
  };
  std::string failure;
  int failure_code = FX_OK;
  auto checks = [&](int64_t k) {  // after stage step k
    if (w.recheck && w.stable_interval > 0 && k % w.stable_interval == 0) {
      // the bound never overstates the step; where it falls below dt the exact check decides
      double dtc = min_critical_dt_bound(s, scheme, st);
      if (dt > dtc) dtc = general_min_critical_dt(s, scheme, nullptr, s.count, nullptr, st);
      if (dt > dtc && !w.warned) {
        if (!w.allow_unstable) {
          failure_code = FX_E_UNSTABLE;
          failure = "fx_explicit_stage: at step " + std::to_string(k) + " the stable step fell to " +
                    std::to_string(dtc) + " (" + std::to_string(w.stage_dt_crit) + " at the start of the stage), below dt = " +
                    std::to_string(dt) + ": the material stiffened";
          return false;
        }
        w.warned = true;
      }
    }
    if (w.nan_interval > 0 && k % w.nan_interval == 0 && count_nonfinite(w, u, n, st) > 0) {
      failure_code = FX_E_DIVERGED;
      failure = "fx_explicit_stage: displacements are not finite at step " + std::to_string(k) +
                ": the analysis is unstable";
      return false;
    }
    return true;
  };
  bool ok = checks(w.stage_step + done);
  while (ok && done < steps) {
    const int64_t k = w.stage_step + done;
    const int64_t piece = std::min<int64_t>({steps - done, to_next(w.nan_interval, k), to_next(w.stable_interval, k)});
    for (int64_t i = 0; i < piece;) {
      if (piece - i > block) {
        if (!exec) {
          cudaGraph_t g = nullptr;
          FX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
          for (int j = 0; j < block; ++j) one_step(1);
          FX_CUDA(cudaStreamEndCapture(st, &g));
          const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
          cudaGraphDestroy(g);
          FX_CUDA(e);
        }
        FX_CUDA(cudaGraphLaunch(exec, st));
        i += block;
      } else {
        one_step(steps - (done + i) > 1);
        ++i;
      }
    }
    done += static_cast<int>(piece);
    ok = checks(w.stage_step + done);
  }
  w.stage_step += done;
  if (ok && count_nonfinite(w, u, n, st) > 0) {  // the end of every call
    failure_code = FX_E_DIVERGED;
    failure = "fx_explicit_stage: displacements are not finite at the end of the stage (step " +
              std::to_string(w.stage_step) + ")";
  }
  finish();
  if (failure_code != FX_OK) throw Error(failure_code, failure);
}
}  // namespace

extern "C" {

int fx_motions_create(fx_motions** out) {
  return guard([&] {
    if (!out) throw fx::Error(FX_E_INVALID, "fx_motions_create: null output");
    auto m = std::make_unique<fx_motions>();
    FX_CUDA(cudaGetDevice(&m->device));
    *out = m.release();
  });
}

int fx_motions_destroy(fx_motions* m) {
  delete m;
  return FX_OK;
}

int fx_motions_add(fx_motions* m, int32_t dof, double fact, const double* values, const double* times, int32_t n,
                   double dt, double factor, int32_t use_last, int32_t prepend_zero) {
  return guard([&] {
    if (!m || !values || n < 1 || dof < 0 || dof > 2) throw fx::Error(FX_E_INVALID, "fx_motions_add: bad arguments");
    if (!times && !(dt > 0.0)) throw fx::Error(FX_E_INVALID, "fx_motions_add: a uniform series needs dt > 0");
    if (times && n < 2) throw fx::Error(FX_E_INVALID, "fx_motions_add: a time series needs two samples");
    fx::MotionPattern p{};
    p.dof = dof;
    p.uniform = times ? 0 : 1;
    p.use_last = use_last ? 1 : 0;
    p.fact = fact;
    p.dt = dt;
    p.factor = factor;
    // values and times run in parallel (a uniform series' times stay 0)
    p.off = static_cast<int64_t>(m->values.size());
    // PathSeries' constructor puts a zero first when asked (ground_motion.cpp:88)
    if (!times && prepend_zero) m->values.push_back(0.0);
    m->values.insert(m->values.end(), values, values + n);
    p.n = static_cast<int64_t>(m->values.size()) - p.off;
    if (times) m->times.insert(m->times.end(), times, times + n);
    m->times.resize(m->values.size(), 0.0);
    m->pats.push_back(p);
    m->uploaded = false;
  });
}

int fx_motions_evaluate(fx_motions* m, double t, double* accel) {
  return guard([&] {
    if (!m || (!accel && !m->pats.empty())) throw fx::Error(FX_E_INVALID, "fx_motions_evaluate: bad arguments");
    m->upload();
    FX_CUDA(cudaMemcpy(m->d_time.ptr, &t, sizeof(double), cudaMemcpyHostToDevice));
    fx::k_motions<<<1, 32>>>(m->d_pats.ptr, static_cast<int>(m->pats.size()), m->d_values.ptr, m->d_times.ptr,
                             m->d_loc.ptr, m->d_accel.ptr, m->d_time.ptr, nullptr, 0.0, 0);
    FX_LAUNCH_CHECK("motions_evaluate");
    if (!m->pats.empty())
      FX_CUDA(cudaMemcpy(accel, m->d_accel.ptr, sizeof(double) * m->pats.size(), cudaMemcpyDeviceToHost));
  });
}

int fx_explicit_stage(fx_force* f, int32_t scheme, const double* mass, const double* alpha_mass, fx_motions* motions,
                      int32_t steps, double dt, double* time, double* u, double* v, double* a, int32_t resume,
                      void* stream) {
  return guard([&] {
    if (!f || (f->s.neq > 0 && (!mass || !u || !v || !a))) throw fx::Error(FX_E_INVALID, "fx_explicit_stage: bad arguments");
    explicit_stage(f, scheme, mass, alpha_mass, motions, steps, dt, time, u, v, a, resume,
                   static_cast<cudaStream_t>(stream));
  });
}

int fx_explicit_run(fx_force* f, const double* mass, int32_t dir, const double* ag_host, int32_t steps, double dt,
                    double* u, double* vh, double* a, double* v, void* stream) {
  return guard([&] {
    if (!f || (f->s.neq > 0 && (!mass || !u || !vh || !a || !v))) throw fx::Error(FX_E_INVALID, "fx_explicit_run: bad arguments");
    explicit_run<double>(f, mass, dir, ag_host, steps, dt, u, vh, a, v, static_cast<cudaStream_t>(stream));
  });
}

int fx_explicit_run_f32(fx_force* f, const float* mass, int32_t dir, const double* ag_host, int32_t steps, double dt,
                        float* u, float* vh, float* a, float* v, void* stream) {
  return guard([&] {
    if (!f || (f->s.neq > 0 && (!mass || !u || !vh || !a || !v)))
      throw fx::Error(FX_E_INVALID, "fx_explicit_run_f32: bad arguments");
    explicit_run<float>(f, mass, dir, ag_host, steps, dt, u, vh, a, v, static_cast<cudaStream_t>(stream));
  });
}

int fx_explicit_record(fx_force* f, int32_t eq, double* hist_dev, int32_t count) {
  return guard([&] {
    if (!f || eq >= f->s.neq || count < 0) throw fx::Error(FX_E_INVALID, "fx_explicit_record: bad arguments");
    fx::ExplicitWork& w = work_of(f);
    if (hist_dev == nullptr) {
      w.record_eq = eq < 0 ? -1 : eq;
      return;
    }
    if (w.hist.n == 0) throw fx::Error(FX_E_INVALID, "fx_explicit_record: nothing recorded");
    const size_t n = std::min(static_cast<size_t>(count), w.hist.n);
    FX_CUDA(cudaMemcpy(hist_dev, w.hist.ptr, n * sizeof(double), cudaMemcpyDeviceToDevice));
  });
}

int fx_newmark_predict(int64_t n, double* u, double* v, double* a, double* ut, double* vt, double* at, double a1,
                       double a2, double a3, double a4, void* stream) {
  return guard([&] {
    if (n <= 0) return;
    fx::k_newmark_predict<<<fx::ew(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(u, v, a, ut, vt, at, a1, a2, a3, a4, n);
    FX_LAUNCH_CHECK("newmark_predict");
  });
}

int fx_newmark_update(int64_t n, const double* du, double* u, double* v, double* a, double c2, double c3,
                      void* stream) {
  return guard([&] {
    if (n <= 0) return;
    fx::k_newmark_update<<<fx::ew(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(du, u, v, a, c2, c3, n);
    FX_LAUNCH_CHECK("newmark_update");
  });
}

int fx_min_critical_dt(fx_force* f, int32_t scheme, double* dt) {
  return guard([&] {
    if (!f || !dt || (scheme != 0 && scheme != 1)) throw fx::Error(FX_E_INVALID, "fx_min_critical_dt: bad arguments");
    *dt = exact_min_dt(f->s, scheme, nullptr);
  });
}

int fx_element_critical_dts(fx_force* f, int32_t scheme, double* dt_dev, void* stream) {
  return guard([&] {
    if (!f || (f->s.count > 0 && !dt_dev) || (scheme != 0 && scheme != 1))
      throw fx::Error(FX_E_INVALID, "fx_element_critical_dts: bad arguments");
    fx::general_min_critical_dt(f->s, scheme, nullptr, f->s.count, dt_dev, static_cast<cudaStream_t>(stream));
  });
}

int fx_stability_prepare(fx_force* f, void* stream) {
  return guard([&] {
    if (!f) throw fx::Error(FX_E_INVALID, "fx_stability_prepare: bad arguments");
    fx::prepare_stability_bounds(f->s, static_cast<cudaStream_t>(stream));
    FX_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  });
}

int fx_min_critical_dt_bound(fx_force* f, int32_t scheme, double* dt, void* stream) {
  return guard([&] {
    if (!f || !dt || (scheme != 0 && scheme != 1)) throw fx::Error(FX_E_INVALID, "fx_min_critical_dt_bound: bad arguments");
    *dt = fx::min_critical_dt_bound(f->s, scheme, static_cast<cudaStream_t>(stream));
  });
}

int fx_stability_may_change(const fx_force* f, int32_t* out) {
  return guard([&] {
    if (!f || !out) throw fx::Error(FX_E_INVALID, "fx_stability_may_change: bad arguments");
    *out = fx::stability_may_change(f->s) ? 1 : 0;
  });
}

int fx_explicit_checks(fx_force* f, int32_t nan_check_interval, int32_t stable_step_check_interval,
                       int32_t allow_unstable_dt) {
  return guard([&] {
    if (!f || nan_check_interval < 0 || stable_step_check_interval < 0)
      throw fx::Error(FX_E_INVALID, "fx_explicit_checks: bad arguments");
    fx::ExplicitWork& w = work_of(f);
    w.nan_interval = nan_check_interval;
    w.stable_interval = stable_step_check_interval;
    w.allow_unstable = allow_unstable_dt != 0;
  });
}

}  // extern "C"
