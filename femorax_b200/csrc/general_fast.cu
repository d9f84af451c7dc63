// Fast form of the Gauss-point path for elastic stdBrick sets (the general meshes: distorted
// bricks, equalDOF ties, per-element materials): eight threads per element, one per Gauss point,
// built with fused multiply-adds. The eight threads of an element stage its corner coordinates and
// values in shared memory (thread a loads corner a), each evaluates its point (shape functions,
// strain, stress, node forces, mass) with the physics of brick_gp.cuh, and the points' 24 values
// are summed over the points in a fixed order (point 0 to 7) by thread j for corner j, which writes
// the corner's three slots. The slot gather of general.cu then sums every equation in (element,
// DOF) order, as in the exact form, so the result is deterministic for any launch; it differs from
// the reference's arithmetic only by rounding (fused multiply-adds, per-point partial sums): within
// 1e-12 of the largest entry. The exact form (general.cu, no contraction) stays the parity mode.
#include "force.hpp"

namespace fx {
namespace {

constexpr int kEl = 16;                 // elements per block
constexpr int kThreads = 8 * kEl;       // one thread per Gauss point
constexpr int kPart = 25;               // a point's 24 values, padded

struct Stage {
  double xl[kEl][3][8];
  double ve[kEl][24];
  double ue[kEl][24];  // the force: u (ve holds v)
  double part[kEl][8][kPart];
};

// Corner a of element e: its coordinates and its values of one or two vectors into the stage.
__device__ __forceinline__ void load_corner(const double* __restrict__ coords, const int32_t* __restrict__ node,
                                            const int32_t* __restrict__ eq, int32_t N, int32_t P, int32_t e, int a,
                                            const double* __restrict__ x, const double* __restrict__ x2,
                                            double (*xl)[8], double* xe, double* xe2) {
  const int32_t n = node[static_cast<int64_t>(a) * P + e];
  for (int d = 0; d < 3; ++d) xl[d][a] = coords[static_cast<int64_t>(d) * N + n];
  for (int d = 0; d < 3; ++d) {
    const int32_t q = eq[static_cast<int64_t>(3 * a + d) * P + e];
    xe[3 * a + d] = q >= 0 ? x[q] : 0.0;
    if (x2) xe2[3 * a + d] = q >= 0 ? x2[q] : 0.0;
  }
}

// Corner j's three values summed over the points, into its slots.
__device__ __forceinline__ void emit_corner(const double (*part)[kPart], int j, int32_t P, int32_t e,
                                            double* __restrict__ slots) {
  for (int q = 0; q < 3; ++q) {
    double s = part[0][3 * j + q];
    for (int g = 1; g < 8; ++g) s += part[g][3 * j + q];
    slots[static_cast<int64_t>(3 * j + q) * P + e] = s;
  }
}

// y_e = K_eff,e x_e (element_operator_apply, element_operator.hpp:82-130) for elastic sets.
__global__ void __launch_bounds__(kThreads, 4) k_apply_fast(const double* __restrict__ coords,
                                                         const int32_t* __restrict__ node,
                                                         const int32_t* __restrict__ eq,
                                                         const int32_t* __restrict__ param,
                                                         const ParamGP* __restrict__ params, int32_t N, int32_t P,
                                                         int32_t count, double ks, double kd, double km,
                                                         const double* __restrict__ x, double* __restrict__ slots,
                                                         const int* skip) {
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char raw[];
  Stage& S = *reinterpret_cast<Stage*>(raw);
  const int le = threadIdx.x >> 3, gp = threadIdx.x & 7;
  const int32_t e = blockIdx.x * kEl + le;
  const bool ok = e < count;
  if (ok) load_corner(coords, node, eq, N, P, e, gp, x, nullptr, S.xl[le], S.ve[le], nullptr);
  __syncthreads();
  if (ok) {
    const ParamGP& p = params[param[e]];
    const OpFactors f = op_factors(p, ks, kd, km);
    PointShape s;
    point_shape(S.xl[le], gp, s);
    const double* xe = S.ve[le];
    double ep[6], sg[6];
    strain_of(s, xe, ep);
    // elastic sets: D_eff = (cK + c0 + cc) D, D the isotropic matrix
    elastic_stress(p, ep, sg);
    const double c = f.cK + f.c0 + f.cc;
    for (int a = 0; a < 6; ++a) sg[a] *= c;
    double vg[3] = {0.0, 0.0, 0.0};
    if (f.cM != 0.0 && p.mass_type == 0)
      for (int k = 0; k < 8; ++k)
        for (int q = 0; q < 3; ++q) vg[q] += s.N[k] * xe[3 * k + q];
    double* out = S.part[le][gp];
    for (int j = 0; j < 8; ++j) {
      double fj[3];
      node_force(s, sg, j, fj);
      if (f.cM != 0.0) {
        const double t = f.cM * (s.N[j] * s.dvol * p.rho);
        for (int q = 0; q < 3; ++q) fj[q] += t * (p.mass_type == 0 ? vg[q] : xe[3 * j + q]);
      }
      for (int q = 0; q < 3; ++q) out[3 * j + q] = fj[q];
    }
  }
  __syncthreads();
  if (ok) emit_corner(S.part[le], gp, P, e, slots);
}

// f_e = internal force + Rayleigh damping forces (StdBrick::compute_with, std_brick.hpp:492-543)
// for elastic sets: per point the stress and damping stress node forces, minus the body force,
// plus the alphaM mass force.
__global__ void __launch_bounds__(kThreads, 4) k_force_fast(const double* __restrict__ coords,
                                                         const int32_t* __restrict__ node,
                                                         const int32_t* __restrict__ eq,
                                                         const int32_t* __restrict__ param,
                                                         const ParamGP* __restrict__ params, int32_t N, int32_t P,
                                                         int32_t count, const double* __restrict__ u,
                                                         const double* __restrict__ v, double* __restrict__ slots) {
  extern __shared__ __align__(16) unsigned char raw[];
  Stage& S = *reinterpret_cast<Stage*>(raw);
  const int le = threadIdx.x >> 3, gp = threadIdx.x & 7;
  const int32_t e = blockIdx.x * kEl + le;
  const bool ok = e < count;
  if (ok) load_corner(coords, node, eq, N, P, e, gp, u, v, S.xl[le], S.ue[le], S.ve[le]);
  __syncthreads();
  if (ok) {
    const ParamGP& p = params[param[e]];
    PointShape s;
    point_shape(S.xl[le], gp, s);
    const double* ue = S.ue[le];
    const double* ve = S.ve[le];
    double ep[6], sg[6], ds[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    strain_of(s, ue, ep);
    elastic_stress(p, ep, sg);
    const double beta = p.betaK + p.betaKinit + p.betaKcomm;
    if (beta != 0.0) {  // the elastic tangent is the current, initial and committed one
      double rate[6];
      strain_of(s, ve, rate);
      elastic_stress(p, rate, ds);
      for (int a = 0; a < 6; ++a) ds[a] *= beta;
    }
    double vg[3] = {0.0, 0.0, 0.0};
    if (p.alphaM != 0.0 && p.mass_type == 0)
      for (int k = 0; k < 8; ++k)
        for (int q = 0; q < 3; ++q) vg[q] += s.N[k] * ve[3 * k + q];
    double* out = S.part[le][gp];
    for (int j = 0; j < 8; ++j) {
      double r[3], dj[3] = {0.0, 0.0, 0.0};
      node_force(s, sg, j, r);
      if (beta != 0.0) node_force(s, ds, j, dj);
      const double t = s.N[j] * s.dvol;
      for (int q = 0; q < 3; ++q) {
        double fq = r[q] - t * p.b[q] + dj[q];
        if (p.alphaM != 0.0) fq += p.alphaM * (t * p.rho) * (p.mass_type == 0 ? vg[q] : ve[3 * j + q]);
        out[3 * j + q] = fq;
      }
    }
  }
  __syncthreads();
  if (ok) emit_corner(S.part[le], gp, P, e, slots);
}

unsigned fast_grid(int32_t count) { return static_cast<unsigned>((count + kEl - 1) / kEl); }

}  // namespace

bool general_fast_applies(const ForceState& s) {
  if (!s.fast_general) return false;
  for (const auto& p : s.params_h)
    if (p.kind != 0 || p.element != 0) return false;
  return true;
}

// the kernels' shared-memory limit, set once (thread-safe)
void fast_attributes() {
  static const bool once = [] {
    FX_CUDA(cudaFuncSetAttribute(k_apply_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, sizeof(Stage)));
    FX_CUDA(cudaFuncSetAttribute(k_force_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, sizeof(Stage)));
    return true;
  }();
  (void)once;
}

void general_apply_fast(ForceState& s, const double k[3], const double* x, double* y, cudaStream_t st, const int* skip) {
  fast_attributes();
  if (s.count > 0)
    k_apply_fast<<<fast_grid(s.count), kThreads, sizeof(Stage), st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                                      s.params.ptr, s.N, s.P, s.count, k[0], k[1], k[2],
                                                                      x, s.slots.ptr, skip);
  FX_LAUNCH_CHECK("element_apply_fast");
  general_gather(s, k, x, y, st, skip);
}

void general_force_fast(ForceState& s, const double* u, const double* v, double* f, cudaStream_t st) {
  fast_attributes();
  if (s.count > 0)
    k_force_fast<<<fast_grid(s.count), kThreads, sizeof(Stage), st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                                      s.params.ptr, s.N, s.P, s.count, u, v,
                                                                      s.slots.ptr);
  FX_LAUNCH_CHECK("element_force_fast");
  general_force_gather(s, v, f, st);
}

}  // namespace fx
