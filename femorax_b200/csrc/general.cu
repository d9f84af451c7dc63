// General execution path: any stdBrick mesh (and the only path for J2 sets, whose material
// matrix differs from point to point). One thread per element evaluates the element with
// the Gauss-point physics of brick_gp.cuh and writes its 24 values to its own slots
// (slots[k * padded + e], coalesced across the warp); a second kernel gives every equation the
// sum of its slots in (element, DOF) order and adds the nodal-mass terms.
//
// This is the reference's deterministic gather scatter (src/exec/assembly.hpp:25-55,
// assembly.cpp:28-38, pair order internal_force.cpp:121-134). Built with --fmad=false, its sums
// are the reference host build's sums bit for bit.
#include <cstring>

#include "force.hpp"
#include "ssp_brick.cuh"

namespace fx {
namespace {

constexpr int kBlock = 128;

// Value k of element e in an SSPbrick per-element array ([k * P + e]).
struct Col {
  const double* p;
  int64_t ld;
  __device__ double operator[](int k) const { return p[k * ld]; }
};
struct ColW {
  double* p;
  int64_t ld;
  __device__ double& operator[](int k) const { return p[k * ld]; }
};

__device__ __forceinline__ void load_coords(const double* __restrict__ coords, const int32_t* __restrict__ node,
                                            int32_t N, int32_t P, int32_t e, double xl[3][8]) {
  for (int a = 0; a < 8; ++a) {
    const int32_t n = node[static_cast<int64_t>(a) * P + e];
    for (int d = 0; d < 3; ++d) xl[d][a] = coords[static_cast<int64_t>(d) * N + n];
  }
}

__global__ void __launch_bounds__(kBlock) k_element_apply(const double* __restrict__ coords, const int32_t* __restrict__ node,
                                                           const int32_t* __restrict__ eq, const int32_t* __restrict__ param,
                                                           const ParamGP* __restrict__ params, int32_t N, int32_t P,
                                                           int32_t count, double ks, double kd, double km, int unit_dir,
                                                           const double* __restrict__ x, double* __restrict__ slots,
                                                           const int* skip, const double* __restrict__ j2tan,
                                                           int initial, const PimySet* __restrict__ pimy,
                                                           const double* __restrict__ ptan,
                                                           const PdmySet* __restrict__ pdmy,
                                                           const double* __restrict__ dtan,
                                                           const double* __restrict__ pcs,
                                                           const double* __restrict__ dcs,
                                                           const double* __restrict__ sgeo,
                                                           const double* __restrict__ scon) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count || (skip && *skip)) return;
  const ParamGP p = params[param[e]];
  double xl[3][8], xe[24], ye[24];
  load_coords(coords, node, N, P, e, xl);
  for (int a = 0; a < 24; ++a) {
    const int32_t q = eq[static_cast<int64_t>(a) * P + e];
    if (unit_dir >= 0) xe[a] = (a % 3) == unit_dir ? 1.0 : 0.0;
    else xe[a] = q >= 0 ? x[q] : 0.0;
  }
  const OpFactors f = op_factors(p, ks, kd, km, initial != 0);
  if (p.element == 1) ssp::element_apply(p, ssp::factors(p, ks, kd, km), Col{sgeo + e, P}, Col{scon + e, P}, xe, ye);
  else if (p.kind == 1) element_apply_d(p, f, xl, xe, ye, J2PointD{&p, j2tan + e, P, initial ? f.c0 : f.cK, initial != 0});
  else if (p.kind == 2) element_apply_d(p, f, xl, xe, ye, PimyPointD{pimy + p.table, ptan + e, pcs + e, P, f.cK, f.cc});
  else if (p.kind == 3) element_apply_d(p, f, xl, xe, ye, PdmyPointD{pdmy + p.table, dtan + e, dcs + e, P, f.cK, f.c0, f.cc});
  else element_apply(p, f, xl, xe, ye);
  for (int a = 0; a < 24; ++a) slots[static_cast<int64_t>(a) * P + e] = ye[a];
}

__global__ void __launch_bounds__(kBlock) k_element_diag(const double* __restrict__ coords, const int32_t* __restrict__ node,
                                                          const int32_t* __restrict__ eq, const int32_t* __restrict__ param,
                                                          const ParamGP* __restrict__ params, int32_t N, int32_t P,
                                                          int32_t count, double ks, double kd, double km,
                                                          double* __restrict__ slots, const double* __restrict__ j2tan,
                                                          int initial, const PimySet* __restrict__ pimy,
                                                          const double* __restrict__ ptan,
                                                          const PdmySet* __restrict__ pdmy,
                                                          const double* __restrict__ dtan,
                                                          const double* __restrict__ pcs,
                                                          const double* __restrict__ dcs,
                                                          const double* __restrict__ sgeo,
                                                          const double* __restrict__ scon) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const ParamGP p = params[param[e]];
  double xl[3][8], de[24];
  int eqe[24];
  load_coords(coords, node, N, P, e, xl);
  for (int a = 0; a < 24; ++a) eqe[a] = eq[static_cast<int64_t>(a) * P + e];
  const OpFactors f = op_factors(p, ks, kd, km, initial != 0);
  if (p.element == 1)
    ssp::element_diagonal(p, ssp::factors(p, ks, kd, km), Col{sgeo + e, P}, Col{scon + e, P}, eqe, de);
  else if (p.kind == 1) element_diagonal_d(p, f, xl, eqe, de, J2PointD{&p, j2tan + e, P, initial ? f.c0 : f.cK, initial != 0});
  else if (p.kind == 2)
    element_diagonal_d(p, f, xl, eqe, de, PimyPointD{pimy + p.table, ptan + e, pcs + e, P, f.cK, f.cc});
  else if (p.kind == 3)
    element_diagonal_d(p, f, xl, eqe, de, PdmyPointD{pdmy + p.table, dtan + e, dcs + e, P, f.cK, f.c0, f.cc});
  else element_diagonal(p, f, xl, eqe, de);
  for (int a = 0; a < 24; ++a) slots[static_cast<int64_t>(a) * P + e] = de[a];
}

__global__ void __launch_bounds__(kBlock) k_element_force(const double* __restrict__ coords, const int32_t* __restrict__ node,
                                                           const int32_t* __restrict__ eq, const int32_t* __restrict__ param,
                                                           const ParamGP* __restrict__ params, int32_t N, int32_t P,
                                                           int32_t count, const double* __restrict__ u,
                                                           const double* __restrict__ v, double* __restrict__ slots,
                                                           const double* __restrict__ j2c, double* __restrict__ j2t,
                                                           double* __restrict__ j2tan, int* __restrict__ plastic,
                                                           const double* __restrict__ sgeo,
                                                           const double* __restrict__ scon) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const ParamGP p = params[param[e]];
  if (p.kind >= 2) return;  // soil materials: k_soil_points + k_soil_force
  double xl[3][8], ue[24], ve[24], fe[24];
  load_coords(coords, node, N, P, e, xl);
  for (int a = 0; a < 24; ++a) {
    const int32_t q = eq[static_cast<int64_t>(a) * P + e];
    ue[a] = q >= 0 ? u[q] : 0.0;
    ve[a] = q >= 0 ? v[q] : 0.0;
  }
  if (p.element == 1) {
    ssp::element_force(p, Col{sgeo + e, P}, Col{scon + e, P}, ue, ve, fe);
  } else if (p.kind == 1) {
    const int np = element_force_j2(p, xl, ue, ve, j2c + e, j2t + e, j2tan + e, P, fe);
    if (np) atomicAdd(plastic, np);
  } else {
    element_force(p, xl, ue, ve, fe);
  }
  for (int a = 0; a < 24; ++a) slots[static_cast<int64_t>(a) * P + e] = fe[a];
}

// Soil-material sets (PressureIndependMultiYield: kind 2, PressureDependMultiYield: kind 3), point by
// point: thread t is point gp = t / P of element e = t % P (consecutive threads, consecutive elements:
// every state value is read and written as whole lines); stress and compact tangent out. Yielding
// and failed points counted per warp.
FX_HD bool soil_point_update(const PimySet& m, const double xl[3][8], const double* ue, int gp, const double* c,
                             double* t, int64_t stride, double* sg, double* tc, bool* pl) {
  return point_update_pimy(m, xl, ue, gp, c, t, stride, sg, tc, pl);
}
FX_HD bool soil_point_update(const PdmySet& m, const double xl[3][8], const double* ue, int gp, const double* c,
                             double* t, int64_t stride, double* sg, double* tc, bool* pl) {
  return point_update_pdmy(m, xl, ue, gp, c, t, stride, sg, tc, pl);
}
FX_HD void soil_compact_D(const PimySet&, const double* t, double* D) { pimy::compact_D(t, D); }
FX_HD void soil_compact_D(const PdmySet& m, const double* t, double* D) { pdmy::compact_D(m.p, t, D); }
template <class Set, int KIND, int KTAN, int MINB>
__global__ void __launch_bounds__(128, MINB) k_soil_points(const double* __restrict__ coords, const int32_t* __restrict__ node,
                                                     const int32_t* __restrict__ eq, const int32_t* __restrict__ param,
                                                     const ParamGP* __restrict__ params, const Set* __restrict__ sets,
                                                     int32_t N, int32_t P, int32_t count, const double* __restrict__ u,
                                                     const double* __restrict__ pc, double* __restrict__ pt,
                                                     double* __restrict__ ptan, double* __restrict__ psig,
                                                     int* __restrict__ plastic, int* __restrict__ failed,
                                                     const double* __restrict__ v, double* __restrict__ psd) {
  const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  const int32_t e = static_cast<int32_t>(t % P), gp = static_cast<int32_t>(t / P);
  bool pl = false, bad = false;
  if (gp < 8 && e < count) {
    const ParamGP p = params[param[e]];
    if (p.kind == KIND) {
      double xl[3][8], ue[24], sg[6], tc[KTAN];
      load_coords(coords, node, N, P, e, xl);
      for (int a = 0; a < 24; ++a) {
        const int32_t q = eq[static_cast<int64_t>(a) * P + e];
        ue[a] = q >= 0 ? u[q] : 0.0;
      }
      bad = !soil_point_update(sets[p.table], xl, ue, gp, pc + e, pt + e, P, sg, tc, &pl);
      for (int c = 0; c < 6; ++c) psig[(static_cast<int64_t>(c) * 8 + gp) * P + e] = sg[c];
      for (int c = 0; c < KTAN; ++c) ptan[(static_cast<int64_t>(c) * 8 + gp) * P + e] = tc[c];
      if (psd && (p.betaK != 0.0 || p.betaKcomm != 0.0)) {  // the damping stress: betaK times this
        double D[36], ve[24], sd[6];                         // update's tangent + betaKcomm times the
        soil_compact_D(sets[p.table], tc, D);                // committed one
        for (int i = 0; i < 36; ++i) D[i] = p.betaK * D[i];
        if (p.betaKcomm != 0.0) add_committed_D(sets[p.table], pc + e, gp, P, p.betaKcomm, D);
        for (int a = 0; a < 24; ++a) {
          const int32_t q = eq[static_cast<int64_t>(a) * P + e];
          ve[a] = q >= 0 ? v[q] : 0.0;
        }
        damping_stress(D, xl, ve, gp, sd);
        for (int c = 0; c < 6; ++c) psd[(static_cast<int64_t>(c) * 8 + gp) * P + e] = sd[c];
      }
    }
  }
  const unsigned np = __popc(__ballot_sync(0xffffffffu, pl)), nb = __popc(__ballot_sync(0xffffffffu, bad));
  if ((threadIdx.x & 31) == 0) {
    if (np) atomicAdd(plastic, static_cast<int>(np));
    if (nb) atomicAdd(failed, static_cast<int>(nb));
  }
}

// ---- the compacted plastic corrector (src/exec/compacted_kernels.hpp:1-25, 135-181): the same point
// updates in three passes, so that the branchy, expensive corrector runs on full warps of plastic
// points only. 1. predict (one thread per point): strain, the material's predictor; a point that
// stays elastic is finished (stress, compact tangent, trial state, damping stress), a plastic one is
// flagged with its strain (and strain rate) kept; 2. compaction: the flagged points listed in point
// order (block counts, one block's scan, an ordered write), the count left on the device; 3. correct
// (one thread per listed point): the whole update from the committed state. The corrector is the
// fused path's function, so every point's results are the fused path's bits.
FX_HD bool soil_predict(const PimySet& m, const double* eps, int gp, const double* c, double* t, int64_t stride,
                        double* sg, double* tc, bool* ok) {
  return pimy::predict_compact(m.p, m.stage, pimy::Slab<const double>{c + gp * stride, 8 * stride},
                               pimy::Slab<double>{t + gp * stride, 8 * stride}, eps, sg, tc, ok);
}
FX_HD bool soil_predict(const PdmySet& m, const double* eps, int gp, const double* c, double* t, int64_t stride,
                        double* sg, double* tc, bool* ok) {
  return pdmy::predict_compact(m.p, m.stage, pimy::Slab<const double>{c + gp * stride, 8 * stride},
                               pimy::Slab<double>{t + gp * stride, 8 * stride}, eps, sg, tc, ok);
}
FX_HD bool soil_update_strain(const PimySet& m, const double* eps, int gp, const double* c, double* t, int64_t stride,
                              double* sg, double* tc, bool* pl) {
  return pimy::update_compact(m.p, m.stage, pimy::Slab<const double>{c + gp * stride, 8 * stride},
                              pimy::Slab<double>{t + gp * stride, 8 * stride}, eps, sg, tc, pl);
}
FX_HD bool soil_update_strain(const PdmySet& m, const double* eps, int gp, const double* c, double* t, int64_t stride,
                              double* sg, double* tc, bool* pl) {
  return pdmy::update_compact(m.p, m.stage, pimy::Slab<const double>{c + gp * stride, 8 * stride},
                              pimy::Slab<double>{t + gp * stride, 8 * stride}, eps, sg, tc, pl);
}

// The damping stress of a point from its strain rate: betaK times this update's tangent plus betaKcomm
// times the committed one (damping_stress's sum, the rate already formed).
template <class Set, int KTAN>
__device__ void soil_damping(const Set& m, const ParamGP& p, const double* tc, const double* pc, int gp, int64_t P,
                             const double rate[6], double sd[6]) {
  double D[36];
  soil_compact_D(m, tc, D);
  for (int i = 0; i < 36; ++i) D[i] = p.betaK * D[i];
  if (p.betaKcomm != 0.0) add_committed_D(m, pc, gp, P, p.betaKcomm, D);
  for (int a = 0; a < 6; ++a) {
    double sum = 0.0;
    for (int c = 0; c < 6; ++c) sum += D[6 * a + c] * rate[c];
    sd[a] = sum;
  }
}

template <class Set, int KIND, int KTAN, int MINB>
__global__ void __launch_bounds__(128, MINB) k_soil_predict(const double* __restrict__ coords, const int32_t* __restrict__ node,
                                                      const int32_t* __restrict__ eq, const int32_t* __restrict__ param,
                                                      const ParamGP* __restrict__ params, const Set* __restrict__ sets,
                                                      int32_t N, int32_t P, int32_t count, const double* __restrict__ u,
                                                      const double* __restrict__ pc, double* __restrict__ pt,
                                                      double* __restrict__ ptan, double* __restrict__ psig,
                                                      int* __restrict__ failed, const double* __restrict__ v,
                                                      double* __restrict__ psd, double* __restrict__ peps,
                                                      double* __restrict__ prate, int* __restrict__ flag) {
  const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  const int32_t e = static_cast<int32_t>(t % P), gp = static_cast<int32_t>(t / P);
  bool bad = false;
  if (gp < 8) {  // every point of the padded batch gets its flag (padding: 0)
    int f = 0;
    const ParamGP p = params[param[e < count ? e : 0]];
    if (e < count && p.kind == KIND) {
      double xl[3][8], ue[24], eps[6], sg[6], tc[KTAN], rate[6];
      load_coords(coords, node, N, P, e, xl);
      for (int a = 0; a < 24; ++a) {
        const int32_t q = eq[static_cast<int64_t>(a) * P + e];
        ue[a] = q >= 0 ? u[q] : 0.0;
      }
      PointShape s;
      point_shape(xl, gp, s);
      strain_of(s, ue, eps);
      const bool damped = psd && (p.betaK != 0.0 || p.betaKcomm != 0.0);
      if (damped) {
        double ve[24];
        for (int a = 0; a < 24; ++a) {
          const int32_t q = eq[static_cast<int64_t>(a) * P + e];
          ve[a] = q >= 0 ? v[q] : 0.0;
        }
        strain_of(s, ve, rate);
      }
      bool ok = true;
      if (soil_predict(sets[p.table], eps, gp, pc + e, pt + e, P, sg, tc, &ok)) {
        f = 1;
        for (int c = 0; c < 6; ++c) peps[(static_cast<int64_t>(c) * 8 + gp) * P + e] = eps[c];
        if (damped)
          for (int c = 0; c < 6; ++c) prate[(static_cast<int64_t>(c) * 8 + gp) * P + e] = rate[c];
      } else {
        bad = !ok;
        for (int c = 0; c < 6; ++c) psig[(static_cast<int64_t>(c) * 8 + gp) * P + e] = sg[c];
        for (int c = 0; c < KTAN; ++c) ptan[(static_cast<int64_t>(c) * 8 + gp) * P + e] = tc[c];
        if (damped) {
          double sd[6];
          soil_damping<Set, KTAN>(sets[p.table], p, tc, pc + e, gp, P, rate, sd);
          for (int c = 0; c < 6; ++c) psd[(static_cast<int64_t>(c) * 8 + gp) * P + e] = sd[c];
        }
      }
    }
    flag[t] = f;
  }
  const unsigned nb = __popc(__ballot_sync(0xffffffffu, bad));
  if ((threadIdx.x & 31) == 0 && nb) atomicAdd(failed, static_cast<int>(nb));
}

constexpr int kScanBlock = 256;
// Flagged entries per block of kScanBlock.
__global__ void __launch_bounds__(kScanBlock) k_flag_counts(const int* __restrict__ flag, int64_t n,
                                                            int* __restrict__ counts) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(kScanBlock) + threadIdx.x;
  const int c = __syncthreads_count(i < n && flag[i]);
  if (threadIdx.x == 0) counts[blockIdx.x] = c;
}
// One block: the exclusive prefix sums of the block counts, in place, and their total.
__global__ void __launch_bounds__(1024) k_flag_offsets(int* __restrict__ counts, int nb, int* __restrict__ total) {
  __shared__ int part[1024];
  const int per = (nb + 1023) / 1024, lo = threadIdx.x * per, hi = min(nb, lo + per);
  int sum = 0;
  for (int b = lo; b < hi; ++b) sum += counts[b];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {  // inclusive scan of the thread sums
    const int add = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  int run = part[threadIdx.x] - sum;
  for (int b = lo; b < hi; ++b) {
    const int c = counts[b];
    counts[b] = run;
    run += c;
  }
  if (threadIdx.x == 1023) *total = part[1023];
}
// The flagged entries' indices in order.
__global__ void __launch_bounds__(kScanBlock) k_flag_list(const int* __restrict__ flag, int64_t n,
                                                          const int* __restrict__ offsets, int* __restrict__ list) {
  __shared__ int warp_base[kScanBlock / 32];
  const int64_t i = blockIdx.x * static_cast<int64_t>(kScanBlock) + threadIdx.x;
  const bool f = i < n && flag[i];
  const unsigned ball = __ballot_sync(0xffffffffu, f);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) warp_base[w] = __popc(ball);
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int k = 0; k < kScanBlock / 32; ++k) {
      const int c = warp_base[k];
      warp_base[k] = run;
      run += c;
    }
  }
  __syncthreads();
  if (f) list[offsets[blockIdx.x] + warp_base[w] + __popc(ball & ((1u << lane) - 1u))] = static_cast<int>(i);
}

template <class Set, int KIND, int KTAN, int MINB>
__global__ void __launch_bounds__(128, MINB) k_soil_correct(const int32_t* __restrict__ param,
                                                      const ParamGP* __restrict__ params, const Set* __restrict__ sets,
                                                      int32_t P, const int* __restrict__ list,
                                                      const int* __restrict__ total, const double* __restrict__ pc,
                                                      double* __restrict__ pt, double* __restrict__ ptan,
                                                      double* __restrict__ psig, int* __restrict__ plastic,
                                                      int* __restrict__ failed, const double* __restrict__ peps,
                                                      const double* __restrict__ prate, double* __restrict__ psd) {
  const int n = *total;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int64_t t = list[i];
    const int32_t e = static_cast<int32_t>(t % P), gp = static_cast<int32_t>(t / P);
    const ParamGP p = params[param[e]];
    double eps[6], sg[6], tc[KTAN];
    for (int c = 0; c < 6; ++c) eps[c] = peps[(static_cast<int64_t>(c) * 8 + gp) * P + e];
    bool pl = false;
    const bool ok = soil_update_strain(sets[p.table], eps, gp, pc + e, pt + e, P, sg, tc, &pl);
    for (int c = 0; c < 6; ++c) psig[(static_cast<int64_t>(c) * 8 + gp) * P + e] = sg[c];
    for (int c = 0; c < KTAN; ++c) ptan[(static_cast<int64_t>(c) * 8 + gp) * P + e] = tc[c];
    if (psd && (p.betaK != 0.0 || p.betaKcomm != 0.0)) {
      double rate[6], sd[6];
      for (int c = 0; c < 6; ++c) rate[c] = prate[(static_cast<int64_t>(c) * 8 + gp) * P + e];
      soil_damping<Set, KTAN>(sets[p.table], p, tc, pc + e, gp, P, rate, sd);
      for (int c = 0; c < 6; ++c) psd[(static_cast<int64_t>(c) * 8 + gp) * P + e] = sd[c];
    }
    if (pl) atomicAdd(plastic, 1);
    if (!ok) atomicAdd(failed, 1);
  }
}

// ... then their elements' internal forces from the points' stresses, into the slots
__global__ void __launch_bounds__(kBlock) k_soil_force(const double* __restrict__ coords, const int32_t* __restrict__ node,
                                                        const int32_t* __restrict__ eq, const int32_t* __restrict__ param,
                                                        const ParamGP* __restrict__ params, int32_t N, int32_t P,
                                                        int32_t count, const double* __restrict__ v,
                                                        const double* __restrict__ psig,
                                                        const double* __restrict__ psd, double* __restrict__ slots,
                                                        int kind) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const ParamGP p = params[param[e]];
  if (p.kind != kind) return;
  double xl[3][8], ve[24], fe[24];
  load_coords(coords, node, N, P, e, xl);
  for (int a = 0; a < 24; ++a) {
    const int32_t q = eq[static_cast<int64_t>(a) * P + e];
    ve[a] = q >= 0 ? v[q] : 0.0;
  }
  const bool damped = psd && (p.betaK != 0.0 || p.betaKinit != 0.0 || p.betaKcomm != 0.0);
  element_force_from_stress(p, xl, ve, psig + e, damped ? psd + e : nullptr, P, fe);
  for (int a = 0; a < 24; ++a) slots[static_cast<int64_t>(a) * P + e] = fe[a];
}

// commitState of the PressureIndependMultiYield points: the scalar values of every point, the
// surfaces of the points whose last update changed them (the others' committed surfaces stand).
__global__ void __launch_bounds__(256) k_pimy_commit(const int32_t* __restrict__ param,
                                                     const ParamGP* __restrict__ params,
                                                     const PimySet* __restrict__ pimy, int32_t P, int32_t count,
                                                     double* __restrict__ pc, const double* __restrict__ pt) {
  const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  const int32_t e = static_cast<int32_t>(t % P), gp = static_cast<int32_t>(t / P);
  if (gp >= 8 || e >= count) return;
  const ParamGP& p = params[param[e]];
  if (p.kind != 2) return;
  const int64_t base = static_cast<int64_t>(gp) * P + e, ld = 8 * static_cast<int64_t>(P);
  for (int k = 0; k < pimy::S_SURF; ++k) pc[base + k * ld] = pt[base + k * ld];
  if (pt[base + pimy::S_CHANGED * ld] != 0.0) {
    const int n = pimy::nstate(pimy[p.table].p.ns);
    for (int k = pimy::S_SURF; k < n; ++k) pc[base + k * ld] = pt[base + k * ld];
  }
}

// The sum of slots[list[j]] for j in [j0, j1), in list order. The loads run ahead of the additions, 8
// list entries and then their 8 slots at a time, so that a thread waits on memory once per 8 terms
// rather than twice per term; the additions keep their order.
template <class T>
__device__ __forceinline__ T slot_sum(const int32_t* __restrict__ list, const T* __restrict__ slots, int32_t j0,
                                      int32_t j1) {
  T sum = T(0);
  int32_t j = j0;
  for (; j + 8 <= j1; j += 8) {
    int32_t idx[8];
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) idx[u] = list[j + u];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = slots[idx[u]];
#pragma unroll
    for (int u = 0; u < 8; ++u) sum += v[u];
  }
  if (j + 4 <= j1) {
    int32_t idx[4];
    T v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) idx[u] = list[j + u];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = slots[idx[u]];
#pragma unroll
    for (int u = 0; u < 4; ++u) sum += v[u];
    j += 4;
  }
  for (; j < j1; ++j) sum += slots[list[j]];
  return sum;
}

// The same sum by one warp, for equations with many slots (a tied DOF gathers whole rows of
// elements): 32 slots loaded at once, then added in list order by every lane.
template <class T>
__device__ __forceinline__ T slot_sum_warp(const int32_t* __restrict__ list, const T* __restrict__ slots, int32_t j0,
                                           int32_t j1) {
  const int lane = threadIdx.x & 31;
  T sum = T(0);
  for (int32_t b = j0; b < j1; b += 32) {
    const int32_t j = b + lane;
    const T v = j < j1 ? slots[list[j]] : T(0);
    const int cnt = j1 - b < 32 ? j1 - b : 32;
    for (int u = 0; u < cnt; ++u) sum += __shfl_sync(0xffffffffu, v, u);
  }
  return sum;
}

// y[q] = sum of q's slots in list order, then + c1 m1[q] x1[q] + c2 m2[q] x2[q] (the nodal-mass
// kernels of internal_force.cpp:368-375, 442-448, same expression, same order). The first `hblocks`
// blocks take the equations heavy[0 .. nheavy) (more than kHeavySlots slots each: tied DOFs) a warp
// each, so that their long sums start first and overlap the others; the other blocks a thread per
// equation, leaving the heavy ones.
__global__ void __launch_bounds__(256) k_gather(const int32_t* __restrict__ start, const int32_t* __restrict__ list,
                                                 const double* __restrict__ slots, int32_t neq,
                                                 const int32_t* __restrict__ heavy, int32_t nheavy, int32_t hblocks,
                                                 double c1, const double* __restrict__ m1,
                                                 const double* __restrict__ x1, double c2,
                                                 const double* __restrict__ m2, const double* __restrict__ x2,
                                                 double* __restrict__ y, const int* skip) {
  if (skip && *skip) return;
  double sum;
  int32_t q;
  if (static_cast<int32_t>(blockIdx.x) < hblocks) {
    const int32_t w = static_cast<int32_t>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (w >= nheavy) return;  // (the same for the whole warp)
    q = heavy[w];
    sum = slot_sum_warp(list, slots, start[q], start[q + 1]);
    if ((threadIdx.x & 31) != 0) return;
  } else {
    q = (static_cast<int32_t>(blockIdx.x) - hblocks) * static_cast<int32_t>(blockDim.x) + static_cast<int32_t>(threadIdx.x);
    if (q >= neq) return;
    const int32_t j0 = start[q], j1 = start[q + 1];
    if (j1 - j0 > kHeavySlots) return;
    sum = slot_sum(list, slots, j0, j1);
  }
  if (m1) sum += c1 * m1[q] * (x1 ? x1[q] : 1.0);
  if (m2) sum += c2 * m2[q] * (x2 ? x2[q] : 1.0);
  y[q] = sum;
}

// y = every equation's slot sum and nodal terms (one k_gather launch)
void gather_slots(const ForceState& s, double c1, const double* m1, const double* x1, double c2, const double* m2,
                  const double* x2, double* y, const int* skip, cudaStream_t st) {
  if (s.neq <= 0) return;
  const int32_t hblocks = static_cast<int32_t>(s.nheavy > 0 ? grid_for(32 * static_cast<int64_t>(s.nheavy), 256) : 0);
  k_gather<<<hblocks + grid_for(s.neq, 256), 256, 0, st>>>(s.gstart.ptr, s.glist.ptr, s.slots.ptr, s.neq,
                                                           s.gheavy.ptr, s.nheavy, hblocks, c1, m1, x1, c2, m2, x2, y,
                                                           skip);
}

// ---- FP32 operator (the inner solves of FP32 CG in FP64 refinement on any mesh)
// FP32 geometric factors of the Gauss points, computed once in FP64 by point_shape and rounded:
// component c < 24 (dN/dx of node c % 8 along axis c / 8) and c = 24 (dvol) of point gp of
// element e at [(c * 8 + gp) * P + e]; the shape values of the points (the same for every
// element) at nshape[gp * 8 + k].
constexpr int kGeom32 = 25;
__global__ void __launch_bounds__(kBlock) k_geom32(const double* __restrict__ coords, const int32_t* __restrict__ node,
                                                    int32_t N, int32_t P, int32_t count, float* __restrict__ geom,
                                                    float* __restrict__ nshape) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  double xl[3][8];
  load_coords(coords, node, N, P, e, xl);
  for (int gp = 0; gp < 8; ++gp) {
    PointShape s;
    point_shape(xl, gp, s);
    for (int d = 0; d < 3; ++d)
      for (int j = 0; j < 8; ++j) geom[static_cast<int64_t>(((d * 8 + j) * 8) + gp) * P + e] = static_cast<float>(s.dN[d][j]);
    geom[static_cast<int64_t>(24 * 8 + gp) * P + e] = static_cast<float>(s.dvol);
    if (e == 0)
      for (int j = 0; j < 8; ++j) nshape[gp * 8 + j] = static_cast<float>(s.N[j]);
  }
}

// y_e = K_eff,e x_e in FP32 point by point: strain B x, stress D_eff eps with the point's material
// matrix in the compact form K 1 (x) 1 + 2 G theta I_dev - 2 G thetab n (x) n (elastic sets and
// `initial`: theta = 1, thetab = 0, the elastic matrix), scaled by the stiffness factor, then
// B^T sigma dvol and the mass term, into FP32 slots.
__global__ void __launch_bounds__(kBlock) k_element_apply32(const int32_t* __restrict__ eq,
                                                             const int32_t* __restrict__ param,
                                                             const ParamGP* __restrict__ params, int32_t P,
                                                             int32_t count, double ks, double kd, double km,
                                                             const float* __restrict__ geom,
                                                             const float* __restrict__ nshape,
                                                             const float* __restrict__ x, float* __restrict__ slots,
                                                             const int* skip, const double* __restrict__ j2tan,
                                                             int initial) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count || (skip && *skip)) return;
  const ParamGP p = params[param[e]];
  const OpFactors f = op_factors(p, ks, kd, km, initial != 0);
  // the elastic tangents are one matrix: D_eff = (cK + c0 + cc) D (J2 sets carry no
  // stiffness-proportional damping, so c0 = cc = 0 there)
  const float sk = static_cast<float>(f.cK + f.c0 + f.cc), cm = static_cast<float>(f.cM);
  double Kd, Gd;
  j2_moduli(p, Kd, Gd);
  const float K = static_cast<float>(Kd), G2 = static_cast<float>(2.0 * Gd);
  const float rho = static_cast<float>(p.rho);
  const bool j2 = p.kind == 1 && !initial;
  float xe[24], ye[24];
  for (int a = 0; a < 24; ++a) {
    const int32_t q = eq[static_cast<int64_t>(a) * P + e];
    xe[a] = q >= 0 ? x[q] : 0.f;
    ye[a] = 0.f;
  }
  for (int gp = 0; gp < 8; ++gp) {
    float dN[3][8];
    for (int d = 0; d < 3; ++d)
      for (int j = 0; j < 8; ++j) dN[d][j] = geom[static_cast<int64_t>(((d * 8 + j) * 8) + gp) * P + e];
    const float dvol = geom[static_cast<int64_t>(24 * 8 + gp) * P + e];
    float eps[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int j = 0; j < 8; ++j) {
      const float dx = dN[0][j], dy = dN[1][j], dz = dN[2][j];
      const float u0 = xe[3 * j], u1 = xe[3 * j + 1], u2 = xe[3 * j + 2];
      eps[0] += dx * u0;
      eps[1] += dy * u1;
      eps[2] += dz * u2;
      eps[3] += dy * u0 + dx * u1;
      eps[4] += dz * u1 + dy * u2;
      eps[5] += dz * u0 + dx * u2;
    }
    float theta = 1.f, thetab = 0.f, n[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (j2) {
      const double* t = j2tan + e;
      theta = static_cast<float>(t[static_cast<int64_t>(0 * 8 + gp) * P]);
      thetab = static_cast<float>(t[static_cast<int64_t>(1 * 8 + gp) * P]);
      for (int c = 0; c < 6; ++c) n[c] = static_cast<float>(t[static_cast<int64_t>((2 + c) * 8 + gp) * P]);
    }
    const float tr = eps[0] + eps[1] + eps[2];
    float ne = 0.f;
    for (int c = 0; c < 6; ++c) ne += n[c] * eps[c];
    const float gt = G2 * theta, gb = G2 * thetab * ne;
    float sg[6];
    for (int c = 0; c < 3; ++c) sg[c] = sk * (K * tr + gt * (eps[c] - tr / 3.f) - gb * n[c]);
    for (int c = 3; c < 6; ++c) sg[c] = sk * (0.5f * gt * eps[c] - gb * n[c]);
    for (int c = 0; c < 6; ++c) sg[c] *= dvol;
    for (int j = 0; j < 8; ++j) {
      const float dx = dN[0][j], dy = dN[1][j], dz = dN[2][j];
      ye[3 * j] += dx * sg[0] + dy * sg[3] + dz * sg[5];
      ye[3 * j + 1] += dy * sg[1] + dx * sg[3] + dz * sg[4];
      ye[3 * j + 2] += dz * sg[2] + dy * sg[4] + dx * sg[5];
    }
    if (cm != 0.f) {
      const float* Ng = nshape + gp * 8;
      float v[3] = {0.f, 0.f, 0.f};
      if (p.mass_type == 0)
        for (int k = 0; k < 8; ++k)
          for (int q = 0; q < 3; ++q) v[q] += Ng[k] * xe[3 * k + q];
      for (int j = 0; j < 8; ++j) {
        const float t = cm * Ng[j] * dvol * rho;
        for (int q = 0; q < 3; ++q) ye[3 * j + q] += t * (p.mass_type == 0 ? v[q] : xe[3 * j + q]);
      }
    }
  }
  for (int a = 0; a < 24; ++a) slots[static_cast<int64_t>(a) * P + e] = ye[a];
}

__global__ void __launch_bounds__(256) k_gather32(const int32_t* __restrict__ start, const int32_t* __restrict__ list,
                                                   const float* __restrict__ slots, int32_t neq,
                                                   const int32_t* __restrict__ heavy, int32_t nheavy, int32_t hblocks,
                                                   double c1, const double* __restrict__ m1, double c2,
                                                   const double* __restrict__ m2, const float* __restrict__ x,
                                                   float* __restrict__ y, const int* skip) {
  if (skip && *skip) return;
  float sum;
  int32_t q;
  if (static_cast<int32_t>(blockIdx.x) < hblocks) {  // the heavy equations, a warp each (as k_gather)
    const int32_t w = static_cast<int32_t>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (w >= nheavy) return;
    q = heavy[w];
    sum = slot_sum_warp(list, slots, start[q], start[q + 1]);
    if ((threadIdx.x & 31) != 0) return;
  } else {
    q = (static_cast<int32_t>(blockIdx.x) - hblocks) * static_cast<int32_t>(blockDim.x) + static_cast<int32_t>(threadIdx.x);
    if (q >= neq) return;
    const int32_t j0 = start[q], j1 = start[q + 1];
    if (j1 - j0 > kHeavySlots) return;
    sum = slot_sum(list, slots, j0, j1);
  }
  if (m1) sum += static_cast<float>(c1 * m1[q]) * x[q];
  if (m2) sum += static_cast<float>(c2 * m2[q]) * x[q];
  y[q] = sum;
}

// ---- stable time step (StdBrick::max_omega_sq_with, std_brick.hpp:658-688; the element's
// largest omega^2 of K phi = omega^2 M phi with the lumped mass, by the cyclic Jacobi rotations of
// src/physics/common/sym_eigen.hpp; stable_dt, src/physics/explicit_stability.hpp:16-32).
// One warp per element: the lanes assemble the 24 x 24 matrix M^-1/2 K M^-1/2 in shared memory
// (two of the 64 node pairs each, the Gauss points summed in the reference's order), then apply
// the rotations in the reference's (p, q) order, lane k updating entry k of the two rows and
// columns: each entry sees the reference's operations, so omega^2 is the reference's bit for bit.
constexpr int kDtWarps = 4;

// The stable step's material matrix of point gp (contracts.hpp, stability_tangent): the elastic
// matrix for elastic and J2 sets (J2 unloads elastically); for the multi-yield soils the elastic
// moduli at the committed state (PressureIndependMultiYield::stability_tangent,
// pressure_independ_multi_yield.hpp:170-201; PressureDependMultiYield::stability_tangent,
// pressure_depend_multi_yield.hpp:203-218), or with `reference` their reference tangent
// (stability_reference: the ScaledStability bound's per-element eigenvalue).
__device__ void stability_D(const ParamGP& p, const PimySet* __restrict__ pimy, const PdmySet* __restrict__ pdmy,
                            const double* __restrict__ pcs, const double* __restrict__ dcs, int64_t P, int32_t e,
                            int gp, bool reference, double D[6][6]) {
  if (p.kind == 2) {
    const PimySet& m = pimy[p.table];
    double G = m.p.G0, K = m.p.K0;
    if (!reference) {
      const pimy::Slab<const double> c{pcs + e + static_cast<int64_t>(gp) * P, 8 * P};
      G = c[pimy::S_G];
      K = c[pimy::S_K];
      if (m.stage == 1 && c[pimy::S_E2P] == 0.0 && m.p.phi != 0.) {
        double vol = c[pimy::S_STRESS + 12];
        if (vol > 0.) vol = 0.;  // elast2Plast drops the tension first
        const double con = -(vol - m.p.p_res);
        const double scale = pow(-con / (m.p.pref - m.p.p_res), m.p.n_press);
        G *= scale;
        K *= scale;
      }
    }
    double d[36];
    pimy::elastic_D(G, K, d);
    for (int a = 0; a < 36; ++a) D[a / 6][a % 6] = d[a];
  } else if (p.kind == 3) {
    const PdmySet& m = pdmy[p.table];
    double f = 1.0;
    if (!reference && m.stage == 1) {
      const pimy::Slab<const double> c{dcs + e + static_cast<int64_t>(gp) * P, 8 * P};
      const double h = c[pdmy::S_STRESS + 12] - m.p.p_res;  // getModulusFactor of the committed stress
      f = pow(h / (m.p.pref - m.p.p_res), m.p.n_press);
      f = (1.e-10 > f) ? 1.e-10 : f;
    }
    double d[36];
    pdmy::elastic_D(m.p, f, d);
    for (int a = 0; a < 36; ++a) D[a / 6][a % 6] = d[a];
  } else {
    elastic_D(p, D);
  }
}

__device__ __forceinline__ double stable_dt_of(int scheme, const ParamGP& p, double w2) {
  if (!(w2 > 0.0)) return INFINITY;
  const double w = sqrt(w2);
  if (scheme == 0) return 2.0 / w;
  const double beta = p.betaK + p.betaKinit + p.betaKcomm;
  const double c = p.alphaM + beta * w2;
  return 4.0 / (sqrt(c * c + 4.0 * w2) + c);
}

// dt >= 0 (or +inf) as an unsigned key that orders as the values do: atomicMin over keys is the
// minimum, exactly and in any order.
__device__ __forceinline__ void min_dt(unsigned long long* out, double dt) {
  atomicMin(out, static_cast<unsigned long long>(__double_as_longlong(dt)));
}

// Per element (list[i], or i without a list): omega^2 into w2_out, its stable step into dt_out,
// the minimum step into *dt_min (each optional).
__global__ void __launch_bounds__(32 * kDtWarps)
    k_element_omega_sq(const double* __restrict__ coords, const int32_t* __restrict__ node,
                       const int32_t* __restrict__ param, const ParamGP* __restrict__ params, int32_t N, int32_t P,
                       const int32_t* __restrict__ list, int32_t n, const PimySet* __restrict__ pimy,
                       const PdmySet* __restrict__ pdmy, const double* __restrict__ pcs,
                       const double* __restrict__ dcs, const double* __restrict__ sgeo,
                       const double* __restrict__ scon, int reference, int scheme, double* __restrict__ w2_out,
                       double* __restrict__ dt_out, unsigned long long* __restrict__ dt_min) {
  __shared__ double As[kDtWarps][24][25];  // a padded row: the column updates touch 24 banks
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  double(*A)[25] = As[wp];
  for (int32_t i = blockIdx.x * kDtWarps + wp; i < n; i += gridDim.x * kDtWarps) {
    const int32_t e = list ? list[i] : i;
    const ParamGP p = params[param[e]];
    double xl[3][8], m[8];
    load_coords(coords, node, N, P, e, xl);
    double acc[2][3][3];
    if (p.element == 1) {  // SSPbrick (ssp_brick.hpp max_omega_sq_with): Kstab, then the one point
      const Col g{sgeo + e, P}, c{scon + e, P};
      for (int j = 0; j < 8; ++j) m[j] = p.rho * g[25 + j];
      double D[6][6];
      stability_D(p, pimy, pdmy, pcs, dcs, P, e, 0, reference != 0, D);
      for (int h = 0; h < 2; ++h) {
        const int q = lane + 32 * h, j = q >> 3, k = q & 7;
        double blk[3][3];
        ssp::block(g, D, j, k, blk);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) acc[h][a][b] = ssp::stab_entry(c, 3 * j + a, 3 * k + b) + blk[a][b];
      }
    } else {
      lumped_mass(p, xl, m);
      for (int h = 0; h < 2; ++h)
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) acc[h][a][c] = 0.0;
    }
    for (int gp = 0; gp < (p.element == 1 ? 0 : 8); ++gp) {
      PointShape s;
      point_shape(xl, gp, s);
      double D[6][6];
      stability_D(p, pimy, pdmy, pcs, dcs, P, e, gp, reference != 0, D);
      for (int h = 0; h < 2; ++h) {
        const int q = lane + 32 * h;
        double blk[3][3];
        block_tangent(s, D, q >> 3, q & 7, blk);
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) acc[h][a][c] += blk[a][c];
      }
    }
    bool massless = false;
    double ism[8];
    for (int j = 0; j < 8; ++j) {
      if (!(m[j] > 0.0)) massless = true;
      ism[j] = massless ? 0.0 : 1.0 / sqrt(m[j]);
    }
    double w2 = 0.0;  // a massless element sets no limit
    if (!massless) {
      for (int h = 0; h < 2; ++h) {
        const int q = lane + 32 * h, j = q >> 3, k = q & 7;
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) A[3 * j + a][3 * k + c] = acc[h][a][c] * (ism[j] * ism[k]);
      }
      __syncwarp();
      for (int sweep = 0; sweep < 60; ++sweep) {
        int stop = 0;
        if (lane == 0) {
          double off = 0.0, dg = 0.0;
          for (int r = 0; r < 24; ++r) {
            dg += A[r][r] * A[r][r];
            for (int c = r + 1; c < 24; ++c) off += A[r][c] * A[r][c];
          }
          stop = off <= 1e-30 * dg || off == 0.0;
        }
        if (__shfl_sync(0xffffffffu, stop, 0)) break;
        for (int pp = 0; pp < 23; ++pp)
          for (int qq = pp + 1; qq < 24; ++qq) {
            const double apq = A[pp][qq];
            if (apq == 0.0) continue;  // the same value in every lane
            const double theta = (A[qq][qq] - A[pp][pp]) / (2.0 * apq);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0);
            const double sn = t * c;
            __syncwarp();  // every lane has read the pivot entries
            if (lane < 24) {  // A <- A J
              const double akp = A[lane][pp], akq = A[lane][qq];
              A[lane][pp] = c * akp - sn * akq;
              A[lane][qq] = sn * akp + c * akq;
            }
            __syncwarp();
            if (lane < 24) {  // A <- J^T A
              const double apk = A[pp][lane], aqk = A[qq][lane];
              A[pp][lane] = c * apk - sn * aqk;
              A[qq][lane] = sn * apk + c * aqk;
            }
            __syncwarp();
            if (lane == 0) A[pp][qq] = A[qq][pp] = 0.0;
            __syncwarp();
          }
      }
      w2 = A[0][0];
      for (int r = 1; r < 24; ++r) w2 = A[r][r] > w2 ? A[r][r] : w2;
      __syncwarp();  // the next element reuses A
    }
    if (lane == 0) {
      if (w2_out) w2_out[i] = w2;
      const double dt = stable_dt_of(scheme, p, w2);
      if (dt_out) dt_out[i] = dt;
      if (dt_min) min_dt(dt_min, dt);
    }
  }
}

// The periodic re-check's bound (StdBrick::max_omega_sq_bound, std_brick.hpp:645-656): for the
// multi-yield soil sets the largest stability factor of the element's points times its reference
// omega^2, a hair above (never below the element's omega^2); the other sets keep w2_ref, their
// exact omega^2 (their stable tangent does not change). One thread per element of the list.
__global__ void k_element_dt_bound(const int32_t* __restrict__ param, const ParamGP* __restrict__ params, int32_t P,
                                   const int32_t* __restrict__ list, int32_t n, const PimySet* __restrict__ pimy,
                                   const PdmySet* __restrict__ pdmy, const double* __restrict__ pcs,
                                   const double* __restrict__ dcs, const double* __restrict__ w2_ref, int scheme,
                                   unsigned long long* __restrict__ dt_min) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t e = list ? list[i] : i;
  const ParamGP p = params[param[e]];
  double w2 = w2_ref[i];
  if (p.kind >= 2) {
    double sc = 0.0;
    for (int gp = 0; gp < 8; ++gp) {
      double si;
      if (p.kind == 2) {
        const PimySet& m = pimy[p.table];
        const pimy::Slab<const double> c{pcs + e + static_cast<int64_t>(gp) * P, 8 * P};
        double G = c[pimy::S_G];  // stability_scale: the stability modulus over the reference one
        if (m.stage == 1 && c[pimy::S_E2P] == 0.0 && m.p.phi != 0.) {
          double vol = c[pimy::S_STRESS + 12];
          if (vol > 0.) vol = 0.;
          const double con = -(vol - m.p.p_res);
          G *= pow(-con / (m.p.pref - m.p.p_res), m.p.n_press);
        }
        si = G / m.p.G0;
      } else {
        const PdmySet& m = pdmy[p.table];
        si = 1.0;
        if (m.stage == 1) {
          const pimy::Slab<const double> c{dcs + e + static_cast<int64_t>(gp) * P, 8 * P};
          si = pow((c[pdmy::S_STRESS + 12] - m.p.p_res) / (m.p.pref - m.p.p_res), m.p.n_press);
          si = (1.e-10 > si) ? 1.e-10 : si;
        }
      }
      sc = si > sc ? si : sc;
    }
    w2 = sc * w2 * (1.0 + 1e-12);
  }
  min_dt(dt_min, stable_dt_of(scheme, p, w2));
}

}  // namespace

void general_apply_f32(ForceState& s, const double k[3], const float* x, float* y, cudaStream_t st, const int* skip) {
  if (s.has_pimy || s.has_pdmy)
    throw Error(FX_E_UNSUPPORTED, "the FP32 operator has no multi-yield soil tangent form");
  if (s.has_ssp) throw Error(FX_E_UNSUPPORTED, "the FP32 operator has no SSPbrick form");
  if (s.count > 0 && s.geom32.n == 0) {  // the FP32 geometric factors, once
    s.geom32.alloc(static_cast<size_t>(kGeom32) * 8 * s.P);
    s.nshape32.alloc(64);
    s.slots32.alloc(static_cast<size_t>(24) * s.P);
    k_geom32<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.coords.ptr, s.node.ptr, s.N, s.P, s.count, s.geom32.ptr,
                                                           s.nshape32.ptr);
    FX_LAUNCH_CHECK("geom32");
  }
  if (s.count > 0)
    k_element_apply32<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.eq.ptr, s.param.ptr, s.params.ptr, s.P, s.count,
                                                                     k[0], k[1], k[2], s.geom32.ptr, s.nshape32.ptr, x,
                                                                     s.slots32.ptr, skip, s.j2_tan.ptr, s.initial);
  FX_LAUNCH_CHECK("element_apply32");
  const double* m1 = (k[2] != 0.0 && s.has_nodal_mass) ? s.nodal_mass.ptr : nullptr;
  const double* m2 = (k[1] != 0.0 && s.has_nodal_alpha) ? s.nodal_alpha_mass.ptr : nullptr;
  if (s.neq > 0)
    k_gather32<<<(s.nheavy > 0 ? grid_for(32 * static_cast<int64_t>(s.nheavy), 256) : 0) + grid_for(s.neq, 256), 256, 0,
                 st>>>(s.gstart.ptr, s.glist.ptr, s.slots32.ptr, s.neq, s.gheavy.ptr, s.nheavy,
                       static_cast<int32_t>(s.nheavy > 0 ? grid_for(32 * static_cast<int64_t>(s.nheavy), 256) : 0),
                       k[2], m1, k[1], m2, x, y, skip);
  FX_LAUNCH_CHECK("slot_gather32");
}

// ModifiedNewton -initial with PressureIndependMultiYield is refused, as the reference refuses it
// (src/io/support.cpp:120-127): OpenSees scales that material's initial tangent per point at the
// switch to the plastic stage, and that scaled tangent is not kept.
static void refuse_pimy_initial(const ForceState& s) {
  if (s.initial && s.has_pimy)
    throw Error(FX_E_UNSUPPORTED, "ModifiedNewton -initial (the initial stiffness in the operator) with "
                                  "PressureIndependMultiYield");
}

void general_gather(ForceState& s, const double k[3], const double* x, double* y, cudaStream_t st, const int* skip) {
  const double* m1 = (k[2] != 0.0 && s.has_nodal_mass) ? s.nodal_mass.ptr : nullptr;
  const double* m2 = (k[1] != 0.0 && s.has_nodal_alpha) ? s.nodal_alpha_mass.ptr : nullptr;
  if (s.neq > 0)
    gather_slots(s, k[2], m1, x, k[1], m2, x, y, skip, st);
  FX_LAUNCH_CHECK("slot_gather");
}

void general_force_gather(ForceState& s, const double* v, double* f, cudaStream_t st) {
  const double* m2 = s.has_nodal_alpha ? s.nodal_alpha_mass.ptr : nullptr;
  if (s.neq > 0)
    gather_slots(s, 0.0, nullptr, nullptr, 1.0, m2, v, f, nullptr, st);
  FX_LAUNCH_CHECK("slot_gather");
}

void general_apply(ForceState& s, const double k[3], const double* x, double* y, cudaStream_t st, const int* skip) {
  refuse_pimy_initial(s);
  if (general_fast_applies(s)) return general_apply_fast(s, k, x, y, st, skip);
  if (s.count > 0)
    k_element_apply<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                                   s.params.ptr, s.N, s.P, s.count, k[0], k[1], k[2],
                                                                   -1, x, s.slots.ptr, skip, s.j2_tan.ptr, s.initial,
                                                                   s.pimy_dev.ptr, s.pimy_tan.ptr, s.pdmy_dev.ptr,
                                                                   s.pdmy_tan.ptr, s.pimy_committed.ptr,
                                                                   s.pdmy_committed.ptr, s.ssp_geo.ptr, s.ssp_con.ptr);
  FX_LAUNCH_CHECK("element_apply");
  const double* m1 = (k[2] != 0.0 && s.has_nodal_mass) ? s.nodal_mass.ptr : nullptr;
  const double* m2 = (k[1] != 0.0 && s.has_nodal_alpha) ? s.nodal_alpha_mass.ptr : nullptr;
  if (s.neq > 0)
    gather_slots(s, k[2], m1, x, k[1], m2, x, y, skip, st);
  FX_LAUNCH_CHECK("slot_gather");
}

void general_diagonal(ForceState& s, const double k[3], double* d, cudaStream_t st) {
  refuse_pimy_initial(s);
  if (s.count > 0)
    k_element_diag<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                                  s.params.ptr, s.N, s.P, s.count, k[0], k[1], k[2],
                                                                  s.slots.ptr, s.j2_tan.ptr, s.initial,
                                                                  s.pimy_dev.ptr, s.pimy_tan.ptr, s.pdmy_dev.ptr,
                                                                  s.pdmy_tan.ptr, s.pimy_committed.ptr,
                                                                  s.pdmy_committed.ptr, s.ssp_geo.ptr, s.ssp_con.ptr);
  FX_LAUNCH_CHECK("element_diagonal");
  const double* m1 = (k[2] != 0.0 && s.has_nodal_mass) ? s.nodal_mass.ptr : nullptr;
  const double* m2 = (k[1] != 0.0 && s.has_nodal_alpha) ? s.nodal_alpha_mass.ptr : nullptr;
  if (s.neq > 0)
    gather_slots(s, k[2], m1, nullptr, k[1], m2, nullptr, d, nullptr, st);
  FX_LAUNCH_CHECK("slot_gather");
}

// The compacted corrector's passes for the points of one soil kind (the per-point buffers allocated
// at the first call: strain and strain rate, 48 bytes per point each, a flag and a list entry).
template <class Set, int KIND, int KTAN, int MINB>
void soil_points_compacted(ForceState& s, const Set* sets, const double* u, const double* v, const double* pc,
                           double* pt, double* ptan, double* psig, cudaStream_t st) {
  const int64_t points = static_cast<int64_t>(8) * s.P;
  const unsigned nb = static_cast<unsigned>((points + kScanBlock - 1) / kScanBlock);
  if (s.soil_eps.n < static_cast<size_t>(6 * points)) {
    s.soil_eps.alloc(static_cast<size_t>(6 * points));
    if (s.soil_sd.n) s.soil_rate.alloc(static_cast<size_t>(6 * points));
    s.soil_flag.alloc(static_cast<size_t>(points));
    s.soil_list.alloc(static_cast<size_t>(points));
    s.soil_counts.alloc(nb);
    s.soil_total.alloc(1);
  }
  k_soil_predict<Set, KIND, KTAN, MINB><<<static_cast<unsigned>((points + 127) / 128), 128, 0, st>>>(
      s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr, s.params.ptr, sets, s.N, s.P, s.count, u, pc, pt, ptan, psig,
      s.pimy_failed.ptr, v, s.soil_sd.ptr, s.soil_eps.ptr, s.soil_rate.ptr, s.soil_flag.ptr);
  FX_LAUNCH_CHECK("soil_predict");
  k_flag_counts<<<nb, kScanBlock, 0, st>>>(s.soil_flag.ptr, points, s.soil_counts.ptr);
  k_flag_offsets<<<1, 1024, 0, st>>>(s.soil_counts.ptr, static_cast<int>(nb), s.soil_total.ptr);
  k_flag_list<<<nb, kScanBlock, 0, st>>>(s.soil_flag.ptr, points, s.soil_counts.ptr, s.soil_list.ptr);
  FX_LAUNCH_CHECK("soil_compaction");
  const unsigned cg = static_cast<unsigned>(std::min<int64_t>((points + 127) / 128, static_cast<int64_t>(num_sms()) * 8));
  k_soil_correct<Set, KIND, KTAN, MINB><<<cg, 128, 0, st>>>(s.param.ptr, s.params.ptr, sets, s.P, s.soil_list.ptr,
                                                             s.soil_total.ptr, pc, pt, ptan, psig, s.plastic_dev.ptr,
                                                             s.pimy_failed.ptr, s.soil_eps.ptr, s.soil_rate.ptr,
                                                             s.soil_sd.ptr);
  FX_LAUNCH_CHECK("soil_correct");
}

void general_force(ForceState& s, const double* u, const double* v, double* f, cudaStream_t st) {
  if (general_fast_applies(s)) return general_force_fast(s, u, v, f, st);
  if (s.has_j2 || s.has_pimy || s.has_pdmy) FX_CUDA(cudaMemsetAsync(s.plastic_dev.ptr, 0, sizeof(int), st));
  if (s.count > 0)
    k_element_force<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                                   s.params.ptr, s.N, s.P, s.count, u, v, s.slots.ptr,
                                                                   s.j2_committed.ptr, s.j2_trial.ptr, s.j2_tan.ptr,
                                                                   s.plastic_dev.ptr, s.ssp_geo.ptr, s.ssp_con.ptr);
  FX_LAUNCH_CHECK("element_force");
  const int64_t points = static_cast<int64_t>(8) * s.P;
  if (s.has_pimy && s.count > 0 && s.compact_soil) {
    soil_points_compacted<PimySet, 2, pimy::kTan, 6>(s, s.pimy_dev.ptr, u, v, s.pimy_committed.ptr, s.pimy_trial.ptr,
                                                      s.pimy_tan.ptr, s.pimy_sig.ptr, st);
    k_soil_force<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                               s.params.ptr, s.N, s.P, s.count, v, s.pimy_sig.ptr,
                                                               s.soil_sd.ptr, s.slots.ptr, 2);
    FX_LAUNCH_CHECK("pimy_force");
  } else if (s.has_pimy && s.count > 0) {
    k_soil_points<PimySet, 2, pimy::kTan, 6><<<static_cast<unsigned>((points + 127) / 128), 128, 0, st>>>(
        s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr, s.params.ptr, s.pimy_dev.ptr, s.N, s.P, s.count, u,
        s.pimy_committed.ptr, s.pimy_trial.ptr, s.pimy_tan.ptr, s.pimy_sig.ptr, s.plastic_dev.ptr, s.pimy_failed.ptr,
        v, s.soil_sd.ptr);
    FX_LAUNCH_CHECK("pimy_points");
    k_soil_force<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                               s.params.ptr, s.N, s.P, s.count, v, s.pimy_sig.ptr,
                                                               s.soil_sd.ptr, s.slots.ptr, 2);
    FX_LAUNCH_CHECK("pimy_force");
  }
  if (s.has_pdmy && s.count > 0 && s.compact_soil) {
    soil_points_compacted<PdmySet, 3, pdmy::kTan, 4>(s, s.pdmy_dev.ptr, u, v, s.pdmy_committed.ptr, s.pdmy_trial.ptr,
                                                      s.pdmy_tan.ptr, s.pdmy_sig.ptr, st);
    k_soil_force<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                               s.params.ptr, s.N, s.P, s.count, v, s.pdmy_sig.ptr,
                                                               s.soil_sd.ptr, s.slots.ptr, 3);
    FX_LAUNCH_CHECK("pdmy_force");
  } else if (s.has_pdmy && s.count > 0) {
    k_soil_points<PdmySet, 3, pdmy::kTan, 4><<<static_cast<unsigned>((points + 127) / 128), 128, 0, st>>>(
        s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr, s.params.ptr, s.pdmy_dev.ptr, s.N, s.P, s.count, u,
        s.pdmy_committed.ptr, s.pdmy_trial.ptr, s.pdmy_tan.ptr, s.pdmy_sig.ptr, s.plastic_dev.ptr, s.pimy_failed.ptr,
        v, s.soil_sd.ptr);
    FX_LAUNCH_CHECK("pdmy_points");
    k_soil_force<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                               s.params.ptr, s.N, s.P, s.count, v, s.pdmy_sig.ptr,
                                                               s.soil_sd.ptr, s.slots.ptr, 3);
    FX_LAUNCH_CHECK("pdmy_force");
  }
  const double* m2 = s.has_nodal_alpha ? s.nodal_alpha_mass.ptr : nullptr;
  if (s.neq > 0)
    gather_slots(s, 0.0, nullptr, nullptr, 1.0, m2, v, f, nullptr, st);
  FX_LAUNCH_CHECK("slot_gather");
}

void pimy_commit(ForceState& s, cudaStream_t st) {
  if (s.has_pdmy)  // written in full: the whole trial state
    FX_CUDA(cudaMemcpyAsync(s.pdmy_committed.ptr, s.pdmy_trial.ptr, s.pdmy_committed.bytes(), cudaMemcpyDeviceToDevice,
                            st));
  if (!s.has_pimy || s.count == 0) return;
  const int64_t points = static_cast<int64_t>(8) * s.P;
  k_pimy_commit<<<static_cast<unsigned>((points + 255) / 256), 256, 0, st>>>(
      s.param.ptr, s.params.ptr, s.pimy_dev.ptr, s.P, s.count, s.pimy_committed.ptr, s.pimy_trial.ptr);
  FX_LAUNCH_CHECK("pimy_commit");
}

// M r_dir: the operator with k = (0, 0, 1) on the rigid unit translation at every element DOF,
// then the free nodal masses in that direction (internal_force.cpp:601-626).
__global__ void k_ground_nodal(const double* __restrict__ nm, const int8_t* __restrict__ dof, int32_t neq, int dir,
                               double* __restrict__ y) {
  const int32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= neq) return;
  if (dof[q] == dir) y[q] += nm[q];
}

void general_mass_times_ground(ForceState& s, int dir, double* y, cudaStream_t st) {
  if (s.count > 0)
    k_element_apply<<<grid_for(s.count, kBlock), kBlock, 0, st>>>(s.coords.ptr, s.node.ptr, s.eq.ptr, s.param.ptr,
                                                                   s.params.ptr, s.N, s.P, s.count, 0.0, 0.0, 1.0, dir,
                                                                   nullptr, s.slots.ptr, nullptr, s.j2_tan.ptr, 0,
                                                                   s.pimy_dev.ptr, s.pimy_tan.ptr, s.pdmy_dev.ptr,
                                                                   s.pdmy_tan.ptr, s.pimy_committed.ptr,
                                                                   s.pdmy_committed.ptr, s.ssp_geo.ptr, s.ssp_con.ptr);
  FX_LAUNCH_CHECK("element_apply_unit");
  if (s.neq > 0)
    gather_slots(s, 0.0, nullptr, nullptr, 0.0, nullptr, nullptr, y, nullptr, st);
  if (s.has_nodal_mass && s.neq > 0)
    k_ground_nodal<<<grid_for(s.neq, 256), 256, 0, st>>>(s.nodal_mass.ptr, s.eq_dof.ptr, s.neq, dir, y);
  FX_LAUNCH_CHECK("ground_mass");
}


namespace {
// SSPbrick sets: one thread per element computes its geometry record and stabilization constants
// (ssp::element_setup) from the material's initial tangent (C1 = D00, C2 = D01, C3 = D33).
__global__ void k_ssp_setup(const double* __restrict__ coords, const int32_t* __restrict__ node,
                            const int32_t* __restrict__ param, const ParamGP* __restrict__ params, int32_t N,
                            int32_t P, int32_t count, double* __restrict__ geo, double* __restrict__ con) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const ParamGP p = params[param[e]];
  if (p.element != 1) return;
  double xl[3][8], D[6][6];
  load_coords(coords, node, N, P, e, xl);
  elastic_D(p, D);
  ssp::element_setup(xl, D[0][0], D[0][1], D[3][3], ColW{geo + e, P}, ColW{con + e, P});
}
}  // namespace

void ssp_setup(ForceState& s) {
  s.ssp_geo.alloc(static_cast<size_t>(ssp::kGeo) * std::max(s.P, 1));
  s.ssp_con.alloc(static_cast<size_t>(ssp::kCon) * std::max(s.P, 1));
  FX_CUDA(cudaMemset(s.ssp_geo.ptr, 0, s.ssp_geo.bytes()));
  FX_CUDA(cudaMemset(s.ssp_con.ptr, 0, s.ssp_con.bytes()));
  if (s.count > 0)
    k_ssp_setup<<<grid_for(s.count, 64), 64>>>(s.coords.ptr, s.node.ptr, s.param.ptr, s.params.ptr, s.N, s.P,
                                               s.count, s.ssp_geo.ptr, s.ssp_con.ptr);
  FX_LAUNCH_CHECK("ssp_setup");
  FX_CUDA(cudaDeviceSynchronize());
}

namespace {
unsigned long long* dt_min_slot(ForceState& s) {
  if (s.dt_key.n == 0) s.dt_key.alloc(1);
  return s.dt_key.ptr;
}
double read_dt_min(ForceState& s, cudaStream_t st) {
  unsigned long long key = 0;
  FX_CUDA(cudaMemcpyAsync(&key, s.dt_key.ptr, sizeof(key), cudaMemcpyDeviceToHost, st));
  FX_CUDA(cudaStreamSynchronize(st));
  double dt;
  static_assert(sizeof(dt) == sizeof(key), "64-bit keys");
  std::memcpy(&dt, &key, sizeof(dt));
  return dt;
}
void reset_dt_min(ForceState& s, cudaStream_t st) {
  const double inf = INFINITY;
  unsigned long long key;
  std::memcpy(&key, &inf, sizeof(key));
  FX_CUDA(cudaMemcpyAsync(dt_min_slot(s), &key, sizeof(key), cudaMemcpyHostToDevice, st));
}
unsigned dt_grid(int32_t n) {
  const int64_t blocks = (static_cast<int64_t>(n) + kDtWarps - 1) / kDtWarps;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(blocks, static_cast<int64_t>(num_sms()) * 16)));
}
}  // namespace

double general_min_critical_dt(ForceState& s, int scheme, const int32_t* list, int32_t n, double* dt_out,
                               cudaStream_t st) {
  reset_dt_min(s, st);
  if (n > 0)
    k_element_omega_sq<<<dt_grid(n), 32 * kDtWarps, 0, st>>>(
        s.coords.ptr, s.node.ptr, s.param.ptr, s.params.ptr, s.N, s.P, list, n, s.pimy_dev.ptr, s.pdmy_dev.ptr,
        s.pimy_committed.ptr, s.pdmy_committed.ptr, s.ssp_geo.ptr, s.ssp_con.ptr, 0, scheme, nullptr, dt_out,
        s.dt_key.ptr);
  FX_LAUNCH_CHECK("element_critical_dt");
  return read_dt_min(s, st);
}

bool stability_may_change(const ForceState& s) { return s.has_pimy || s.has_pdmy; }

void prepare_stability_bounds(ForceState& s, cudaStream_t st) {
  const int32_t n = s.count;
  if (s.w2_ref.n < static_cast<size_t>(std::max(n, 1))) s.w2_ref.alloc(static_cast<size_t>(std::max(n, 1)));
  if (n > 0)
    k_element_omega_sq<<<dt_grid(n), 32 * kDtWarps, 0, st>>>(
        s.coords.ptr, s.node.ptr, s.param.ptr, s.params.ptr, s.N, s.P, nullptr, n, s.pimy_dev.ptr, s.pdmy_dev.ptr,
        s.pimy_committed.ptr, s.pdmy_committed.ptr, s.ssp_geo.ptr, s.ssp_con.ptr, 1, 0, s.w2_ref.ptr, nullptr,
        nullptr);
  FX_LAUNCH_CHECK("element_reference_omega_sq");
  s.bounds_ready = true;
}

double min_critical_dt_bound(ForceState& s, int scheme, cudaStream_t st) {
  if (!s.bounds_ready) throw Error(FX_E_INVALID, "the stability bounds are not prepared (fx_stability_prepare)");
  reset_dt_min(s, st);
  if (s.count > 0)
    k_element_dt_bound<<<grid_for(s.count, 256), 256, 0, st>>>(s.param.ptr, s.params.ptr, s.P, nullptr, s.count,
                                                                s.pimy_dev.ptr, s.pdmy_dev.ptr, s.pimy_committed.ptr,
                                                                s.pdmy_committed.ptr, s.w2_ref.ptr, scheme,
                                                                s.dt_key.ptr);
  FX_LAUNCH_CHECK("element_dt_bound");
  return read_dt_min(s, st);
}

}  // namespace fx
