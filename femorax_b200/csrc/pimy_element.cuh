// stdBrick with PressureIndependMultiYield points (the reference's StdBrick<PressureIndependMultiYield<NS>>,
// src/physics/elements/std_brick.hpp:398-540, with the material of pimy.cuh): the internal force
// through the material update of every Gauss point, and the operator's material matrix from the
// compact tangents that update stored. Point gp of element e keeps value k of its state at
// [(k * 8 + gp) * P + e] and value c of its compact tangent at [(c * 8 + gp) * P + e].
#pragma once

#include "brick_gp.cuh"
#include "pdmy.cuh"
#include "pimy.cuh"

namespace fx {

// A parameter set's material (ParamGP::table indexes the table) and its stage.
struct PimySet {
  pimy::Params p;
  int stage;  // 0 elastic, 1 plastic (updateMaterialStage)
};

// A parameter set's PressureDependMultiYield material (ParamGP::table indexes its table) and stage.
struct PdmySet {
  pdmy::Params p;
  int stage;
};

// The update of point gp of element e (the reference's point_update_shape without stiffness
// damping): strain at the point from the element's displacements, the material update from the
// committed state to the trial one; the stress and the compact tangent out. Returns the update's ok.
FX_HD bool point_update_pimy(const PimySet& m, const double xl[3][8], const double* ue, int gp,
                             const double* committed, double* trial, int64_t stride, double sg[6],
                             double t[pimy::kTan], bool* plastic) {
  PointShape s;
  point_shape(xl, gp, s);
  double e[6];
  strain_of(s, ue, e);
  return pimy::update_compact(m.p, m.stage, pimy::Slab<const double>{committed + gp * stride, 8 * stride},
                              pimy::Slab<double>{trial + gp * stride, 8 * stride}, e, sg, t, plastic);
}

// The same for a PressureDependMultiYield point (its trial state written in full).
FX_HD bool point_update_pdmy(const PdmySet& m, const double xl[3][8], const double* ue, int gp,
                             const double* committed, double* trial, int64_t stride, double sg[6],
                             double t[pdmy::kTan], bool* plastic) {
  PointShape s;
  point_shape(xl, gp, s);
  double e[6];
  strain_of(s, ue, e);
  return pdmy::update_compact(m.p, m.stage, pimy::Slab<const double>{committed + gp * stride, 8 * stride},
                              pimy::Slab<double>{trial + gp * stride, 8 * stride}, e, sg, t, plastic);
}

// Out of line on the device: only betaKcomm sets form the committed tangent, and inlined it would take
// registers from the common path of the kernels that call it.
#if defined(__CUDACC__)
#define FX_HD_COLD inline __host__ __device__ __noinline__
#else
#define FX_HD_COLD inline
#endif

// M[6 i + j] += f Dc[6 i + j], Dc the tangent at the committed state of point gp (betaKcomm
// damping) as the material returns it (the reference's Mat::committed_tangent; not mirrored).
FX_HD_COLD void add_committed_D(const PimySet& m, const double* committed, int gp, int64_t stride, double f,
                                double* M) {
  double t[pimy::kTan], Dc[36];
  pimy::committed_compact(m.p, m.stage, pimy::Slab<const double>{committed + gp * stride, 8 * stride}, t);
  pimy::compact_D(t, Dc);
  for (int i = 0; i < 36; ++i) M[i] += f * Dc[i];
}
FX_HD_COLD void add_committed_D(const PdmySet& m, const double* committed, int gp, int64_t stride, double f,
                                double* M) {
  double t[pdmy::kTan], Dc[36];
  pdmy::committed_compact(m.p, m.stage, pimy::Slab<const double>{committed + gp * stride, 8 * stride}, t);
  pdmy::compact_D(m.p, t, Dc);
  for (int i = 0; i < 36; ++i) M[i] += f * Dc[i];
}

// Stiffness-proportional damping stress of a point (the reference's point_update_shape,
// src/physics/elements/std_brick.hpp:419-434, without betaKinit): sd[a] = sum_c Dd[a][c] rate[c],
// Dd = betaK D (+ betaKcomm Dc when betaKcomm is not zero: add_committed_D), D the point's tangent of
// this update (as the material returned it, before any mirroring), Dc its committed tangent, rate
// the strain of the element velocities at the point.
FX_HD void damping_stress(const double* Dd, const double xl[3][8], const double* ve, int gp, double sd[6]) {
  PointShape s;
  point_shape(xl, gp, s);
  double rate[6];
  strain_of(s, ve, rate);
  for (int a = 0; a < 6; ++a) {
    double sum = 0.0;
    for (int c = 0; c < 6; ++c) sum += Dd[6 * a + c] * rate[c];
    sd[a] = sum;
  }
}

// Internal force of one element from its points' stresses (point gp's component c at
// sig[(c * 8 + gp) * stride]) and damping stresses (sdamp, likewise, or NULL), in OpenSees' order:
// per point resid += B^T sigma dvol, resid -= body, fdamp += B^T sigma_d dvol + alphaM M v;
// fe = resid + fdamp.
FX_HD void element_force_from_stress(const ParamGP& p, const double xl[3][8], const double* ve, const double* sig,
                                     const double* sdamp, int64_t stride, double* fe) {
  double resid[24], fdamp[24];
  for (int a = 0; a < 24; ++a) resid[a] = fdamp[a] = 0.0;
  for (int gp = 0; gp < 8; gp++) {
    PointShape s;
    point_shape(xl, gp, s);
    double sg[6], vg[3];
    for (int c = 0; c < 6; ++c) sg[c] = sig[(c * 8 + gp) * stride];
    vg[0] = vg[1] = vg[2] = 0.0;
    if (p.alphaM != 0.0 && p.mass_type == 0)
      for (int j = 0; j < 8; j++)
        for (int q = 0; q < 3; q++) vg[q] += s.N[j] * ve[3 * j + q];
    double sd[6];
    if (sdamp)
      for (int c = 0; c < 6; ++c) sd[c] = sdamp[(c * 8 + gp) * stride];
    for (int j = 0; j < 8; j++) {
      double r[3], body[3], dj[3];
      node_force(s, sg, j, r);
      for (int q = 0; q < 3; q++) body[q] = s.dvol * p.b[q] * s.N[j];
      dj[0] = dj[1] = dj[2] = 0.0;
      if (sdamp) node_force(s, sd, j, dj);
      if (p.alphaM != 0.0) {
        const double tm = s.N[j] * s.dvol * p.rho;
        for (int q = 0; q < 3; q++) {
          const double vq = p.mass_type == 0 ? vg[q] : ve[3 * j + q];
          dj[q] += p.alphaM * tm * vq;
        }
      }
      for (int q = 0; q < 3; q++) {
        resid[3 * j + q] += r[q];
        resid[3 * j + q] -= body[q];
        fdamp[3 * j + q] += dj[q];
      }
    }
  }
  for (int a = 0; a < 24; ++a) fe[a] = resid[a] + fdamp[a];
}

// The material matrix of point gp for the operator (the reference's effective_tangent,
// src/physics/operators/element_operator.hpp:58-75, without betaKinit): the stored tangent of the
// last force evaluation scaled by the stiffness factor, plus cc times the tangent at the committed
// state (betaKcomm damping, not mirrored). ModifiedNewton -initial is refused on these sets, as the
// reference refuses it (general.cu, refuse_pimy_initial).
// The material declares its tangent symmetric, so it is stored as its upper triangle and the lower
// one mirrors it (the reference's TangentStorage, src/physics/common/tangent_storage.hpp:17-31).
struct PimyPointD {
  const PimySet* m;
  const double* tan;
  const double* committed;  // the committed states (read only when cc is not zero)
  int64_t stride;
  double cK, cc;
  FX_HD void operator()(int gp, double De[6][6]) const {
    double D[36];
    double t[pimy::kTan];
    for (int c = 0; c < pimy::kTan; ++c) t[c] = tan[(c * 8 + gp) * stride];
    pimy::compact_D(t, D);
    for (int a = 0; a < 6; ++a)
      for (int c = a + 1; c < 6; ++c) D[6 * c + a] = D[6 * a + c];
    for (int a = 0; a < 6; ++a)
      for (int c = 0; c < 6; ++c) De[a][c] = cK * D[6 * a + c];
    if (cc != 0.0) add_committed_D(*m, committed, gp, stride, cc, &De[0][0]);
  }
};

// The operator's material matrix of a PressureDependMultiYield point (effective_tangent,
// element_operator.hpp:60-75): cK times its stored tangent (upper triangle mirrored), plus c0
// times the material's initial tangent (the reference elastic tangent: the stiffness term under
// ModifiedNewton -initial), plus cc times its committed tangent.
struct PdmyPointD {
  const PdmySet* m;
  const double* tan;
  const double* committed;  // the committed states (read only when cc is not zero)
  int64_t stride;
  double cK, c0, cc;
  FX_HD void operator()(int gp, double De[6][6]) const {
    double D[36];
    double t[pdmy::kTan];
    for (int c = 0; c < pdmy::kTan; ++c) t[c] = tan[(c * 8 + gp) * stride];
    pdmy::compact_D(m->p, t, D);
    for (int a = 0; a < 6; ++a)
      for (int c = a + 1; c < 6; ++c) D[6 * c + a] = D[6 * a + c];
    for (int a = 0; a < 6; ++a)
      for (int c = 0; c < 6; ++c) De[a][c] = cK * D[6 * a + c];
    if (c0 != 0.0) {
      double D0[36];
      pdmy::elastic_D(m->p, 1.0, D0);
      for (int i = 0; i < 36; ++i) (&De[0][0])[i] += c0 * D0[i];
    }
    if (cc != 0.0) add_committed_D(*m, committed, gp, stride, cc, &De[0][0]);
  }
};

}  // namespace fx
