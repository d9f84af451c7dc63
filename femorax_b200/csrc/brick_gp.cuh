// stdBrick (8-node trilinear hexahedron, 2x2x2 Gauss) with ElasticIsotropic, point by point:
// the arithmetic of the general execution path, for host and device.
//
// The operations and their order follow the reference's element so that a build without fused
// multiply-adds (nvcc --fmad=false, host -ffp-contract=off) reproduces its results bit for bit:
//   shape functions          src/physics/elements/std_brick.hpp:45-152 (OpenSees shp3d)
//   Gauss point geometry     std_brick.hpp:203-211 (gp = 4i + 2j + k, weights 1)
//   strain                   std_brick.hpp:276-301 (11 22 33 12 23 31, engineering shear)
//   node force B^T s dvol    std_brick.hpp:305-327
//   elastic stress, tangent  src/physics/materials/elastic_isotropic.hpp:40-94
//   element force + damping  std_brick.hpp:409-464, 492-543
//   element operator         src/physics/operators/element_operator.hpp:45-130
//   lumped mass              std_brick.hpp:609-623
// The bit-exactness is the reason the steps are alike; the code is this project's own.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define FX_HD __host__ __device__ __forceinline__
#else
#define FX_HD inline
#endif

namespace fx {

struct ParamGP {  // one parameter set as the element kernels read it
  double E, nu, rho;
  double b[3];
  double alphaM, betaK, betaKinit, betaKcomm;
  int mass_type;  // 0 consistent, 1 lumped
  int kind;       // 0 elastic, 1 J2, 2 PressureIndependMultiYield
  double sigma_y, H, hk;
  int table;      // kind 2: the set's entry in the PressureIndependMultiYield table
  int element;    // 0 stdBrick, 1 SSPbrick
};

struct PointShape {
  double dN[3][8];  // global derivatives
  double N[8];      // values
  double dvol;
};

// Natural coordinates of Gauss point gp: (s[(gp>>2)&1], s[(gp>>1)&1], s[gp&1]), s = -+1/sqrt(3).
FX_HD void gauss_point(int gp, double g[3]) {
  const double r = 1.0 / sqrt(3.0);
  g[0] = ((gp >> 2) & 1) ? r : -r;
  g[1] = ((gp >> 1) & 1) ? r : -r;
  g[2] = (gp & 1) ? r : -r;
}

// Shape function values and derivatives at natural point (x1, x2, x3), then the Jacobian, its
// adjoint and the global derivatives. The corner factors are formed pairwise per face as the
// reference forms them.
FX_HD void shape_at(const double g[3], const double xl[3][8], PointShape& s) {
  double dn[3][8];
  const double p1 = 1.0 + g[0], m1 = 1.0 - g[0];
  const double p2 = 1.0 + g[1], m2 = 1.0 - g[1];
  const double p3 = 1.0 + g[2], m3 = 1.0 - g[2];
  // face (-,-)
  double a = 0.125 * m1 * m2, b = 0.125 * m2 * m3, c = 0.125 * m1 * m3;
  dn[0][0] = -b;
  dn[0][1] = b;
  dn[1][0] = -c;
  dn[1][3] = c;
  dn[2][0] = -a;
  dn[2][4] = a;
  s.N[0] = a * m3;
  s.N[4] = a * p3;
  // face (+,+)
  a = 0.125 * p1 * p2;
  b = 0.125 * p2 * p3;
  c = 0.125 * p1 * p3;
  dn[0][7] = -b;
  dn[0][6] = b;
  dn[1][5] = -c;
  dn[1][6] = c;
  dn[2][2] = -a;
  dn[2][6] = a;
  s.N[2] = a * m3;
  s.N[6] = a * p3;
  // face (-,+)
  a = 0.125 * m1 * p2;
  b = 0.125 * m2 * p3;
  c = 0.125 * m1 * p3;
  dn[0][4] = -b;
  dn[0][5] = b;
  dn[1][4] = -c;
  dn[1][7] = c;
  dn[2][3] = -a;
  dn[2][7] = a;
  s.N[3] = a * m3;
  s.N[7] = a * p3;
  // face (+,-)
  a = 0.125 * p1 * m2;
  b = 0.125 * p2 * m3;
  c = 0.125 * p1 * m3;
  dn[0][3] = -b;
  dn[0][2] = b;
  dn[1][1] = -c;
  dn[1][2] = c;
  dn[2][1] = -a;
  dn[2][5] = a;
  s.N[1] = a * m3;
  s.N[5] = a * p3;

  double J[3][3], A[3][3];
  for (int d = 0; d < 3; d++) {
    J[d][0] = (xl[d][1] - xl[d][0]) * dn[0][1] + (xl[d][2] - xl[d][3]) * dn[0][2] +
              (xl[d][5] - xl[d][4]) * dn[0][5] + (xl[d][6] - xl[d][7]) * dn[0][6];
    J[d][1] = (xl[d][2] - xl[d][1]) * dn[1][2] + (xl[d][3] - xl[d][0]) * dn[1][3] +
              (xl[d][6] - xl[d][5]) * dn[1][6] + (xl[d][7] - xl[d][4]) * dn[1][7];
    J[d][2] = (xl[d][4] - xl[d][0]) * dn[2][4] + (xl[d][5] - xl[d][1]) * dn[2][5] +
              (xl[d][6] - xl[d][2]) * dn[2][6] + (xl[d][7] - xl[d][3]) * dn[2][7];
  }
  A[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  A[0][1] = J[2][1] * J[0][2] - J[2][2] * J[0][1];
  A[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
  A[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  A[1][1] = J[2][2] * J[0][0] - J[2][0] * J[0][2];
  A[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
  A[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  A[2][1] = J[2][0] * J[0][1] - J[2][1] * J[0][0];
  A[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  const double det = J[0][0] * A[0][0] + J[0][1] * A[1][0] + J[0][2] * A[2][0];
  const double rdet = 1.0 / det;
  double Ji[3][3];
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < 3; i++) Ji[i][j] = A[i][j] * rdet;
  for (int k = 0; k < 8; k++) {
    s.dN[0][k] = dn[0][k] * Ji[0][0] + dn[1][k] * Ji[1][0] + dn[2][k] * Ji[2][0];
    s.dN[1][k] = dn[0][k] * Ji[0][1] + dn[1][k] * Ji[1][1] + dn[2][k] * Ji[2][1];
    s.dN[2][k] = dn[0][k] * Ji[0][2] + dn[1][k] * Ji[1][2] + dn[2][k] * Ji[2][2];
  }
  s.dvol = 1.0 * det;
}

FX_HD void point_shape(const double xl[3][8], int gp, PointShape& s) {
  double g[3];
  gauss_point(gp, g);
  shape_at(g, xl, s);
}

// epsilon = B u at a point.
FX_HD void strain_of(const PointShape& s, const double* u, double e[6]) {
  for (int c = 0; c < 6; ++c) e[c] = 0.0;
  for (int j = 0; j < 8; j++) {
    const double dx = s.dN[0][j], dy = s.dN[1][j], dz = s.dN[2][j];
    const double u0 = u[3 * j], u1 = u[3 * j + 1], u2 = u[3 * j + 2];
    e[0] += dx * u0;
    e[1] += dy * u1;
    e[2] += dz * u2;
    e[3] += dy * u0 + dx * u1;
    e[4] += dz * u1 + dy * u2;
    e[5] += dz * u0 + dx * u2;
  }
}

// B_j^T (sigma dvol).
FX_HD void node_force(const PointShape& s, const double sg[6], int j, double r[3]) {
  const double s0 = sg[0] * s.dvol, s1 = sg[1] * s.dvol, s2 = sg[2] * s.dvol;
  const double s3 = sg[3] * s.dvol, s4 = sg[4] * s.dvol, s5 = sg[5] * s.dvol;
  const double dx = s.dN[0][j], dy = s.dN[1][j], dz = s.dN[2][j];
  r[0] = dx * s0 + dy * s3 + dz * s5;
  r[1] = dy * s1 + dx * s3 + dz * s4;
  r[2] = dz * s2 + dy * s4 + dx * s5;
}

// Elastic constants as ElasticIsotropic forms them: 2G+lambda, lambda, G.
FX_HD void lame(const ParamGP& p, double& l2m, double& lam, double& mu) {
  double m2 = p.E / (1.0 + p.nu);
  lam = p.nu * m2 / (1.0 - 2.0 * p.nu);
  mu = 0.50 * m2;
  l2m = m2 + lam;
}

FX_HD void elastic_D(const ParamGP& p, double D[6][6]) {
  double l2m, lam, mu;
  lame(p, l2m, lam, mu);
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) D[i][j] = 0.0;
  D[0][0] = D[1][1] = D[2][2] = l2m;
  D[0][1] = D[1][0] = D[0][2] = D[2][0] = D[1][2] = D[2][1] = lam;
  D[3][3] = D[4][4] = D[5][5] = mu;
}

FX_HD void elastic_stress(const ParamGP& p, const double e[6], double sg[6]) {
  double l2m, lam, mu;
  lame(p, l2m, lam, mu);
  sg[0] = l2m * e[0] + lam * (e[1] + e[2]);
  sg[1] = l2m * e[1] + lam * (e[0] + e[2]);
  sg[2] = l2m * e[2] + lam * (e[0] + e[1]);
  sg[3] = mu * e[3];
  sg[4] = mu * e[4];
  sg[5] = mu * e[5];
}

// ---------------------------------------------------------------- J2 plasticity
// No counterpart in the reference (which has no J2 material): the von Mises radial return with
// linear hardening H split into isotropic (1 - hk) H and kinematic hk H parts (Simo and Hughes,
// Computational Inelasticity, 1998, box 3.2), on engineering strains in the OpenSees order
// (11 22 33 12 23 31). State per Gauss point (kJ2State values): plastic strain (engineering
// shear) [6], equivalent plastic strain, back stress [6]. Consistent tangent per point, compact
// (kJ2Tan values): theta, thetab, n[6], with
//   D_t = K 1 (x) 1 + 2 G theta I_dev - 2 G thetab n (x) n
// (theta = 1, thetab = 0, n = 0 at an elastic point gives the elastic matrix exactly).
constexpr int kJ2State = 13;
constexpr int kJ2Tan = 8;

FX_HD void j2_moduli(const ParamGP& p, double& K, double& G) {
  K = p.E / (3.0 * (1.0 - 2.0 * p.nu));
  G = p.E / (2.0 * (1.0 + p.nu));
}

// Trial state and stress at total strain eps from the committed state; returns true if plastic.
FX_HD bool j2_update(const ParamGP& p, const double* committed, double* trial, const double eps[6], double sigma[6],
                     double tan[kJ2Tan]) {
  double K, G;
  j2_moduli(p, K, G);
  const double Hkin = p.hk * p.H, Hiso = (1.0 - p.hk) * p.H;
  double ee[6];
  for (int i = 0; i < 6; ++i) ee[i] = (i < 3 ? 1.0 : 0.5) * (eps[i] - committed[i]);
  const double alpha = committed[6];
  const double* back = committed + 7;
  const double tr = ee[0] + ee[1] + ee[2];
  double s_tr[6], xi[6];
  for (int i = 0; i < 6; ++i) s_tr[i] = 2.0 * G * (i < 3 ? ee[i] - tr / 3.0 : ee[i]);
  for (int i = 0; i < 6; ++i) xi[i] = s_tr[i] - back[i];
  const double nxi = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2] +
                          2.0 * (xi[3] * xi[3] + xi[4] * xi[4] + xi[5] * xi[5]));
  const double r23 = sqrt(2.0 / 3.0);
  const double f = nxi - r23 * (p.sigma_y + Hiso * alpha);
  for (int i = 0; i < kJ2State; ++i) trial[i] = committed[i];
  const double pr = K * tr;
  tan[0] = 1.0;
  for (int i = 1; i < kJ2Tan; ++i) tan[i] = 0.0;
  if (f <= 0.0 || nxi == 0.0) {
    for (int i = 0; i < 6; ++i) sigma[i] = s_tr[i] + (i < 3 ? pr : 0.0);
    return false;
  }
  const double dg = f / (2.0 * G + (2.0 / 3.0) * p.H);
  double n[6];
  for (int i = 0; i < 6; ++i) n[i] = xi[i] / nxi;
  for (int i = 0; i < 6; ++i) sigma[i] = s_tr[i] - 2.0 * G * dg * n[i] + (i < 3 ? pr : 0.0);
  for (int i = 0; i < 6; ++i) trial[i] = committed[i] + (i < 3 ? 1.0 : 2.0) * dg * n[i];
  trial[6] = alpha + r23 * dg;
  for (int i = 0; i < 6; ++i) trial[7 + i] = back[i] + (2.0 / 3.0) * Hkin * dg * n[i];
  const double theta = 1.0 - 2.0 * G * dg / nxi;
  tan[0] = theta;
  tan[1] = 1.0 / (1.0 + p.H / (3.0 * G)) - (1.0 - theta);
  for (int i = 0; i < 6; ++i) tan[2 + i] = n[i];
  return true;
}

// The 6 x 6 consistent tangent of a point from its compact form.
FX_HD void j2_D(const ParamGP& p, const double tan[kJ2Tan], double D[6][6]) {
  double K, G;
  j2_moduli(p, K, G);
  const double theta = tan[0], thetab = tan[1];
  const double* n = tan + 2;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double idev;
      if (i < 3 && j < 3) idev = (i == j ? 1.0 : 0.0) - 1.0 / 3.0;
      else idev = (i == j) ? 0.5 : 0.0;
      const double vol = (i < 3 && j < 3) ? K : 0.0;
      D[i][j] = vol + 2.0 * G * theta * idev - 2.0 * G * thetab * n[i] * n[j];
    }
}

// Operator factors (element_operator.hpp:45-56; stdBrick's initial stiffness is not its
// tangent): k = {stiffness, damping, mass}. cK scales the point's tangent, c0 the initial
// (elastic) tangent, cc the committed tangent; with `initial` (ModifiedNewton -initial) the
// stiffness term moves from the tangent to the initial tangent, the damping terms stay.
struct OpFactors {
  double cK, c0, cc, cM;
};
FX_HD OpFactors op_factors(const ParamGP& p, double ks, double kd, double km, bool initial = false) {
  OpFactors f;
  f.cK = initial ? kd * p.betaK : ks + kd * p.betaK;
  f.c0 = initial ? ks + kd * p.betaKinit : kd * p.betaKinit;
  f.cc = kd * p.betaKcomm;
  f.cM = km + kd * p.alphaM;
  return f;
}

// D_eff = cK D + c0 D0 + cc Dc with the constant elastic tangent (D = D0 = Dc).
FX_HD void effective_D(const OpFactors& f, const ParamGP& p, double De[6][6]) {
  double D[6][6];
  elastic_D(p, D);
  for (int a = 0; a < 6; ++a)
    for (int c = 0; c < 6; ++c) {
      double v = f.cK * D[a][c];
      if (f.c0 != 0.0) v += f.c0 * D[a][c];
      if (f.cc != 0.0) v += f.cc * D[a][c];
      De[a][c] = v;
    }
}

// Sources of the effective material matrix at a point: the constant elastic one, or a J2
// element's consistent tangent per point (component c of point gp at tan[(c * 8 + gp) * stride]),
// scaled by the stiffness factor (J2 sets carry no stiffness-proportional damping, so the
// factor is cK, or c0 on the elastic matrix with `initial`: ModifiedNewton -initial).
struct ConstD {
  double De[6][6];
  FX_HD void operator()(int, double D[6][6]) const {
    for (int a = 0; a < 6; ++a)
      for (int c = 0; c < 6; ++c) D[a][c] = De[a][c];
  }
};
struct J2PointD {
  const ParamGP* p;
  const double* tan;
  int64_t stride;
  double cK;
  bool initial;
  FX_HD void operator()(int gp, double De[6][6]) const {
    double t[kJ2Tan];
    for (int c = 0; c < kJ2Tan; ++c) t[c] = initial ? (c == 0 ? 1.0 : 0.0) : tan[(c * 8 + gp) * stride];
    double D[6][6];
    j2_D(*p, t, D);
    for (int a = 0; a < 6; ++a)
      for (int c = 0; c < 6; ++c) De[a][c] = cK * D[a][c];
  }
};

// y_e = K_eff,e x_e point by point, the material matrix of point gp from dsrc.
template <class DSrc>
FX_HD void element_apply_d(const ParamGP& p, const OpFactors& f, const double xl[3][8], const double* xe, double* ye,
                           const DSrc& dsrc) {
  for (int a = 0; a < 24; ++a) ye[a] = 0.0;
  for (int gp = 0; gp < 8; ++gp) {
    PointShape s;
    point_shape(xl, gp, s);
    double De[6][6];
    dsrc(gp, De);
    double e[6], sg[6];
    strain_of(s, xe, e);
    for (int a = 0; a < 6; ++a) {
      double sum = 0.0;
      for (int c = 0; c < 6; ++c) sum += De[a][c] * e[c];
      sg[a] = sum;
    }
    for (int j = 0; j < 8; ++j) {
      double fj[3];
      node_force(s, sg, j, fj);
      for (int q = 0; q < 3; ++q) ye[3 * j + q] += fj[q];
      if (f.cM != 0.0) {
        const double t = s.N[j] * s.dvol * p.rho;
        double mj[3];
        for (int q = 0; q < 3; q++) {
          double vq;
          if (p.mass_type == 0) {
            vq = 0.0;
            for (int k = 0; k < 8; k++) vq += s.N[k] * xe[3 * k + q];
          } else {
            vq = xe[3 * j + q];
          }
          mj[q] = t * vq;
        }
        for (int q = 0; q < 3; ++q) ye[3 * j + q] += f.cM * mj[q];
      }
    }
  }
}

FX_HD void element_apply(const ParamGP& p, const OpFactors& f, const double xl[3][8], const double* xe, double* ye) {
  ConstD c;
  effective_D(f, p, c.De);
  element_apply_d(p, f, xl, xe, ye, c);
}

// 3x3 block (J, K) of B^T D B dvol at one point, in the reference's two-stage form.
FX_HD void block_tangent(const PointShape& s, const double D[6][6], int J, int K, double out[3][3]) {
  // B_J as rows 6 x cols 3 (sparse), written out
  double BJ[6][3] = {}, BK[6][3] = {};
  BJ[0][0] = s.dN[0][J];
  BJ[1][1] = s.dN[1][J];
  BJ[2][2] = s.dN[2][J];
  BJ[3][0] = s.dN[1][J];
  BJ[3][1] = s.dN[0][J];
  BJ[4][1] = s.dN[2][J];
  BJ[4][2] = s.dN[1][J];
  BJ[5][0] = s.dN[2][J];
  BJ[5][2] = s.dN[0][J];
  BK[0][0] = s.dN[0][K];
  BK[1][1] = s.dN[1][K];
  BK[2][2] = s.dN[2][K];
  BK[3][0] = s.dN[1][K];
  BK[3][1] = s.dN[0][K];
  BK[4][1] = s.dN[2][K];
  BK[4][2] = s.dN[1][K];
  BK[5][0] = s.dN[2][K];
  BK[5][2] = s.dN[0][K];
  double T[3][6];
  for (int a = 0; a < 3; a++)
    for (int q = 0; q < 6; q++) {
      double sum = 0.0;
      for (int r = 0; r < 6; r++) sum += BJ[r][a] * (D[r][q] * s.dvol);
      T[a][q] = sum;
    }
  for (int a = 0; a < 3; a++)
    for (int q = 0; q < 3; q++) {
      double sum = 0.0;
      for (int r = 0; r < 6; r++) sum += T[a][r] * BK[r][q];
      out[a][q] = sum;
    }
}

FX_HD double mass_entry(const ParamGP& p, const PointShape& s, int j, int k) {
  const double t = s.N[j] * s.dvol * p.rho;
  if (p.mass_type == 0) return t * s.N[k];
  return j == k ? t : 0.0;
}

// Diagonal of K_eff,e by local DOF, with the terms of local DOFs merged into one equation
// (element_operator.hpp:138-209). eq: the element's 24 equations; the material matrix of point gp
// from dsrc.
template <class DSrc>
FX_HD void element_diagonal_d(const ParamGP& p, const OpFactors& f, const double xl[3][8], const int* eq, double* de,
                              const DSrc& dsrc) {
  for (int a = 0; a < 24; ++a) de[a] = 0.0;
  int first[24];
  bool merged = false;
  for (int a = 0; a < 24; ++a) {
    first[a] = a;
    if (eq[a] < 0) continue;
    for (int b = 0; b < a; ++b)
      if (eq[b] == eq[a]) {
        first[a] = first[b];
        merged = true;
        break;
      }
  }
  for (int gp = 0; gp < 8; ++gp) {
    PointShape s;
    point_shape(xl, gp, s);
    double De[6][6];
    dsrc(gp, De);
    for (int j = 0; j < 8; ++j) {
      double blk[3][3];
      block_tangent(s, De, j, j, blk);
      const double m = f.cM != 0.0 ? f.cM * mass_entry(p, s, j, j) : 0.0;
      for (int q = 0; q < 3; ++q) de[3 * j + q] += blk[q][q] + m;
    }
    if (!merged) continue;
    for (int J = 0; J < 8; ++J)
      for (int K = 0; K < 8; ++K) {
        bool any = false;
        for (int a = 0; a < 3 && !any; ++a)
          for (int c = 0; c < 3; ++c) {
            const int ia = 3 * J + a, ic = 3 * K + c;
            if (ia != ic && eq[ia] >= 0 && eq[ia] == eq[ic]) any = true;
          }
        if (!any) continue;
        double blk[3][3];
        block_tangent(s, De, J, K, blk);
        const double m = (f.cM != 0.0 && J != K) ? f.cM * mass_entry(p, s, J, K) : 0.0;
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) {
            const int ia = 3 * J + a, ic = 3 * K + c;
            if (ia == ic || eq[ia] < 0 || eq[ia] != eq[ic]) continue;
            de[first[ia]] += blk[a][c] + (a == c ? m : 0.0);
          }
      }
  }
}

FX_HD void element_diagonal(const ParamGP& p, const OpFactors& f, const double xl[3][8], const int* eq, double* de) {
  ConstD c;
  effective_D(f, p, c.De);
  element_diagonal_d(p, f, xl, eq, de, c);
}

// Internal force with body force plus the four Rayleigh damping forces (elastic material).
FX_HD void element_force(const ParamGP& p, const double xl[3][8], const double* ue, const double* ve, double* fe) {
  double resid[24], fdamp[24];
  for (int a = 0; a < 24; ++a) resid[a] = fdamp[a] = 0.0;
  double D[6][6];
  elastic_D(p, D);
  const bool stiff = p.betaK != 0.0 || p.betaKinit != 0.0 || p.betaKcomm != 0.0;
  for (int gp = 0; gp < 8; gp++) {
    PointShape s;
    point_shape(xl, gp, s);
    double e[6], sg[6], ds[6], vg[3];
    strain_of(s, ue, e);
    elastic_stress(p, e, sg);
    for (int a = 0; a < 6; ++a) ds[a] = 0.0;
    if (stiff) {
      double rate[6];
      strain_of(s, ve, rate);
      for (int a = 0; a < 6; ++a) {
        double sum = 0.0;
        for (int c = 0; c < 6; ++c) {
          double Dac = p.betaK * D[a][c];
          if (p.betaKinit != 0.0) Dac += p.betaKinit * D[a][c];
          if (p.betaKcomm != 0.0) Dac += p.betaKcomm * D[a][c];
          sum += Dac * rate[c];
        }
        ds[a] = sum;
      }
    }
    vg[0] = vg[1] = vg[2] = 0.0;
    if (p.alphaM != 0.0 && p.mass_type == 0)
      for (int j = 0; j < 8; j++)
        for (int q = 0; q < 3; q++) vg[q] += s.N[j] * ve[3 * j + q];
    for (int j = 0; j < 8; j++) {
      double r[3], body[3], dj[3];
      node_force(s, sg, j, r);
      for (int q = 0; q < 3; q++) body[q] = s.dvol * p.b[q] * s.N[j];
      dj[0] = dj[1] = dj[2] = 0.0;
      if (stiff) node_force(s, ds, j, dj);
      if (p.alphaM != 0.0) {
        const double t = s.N[j] * s.dvol * p.rho;
        for (int q = 0; q < 3; q++) {
          const double vq = p.mass_type == 0 ? vg[q] : ve[3 * j + q];
          dj[q] += p.alphaM * t * vq;
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

// Internal force of a J2 element at displacement ue: the stress of every point by the return map
// from its committed state (component c of point gp at committed[(c * 8 + gp) * stride]), which
// also writes the point's trial state and compact tangent (same layout); minus the body force;
// plus the mass-proportional Rayleigh force at ve (J2 sets carry no stiffness-proportional
// damping). The sums run in element_force's order. Returns the number of plastic points.
FX_HD int element_force_j2(const ParamGP& p, const double xl[3][8], const double* ue, const double* ve,
                           const double* committed, double* trial, double* tan, int64_t stride, double* fe) {
  double resid[24], fdamp[24];
  for (int a = 0; a < 24; ++a) resid[a] = fdamp[a] = 0.0;
  int plastic = 0;
  for (int gp = 0; gp < 8; gp++) {
    PointShape s;
    point_shape(xl, gp, s);
    double e[6], sg[6], vg[3], cst[kJ2State], tst[kJ2State], tn[kJ2Tan];
    strain_of(s, ue, e);
    for (int c = 0; c < kJ2State; ++c) cst[c] = committed[(c * 8 + gp) * stride];
    plastic += j2_update(p, cst, tst, e, sg, tn) ? 1 : 0;
    for (int c = 0; c < kJ2State; ++c) trial[(c * 8 + gp) * stride] = tst[c];
    for (int c = 0; c < kJ2Tan; ++c) tan[(c * 8 + gp) * stride] = tn[c];
    vg[0] = vg[1] = vg[2] = 0.0;
    if (p.alphaM != 0.0 && p.mass_type == 0)
      for (int j = 0; j < 8; j++)
        for (int q = 0; q < 3; q++) vg[q] += s.N[j] * ve[3 * j + q];
    for (int j = 0; j < 8; j++) {
      double r[3], body[3], dj[3];
      node_force(s, sg, j, r);
      for (int q = 0; q < 3; q++) body[q] = s.dvol * p.b[q] * s.N[j];
      dj[0] = dj[1] = dj[2] = 0.0;
      if (p.alphaM != 0.0) {
        const double t = s.N[j] * s.dvol * p.rho;
        for (int q = 0; q < 3; q++) {
          const double vq = p.mass_type == 0 ? vg[q] : ve[3 * j + q];
          dj[q] += p.alphaM * t * vq;
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
  return plastic;
}

// Row-sum lumped mass per corner.
FX_HD void lumped_mass(const ParamGP& p, const double xl[3][8], double m[8]) {
  for (int j = 0; j < 8; j++) m[j] = 0.0;
  for (int gp = 0; gp < 8; gp++) {
    PointShape s;
    point_shape(xl, gp, s);
    for (int j = 0; j < 8; j++) {
      double t = s.N[j] * s.dvol;
      t *= p.rho;
      m[j] += t;
    }
  }
}

}  // namespace fx
