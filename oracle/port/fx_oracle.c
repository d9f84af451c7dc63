/* Oracle (test infrastructure only): plain-C restatement of the reference's hot path.
 * See fx_oracle.h. Built by oracle/Makefile with -ffp-contract=off (no fused multiply-adds),
 * which is how the reference's host builds evaluate these expressions.
 *
 * The order of every floating-point operation follows the cited reference lines; where the
 * reference writes `a += b * c + d * e`, this file writes the same expression, so that the
 * results are bit-identical to the reference's own host build.
 */
#include "fx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NDOF 24
#define NNODE 8
#define NGP 8
#define NS 6

/* ---------------------------------------------------------------- shape functions */
/* shp3d: src/physics/elements/std_brick.hpp:45-152 (OpenSees shp3d.cpp). shp[0..2][i] global
 * derivatives, shp[3][i] values. */
static void shp3d(const double ss[3], double* xsj_out, double shp[4][8], const double xl[3][8]) {
  double rxsj, ap1, am1, ap2, am2, ap3, am3, c1, c2, c3;
  double xs[3][3], ad[3][3], xsj;
  ap1 = 1.0 + ss[0];
  am1 = 1.0 - ss[0];
  ap2 = 1.0 + ss[1];
  am2 = 1.0 - ss[1];
  ap3 = 1.0 + ss[2];
  am3 = 1.0 - ss[2];
  c1 = 0.125 * am1 * am2;
  c2 = 0.125 * am2 * am3;
  c3 = 0.125 * am1 * am3;
  shp[0][0] = -c2;
  shp[0][1] = c2;
  shp[1][0] = -c3;
  shp[1][3] = c3;
  shp[2][0] = -c1;
  shp[2][4] = c1;
  shp[3][0] = c1 * am3;
  shp[3][4] = c1 * ap3;
  c1 = 0.125 * ap1 * ap2;
  c2 = 0.125 * ap2 * ap3;
  c3 = 0.125 * ap1 * ap3;
  shp[0][7] = -c2;
  shp[0][6] = c2;
  shp[1][5] = -c3;
  shp[1][6] = c3;
  shp[2][2] = -c1;
  shp[2][6] = c1;
  shp[3][2] = c1 * am3;
  shp[3][6] = c1 * ap3;
  c1 = 0.125 * am1 * ap2;
  c2 = 0.125 * am2 * ap3;
  c3 = 0.125 * am1 * ap3;
  shp[0][4] = -c2;
  shp[0][5] = c2;
  shp[1][4] = -c3;
  shp[1][7] = c3;
  shp[2][3] = -c1;
  shp[2][7] = c1;
  shp[3][3] = c1 * am3;
  shp[3][7] = c1 * ap3;
  c1 = 0.125 * ap1 * am2;
  c2 = 0.125 * ap2 * am3;
  c3 = 0.125 * ap1 * am3;
  shp[0][3] = -c2;
  shp[0][2] = c2;
  shp[1][1] = -c3;
  shp[1][2] = c3;
  shp[2][1] = -c1;
  shp[2][5] = c1;
  shp[3][1] = c1 * am3;
  shp[3][5] = c1 * ap3;
  for (int j = 0; j < 3; j++) {
    xs[j][0] = (xl[j][1] - xl[j][0]) * shp[0][1] + (xl[j][2] - xl[j][3]) * shp[0][2] +
               (xl[j][5] - xl[j][4]) * shp[0][5] + (xl[j][6] - xl[j][7]) * shp[0][6];
    xs[j][1] = (xl[j][2] - xl[j][1]) * shp[1][2] + (xl[j][3] - xl[j][0]) * shp[1][3] +
               (xl[j][6] - xl[j][5]) * shp[1][6] + (xl[j][7] - xl[j][4]) * shp[1][7];
    xs[j][2] = (xl[j][4] - xl[j][0]) * shp[2][4] + (xl[j][5] - xl[j][1]) * shp[2][5] +
               (xl[j][6] - xl[j][2]) * shp[2][6] + (xl[j][7] - xl[j][3]) * shp[2][7];
  }
  ad[0][0] = xs[1][1] * xs[2][2] - xs[1][2] * xs[2][1];
  ad[0][1] = xs[2][1] * xs[0][2] - xs[2][2] * xs[0][1];
  ad[0][2] = xs[0][1] * xs[1][2] - xs[0][2] * xs[1][1];
  ad[1][0] = xs[1][2] * xs[2][0] - xs[1][0] * xs[2][2];
  ad[1][1] = xs[2][2] * xs[0][0] - xs[2][0] * xs[0][2];
  ad[1][2] = xs[0][2] * xs[1][0] - xs[0][0] * xs[1][2];
  ad[2][0] = xs[1][0] * xs[2][1] - xs[1][1] * xs[2][0];
  ad[2][1] = xs[2][0] * xs[0][1] - xs[2][1] * xs[0][0];
  ad[2][2] = xs[0][0] * xs[1][1] - xs[0][1] * xs[1][0];
  xsj = xs[0][0] * ad[0][0] + xs[0][1] * ad[1][0] + xs[0][2] * ad[2][0];
  rxsj = 1.0 / xsj;
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < 3; i++) xs[i][j] = ad[i][j] * rxsj;
  for (int k = 0; k < 8; k++) {
    c1 = shp[0][k] * xs[0][0] + shp[1][k] * xs[1][0] + shp[2][k] * xs[2][0];
    c2 = shp[0][k] * xs[0][1] + shp[1][k] * xs[1][1] + shp[2][k] * xs[2][1];
    c3 = shp[0][k] * xs[0][2] + shp[1][k] * xs[1][2] + shp[2][k] * xs[2][2];
    shp[0][k] = c1;
    shp[1][k] = c2;
    shp[2][k] = c3;
  }
  *xsj_out = xsj;
}

typedef struct {
  double shp[4][8];
  double dvol;
} point_shape;

/* StdBrick::point_geometry, std_brick.hpp:203-211: gp = 4i + 2j + k, weight 1. */
static void point_geometry(const double xl[3][8], int gp, point_shape* s) {
  const double r = 1.0 / sqrt(3.0);
  const double sg[2] = {-r, r};
  const double g[3] = {sg[(gp >> 2) & 1], sg[(gp >> 1) & 1], sg[gp & 1]};
  double xsj;
  shp3d(g, &xsj, s->shp, xl);
  s->dvol = 1.0 * xsj;
}

static void local_coords(const double* xe, double xl[3][8]) {
  for (int i = 0; i < 8; i++) {
    xl[0][i] = xe[3 * i + 0];
    xl[1][i] = xe[3 * i + 1];
    xl[2][i] = xe[3 * i + 2];
  }
}

/* point_strain, std_brick.hpp:276-301 (11 22 33 12 23 31, engineering shear). */
static void point_strain(const point_shape* s, const double* ul, double strain[NS]) {
  for (int c = 0; c < NS; ++c) strain[c] = 0.0;
  for (int j = 0; j < NNODE; j++) {
    const double b00 = s->shp[0][j], b11 = s->shp[1][j], b22 = s->shp[2][j];
    const double b30 = s->shp[1][j], b31 = s->shp[0][j];
    const double b41 = s->shp[2][j], b42 = s->shp[1][j];
    const double b50 = s->shp[2][j], b52 = s->shp[0][j];
    const double ul0 = ul[3 * j + 0], ul1 = ul[3 * j + 1], ul2 = ul[3 * j + 2];
    strain[0] += b00 * ul0;
    strain[1] += b11 * ul1;
    strain[2] += b22 * ul2;
    strain[3] += b30 * ul0 + b31 * ul1;
    strain[4] += b41 * ul1 + b42 * ul2;
    strain[5] += b50 * ul0 + b52 * ul2;
  }
}

/* point_node_force, std_brick.hpp:305-327: B_j^T (stress * dvol). */
static void point_node_force(const point_shape* s, const double st[NS], int j, double r[3]) {
  const double s0 = st[0] * s->dvol, s1 = st[1] * s->dvol, s2 = st[2] * s->dvol;
  const double s3 = st[3] * s->dvol, s4 = st[4] * s->dvol, s5 = st[5] * s->dvol;
  const double b00 = s->shp[0][j], b11 = s->shp[1][j], b22 = s->shp[2][j];
  const double b30 = s->shp[1][j], b31 = s->shp[0][j];
  const double b41 = s->shp[2][j], b42 = s->shp[1][j];
  const double b50 = s->shp[2][j], b52 = s->shp[0][j];
  r[0] = b00 * s0 + b30 * s3 + b50 * s5;
  r[1] = b11 * s1 + b31 * s3 + b41 * s4;
  r[2] = b22 * s2 + b42 * s4 + b52 * s5;
}

/* ElasticIsotropic: update (stress by the explicit formulas) and the tangent,
 * src/physics/materials/elastic_isotropic.hpp:40-94. */
static void elastic_constants(const fxo_param* p, double* mu2_out, double* lam_out, double* mu_out) {
  double mu2 = p->E / (1.0 + p->nu);
  const double lam = p->nu * mu2 / (1.0 - 2.0 * p->nu);
  const double mu = 0.50 * mu2;
  mu2 += lam;
  *mu2_out = mu2;
  *lam_out = lam;
  *mu_out = mu;
}
static void elastic_tangent(const fxo_param* p, double D[NS][NS]) {
  double mu2, lam, mu;
  elastic_constants(p, &mu2, &lam, &mu);
  for (int i = 0; i < NS; ++i)
    for (int j = 0; j < NS; ++j) D[i][j] = 0.0;
  D[0][0] = D[1][1] = D[2][2] = mu2;
  D[0][1] = D[1][0] = D[0][2] = D[2][0] = D[1][2] = D[2][1] = lam;
  D[3][3] = mu;
  D[4][4] = mu;
  D[5][5] = mu;
}
static void elastic_update(const fxo_param* p, const double eps[NS], double sigma[NS], double D[NS][NS]) {
  double mu2, lam, mu;
  elastic_constants(p, &mu2, &lam, &mu);
  const double e0 = eps[0], e1 = eps[1], e2 = eps[2];
  sigma[0] = mu2 * e0 + lam * (e1 + e2);
  sigma[1] = mu2 * e1 + lam * (e0 + e2);
  sigma[2] = mu2 * e2 + lam * (e0 + e1);
  sigma[3] = mu * eps[3];
  sigma[4] = mu * eps[4];
  sigma[5] = mu * eps[5];
  elastic_tangent(p, D);
}

/* ---------------------------------------------------------------- element force */
/* StdBrick::compute_with, std_brick.hpp:492-543, with point_update_shape (:409-443) and
 * point_node_contribution (:448-464); the tangent as point_block_tangent (:336-356). */
static void block_tangent(const point_shape* s, double dd[NS][NS], int J, int K, double st[3][3]);

void fxo_brick_compute(const fxo_param* p, const double* xe, const double* ue, const double* ve, double* fe,
                       double* Ke) {
  double xl[3][8];
  local_coords(xe, xl);
  double resid[NDOF], fdamp[NDOF];
  for (int a = 0; a < NDOF; ++a) resid[a] = fdamp[a] = 0.0;
  if (Ke)
    for (int a = 0; a < NDOF * NDOF; ++a) Ke[a] = 0.0;
  double D0[NS][NS];
  if (p->betaKinit != 0.0) elastic_tangent(p, D0);
  const int stiff_damping = p->betaK != 0.0 || p->betaKinit != 0.0 || p->betaKcomm != 0.0;
  for (int i = 0; i < NGP; i++) {
    point_shape s;
    point_geometry(xl, i, &s);
    double strain[NS], stress[NS], dd[NS][NS], damp_stress[NS], v_gp[3];
    point_strain(&s, ue, strain);
    elastic_update(p, strain, stress, dd);
    for (int a = 0; a < NS; ++a) damp_stress[a] = 0.0;
    if (stiff_damping) {
      double Dc[NS][NS], rate[NS];
      if (p->betaKcomm != 0.0) elastic_tangent(p, Dc);
      point_strain(&s, ve, rate);
      for (int a = 0; a < NS; ++a) {
        double sum = 0.0;
        for (int c = 0; c < NS; ++c) {
          double Dac = p->betaK * dd[a][c];
          if (p->betaKinit != 0.0) Dac += p->betaKinit * D0[a][c];
          if (p->betaKcomm != 0.0) Dac += p->betaKcomm * Dc[a][c];
          sum += Dac * rate[c];
        }
        damp_stress[a] = sum;
      }
    }
    const double rho = p->rho;
    v_gp[0] = v_gp[1] = v_gp[2] = 0.0;
    if (p->alphaM != 0.0 && p->mass_type == 0) {
      for (int j = 0; j < NNODE; j++)
        for (int q = 0; q < 3; q++) v_gp[q] += s.shp[3][j] * ve[3 * j + q];
    }
    for (int j = 0; j < NNODE; j++) {
      double residJ[3], body[3], dampJ[3];
      point_node_force(&s, stress, j, residJ);
      for (int q = 0; q < 3; q++) body[q] = s.dvol * p->b[q] * s.shp[3][j];
      dampJ[0] = dampJ[1] = dampJ[2] = 0.0;
      if (stiff_damping) point_node_force(&s, damp_stress, j, dampJ);
      if (p->alphaM != 0.0) {
        const double temp = s.shp[3][j] * s.dvol * rho;
        for (int q = 0; q < 3; q++) {
          const double vq = p->mass_type == 0 ? v_gp[q] : ve[3 * j + q];
          dampJ[q] += p->alphaM * temp * vq;
        }
      }
      for (int q = 0; q < 3; q++) {
        resid[3 * j + q] += residJ[q];
        resid[3 * j + q] -= body[q];
        fdamp[3 * j + q] += dampJ[q];
      }
    }
    if (Ke) {
      for (int J = 0; J < NNODE; ++J)
        for (int K = 0; K < NNODE; ++K) {
          double st[3][3];
          block_tangent(&s, dd, J, K, st);
          for (int a = 0; a < 3; a++)
            for (int c = 0; c < 3; c++) Ke[(3 * J + a) * NDOF + 3 * K + c] += st[a][c];
        }
    }
  }
  for (int a = 0; a < NDOF; ++a) fe[a] = resid[a] + fdamp[a];
}

/* computeB, std_brick.hpp:698-710, and point_block_tangent, :336-356. */
static void computeB(int node, const point_shape* s, double B[NS][3]) {
  for (int r = 0; r < NS; ++r)
    for (int c = 0; c < 3; ++c) B[r][c] = 0.0;
  B[0][0] = s->shp[0][node];
  B[1][1] = s->shp[1][node];
  B[2][2] = s->shp[2][node];
  B[3][0] = s->shp[1][node];
  B[3][1] = s->shp[0][node];
  B[4][1] = s->shp[2][node];
  B[4][2] = s->shp[1][node];
  B[5][0] = s->shp[2][node];
  B[5][2] = s->shp[0][node];
}
static void block_tangent(const point_shape* s, double dd[NS][NS], int J, int K, double st[3][3]) {
  double BJ[NS][3], BK[NS][3], BJtranD[3][NS];
  computeB(J, s, BJ);
  computeB(K, s, BK);
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < NS; q++) {
      double sum = 0.0;
      for (int r = 0; r < NS; r++) sum += BJ[r][p] * (dd[r][q] * s->dvol);
      BJtranD[p][q] = sum;
    }
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 3; q++) {
      double sum = 0.0;
      for (int r = 0; r < NS; r++) sum += BJtranD[p][r] * BK[r][q];
      st[p][q] = sum;
    }
}

/* ---------------------------------------------------------------- element operator */
/* Factors, src/physics/operators/element_operator.hpp:45-56 (stdBrick: the initial stiffness
 * is not the tangent). k = {stiffness, damping, mass}. */
typedef struct {
  double cK, c0, cc, cM;
} factors;
static factors make_factors(const fxo_param* p, const double* k) {
  factors f;
  f.cK = k[0] + k[1] * p->betaK;
  f.c0 = k[1] * p->betaKinit;
  f.cc = k[1] * p->betaKcomm;
  f.cM = k[2] + k[1] * p->alphaM;
  return f;
}
/* effective_tangent, element_operator.hpp:60-75, with the constant tangent of the parameter set
 * (D = D0 = Dc for the elastic material). */
static void effective_tangent(const factors* f, const fxo_param* p, double Deff[NS][NS]) {
  double D[NS][NS];
  elastic_tangent(p, D);
  for (int a = 0; a < NS; ++a)
    for (int c = 0; c < NS; ++c) {
      double v = f->cK * D[a][c];
      if (f->c0 != 0.0) v += f->c0 * D[a][c];
      if (f->cc != 0.0) v += f->cc * D[a][c];
      Deff[a][c] = v;
    }
}

/* element_operator_apply, element_operator.hpp:82-130, with point_mass_apply
 * (std_brick.hpp:361-374). */
/* Dp[gp]: the effective material matrix of point gp. */
static void brick_operator_pts(const fxo_param* p, const factors* fp, const double* xe, const double* ve,
                               double Dp[NGP][NS][NS], double* ye) {
  const factors f = *fp;
  double xl[3][8];
  local_coords(xe, xl);
  for (int a = 0; a < NDOF; ++a) ye[a] = 0.0;
  for (int gp = 0; gp < NGP; ++gp) {
    point_shape s;
    point_geometry(xl, gp, &s);
    double eps[NS], sig[NS];
    point_strain(&s, ve, eps);
    for (int a = 0; a < NS; ++a) {
      double sum = 0.0;
      for (int c = 0; c < NS; ++c) sum += Dp[gp][a][c] * eps[c];
      sig[a] = sum;
    }
    for (int j = 0; j < NNODE; ++j) {
      double fj[3];
      point_node_force(&s, sig, j, fj);
      for (int q = 0; q < 3; ++q) ye[3 * j + q] += fj[q];
      if (f.cM != 0.0) {
        const double temp = s.shp[3][j] * s.dvol * p->rho;
        double mj[3];
        for (int q = 0; q < 3; q++) {
          double vq;
          if (p->mass_type == 0) {
            vq = 0.0;
            for (int kk = 0; kk < NNODE; kk++) vq += s.shp[3][kk] * ve[3 * kk + q];
          } else {
            vq = ve[3 * j + q];
          }
          mj[q] = temp * vq;
        }
        for (int q = 0; q < 3; ++q) ye[3 * j + q] += f.cM * mj[q];
      }
    }
  }
}

void fxo_brick_operator(const fxo_param* p, const double* k, const double* xe, const double* ve, double* ye) {
  const factors f = make_factors(p, k);
  double Dp[NGP][NS][NS];
  effective_tangent(&f, p, Dp[0]);
  for (int gp = 1; gp < NGP; ++gp) memcpy(Dp[gp], Dp[0], sizeof(Dp[0]));
  brick_operator_pts(p, &f, xe, ve, Dp, ye);
}

/* point_mass_entry, std_brick.hpp:379-383. */
static double mass_entry(const fxo_param* p, const point_shape* s, int j, int k) {
  const double temp = s->shp[3][j] * s->dvol * p->rho;
  if (p->mass_type == 0) return temp * s->shp[3][k];
  return j == k ? temp : 0.0;
}

/* element_operator_diagonal, element_operator.hpp:138-209 (with the merged-equation terms). */
static void brick_diagonal_pts(const fxo_param* p, const factors* fp, const double* xe, const int32_t* eq,
                               double Dp[NGP][NS][NS], double* de) {
  const factors f = *fp;
  double xl[3][8];
  local_coords(xe, xl);
  for (int a = 0; a < NDOF; ++a) de[a] = 0.0;
  int first[NDOF];
  int merged = 0;
  for (int a = 0; a < NDOF; ++a) {
    first[a] = a;
    if (eq[a] < 0) continue;
    for (int b = 0; b < a; ++b)
      if (eq[b] == eq[a]) {
        first[a] = first[b];
        merged = 1;
        break;
      }
  }
  for (int gp = 0; gp < NGP; ++gp) {
    point_shape s;
    point_geometry(xl, gp, &s);
    double (*Deff)[NS] = Dp[gp];
    for (int j = 0; j < NNODE; ++j) {
      double blk[3][3];
      block_tangent(&s, Deff, j, j, blk);
      const double m = f.cM != 0.0 ? f.cM * mass_entry(p, &s, j, j) : 0.0;
      for (int q = 0; q < 3; ++q) de[3 * j + q] += blk[q][q] + m;
    }
    if (!merged) continue;
    for (int J = 0; J < NNODE; ++J)
      for (int K = 0; K < NNODE; ++K) {
        int any = 0;
        for (int a = 0; a < 3 && !any; ++a)
          for (int c = 0; c < 3; ++c) {
            const int ia = 3 * J + a, ic = 3 * K + c;
            if (ia != ic && eq[ia] >= 0 && eq[ia] == eq[ic]) any = 1;
          }
        if (!any) continue;
        double blk[3][3];
        block_tangent(&s, Deff, J, K, blk);
        const double m = (f.cM != 0.0 && J != K) ? f.cM * mass_entry(p, &s, J, K) : 0.0;
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) {
            const int ia = 3 * J + a, ic = 3 * K + c;
            if (ia == ic || eq[ia] < 0 || eq[ia] != eq[ic]) continue;
            de[first[ia]] += blk[a][c] + (a == c ? m : 0.0);
          }
      }
  }
}

void fxo_brick_diagonal(const fxo_param* p, const double* k, const double* xe, const int32_t* eq, double* de) {
  const factors f = make_factors(p, k);
  double Dp[NGP][NS][NS];
  effective_tangent(&f, p, Dp[0]);
  for (int gp = 1; gp < NGP; ++gp) memcpy(Dp[gp], Dp[0], sizeof(Dp[0]));
  brick_diagonal_pts(p, &f, xe, eq, Dp, de);
}

/* StdBrick::mass and lumped_mass, std_brick.hpp:582-623 (row-major 24x24). */
void fxo_brick_mass(const fxo_param* p, const double* xe, double* Me) {
  double xl[3][8];
  local_coords(xe, xl);
  for (int a = 0; a < NDOF * NDOF; ++a) Me[a] = 0.0;
  const double rho = p->rho;
  for (int i = 0; i < NGP; i++) {
    point_shape s;
    point_geometry(xl, i, &s);
    for (int j = 0; j < NNODE; j++) {
      double temp = s.shp[3][j] * s.dvol;
      temp *= rho;
      for (int kk = 0; kk < NNODE; kk++) {
        double mjk;
        if (p->mass_type == 0) {
          mjk = temp * s.shp[3][kk];
        } else {
          if (j != kk) continue;
          mjk = temp;
        }
        for (int q = 0; q < 3; q++) Me[(3 * j + q) * NDOF + 3 * kk + q] += mjk;
      }
    }
  }
}
void fxo_brick_lumped_mass(const fxo_param* p, const double* xe, double* m) {
  double xl[3][8];
  local_coords(xe, xl);
  for (int j = 0; j < NNODE; j++) m[j] = 0.0;
  for (int i = 0; i < NGP; i++) {
    point_shape s;
    point_geometry(xl, i, &s);
    for (int j = 0; j < NNODE; j++) {
      double temp = s.shp[3][j] * s.dvol;
      temp *= p->rho;
      m[j] += temp;
    }
  }
}

/* ---------------------------------------------------------------- system level */
static void element_coords(const fxo_mesh* m, int32_t e, double* xe) {
  for (int a = 0; a < NNODE; ++a) {
    const int32_t n = m->node[(int64_t)a * m->padded + e];
    for (int d = 0; d < 3; ++d) xe[3 * a + d] = m->coords[(int64_t)d * m->num_nodes + n];
  }
}

/* InternalForce::apply_operator (src/exec/internal_force.cpp:545-573) with the gather scatter:
 * the element values are summed per equation in (element, DOF) order (the gather pairs,
 * internal_force.cpp:121-134, summed by SlotGather::gather, assembly.cpp:28-38). A serial
 * scatter in that order makes the same sums. Then the nodal masses (add_nodal_mass, :442-448). */
void fxo_apply_operator(const fxo_mesh* m, const double* k, const double* x, double* y) {
  for (int32_t q = 0; q < m->num_equations; ++q) y[q] = 0.0;
  for (int32_t e = 0; e < m->count; ++e) {
    double xe[24], ve[24], ye[24];
    element_coords(m, e, xe);
    for (int a = 0; a < NDOF; ++a) {
      const int32_t q = m->eq[(int64_t)a * m->padded + e];
      ve[a] = q >= 0 ? x[q] : 0.0;
    }
    fxo_brick_operator(&m->params[m->param[e]], k, xe, ve, ye);
    for (int a = 0; a < NDOF; ++a) {
      const int32_t q = m->eq[(int64_t)a * m->padded + e];
      if (q >= 0) y[q] += ye[a];
    }
  }
  if (k[2] != 0.0 && m->nodal_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) y[q] += k[2] * m->nodal_mass[q] * x[q];
  if (k[1] != 0.0 && m->nodal_alpha_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) y[q] += k[1] * m->nodal_alpha_mass[q] * x[q];
}

/* InternalForce::operator_diagonal, internal_force.cpp:575-599. */
void fxo_operator_diagonal(const fxo_mesh* m, const double* k, double* d) {
  for (int32_t q = 0; q < m->num_equations; ++q) d[q] = 0.0;
  for (int32_t e = 0; e < m->count; ++e) {
    double xe[24], de[24];
    int32_t eqe[24];
    element_coords(m, e, xe);
    for (int a = 0; a < NDOF; ++a) eqe[a] = m->eq[(int64_t)a * m->padded + e];
    fxo_brick_diagonal(&m->params[m->param[e]], k, xe, eqe, de);
    for (int a = 0; a < NDOF; ++a)
      if (eqe[a] >= 0) d[eqe[a]] += de[a];
  }
  if (k[2] != 0.0 && m->nodal_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) d[q] += k[2] * m->nodal_mass[q] * 1.0;
  if (k[1] != 0.0 && m->nodal_alpha_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) d[q] += k[1] * m->nodal_alpha_mass[q] * 1.0;
}

/* InternalForce::compute (internal_force.cpp:354-377) with the flat kernel
 * (element_kernels.hpp:197-235): u and v gathered (fixed DOFs 0), element force, gather
 * scatter, then the nodal masses' alphaM damping. */
void fxo_force(const fxo_mesh* m, const double* u, const double* v, double* f) {
  for (int32_t q = 0; q < m->num_equations; ++q) f[q] = 0.0;
  for (int32_t e = 0; e < m->count; ++e) {
    double xe[24], ue[24], ve[24], fe[24];
    element_coords(m, e, xe);
    for (int a = 0; a < NDOF; ++a) {
      const int32_t q = m->eq[(int64_t)a * m->padded + e];
      ue[a] = q >= 0 ? u[q] : 0.0;
      ve[a] = q >= 0 ? v[q] : 0.0;
    }
    fxo_brick_compute(&m->params[m->param[e]], xe, ue, ve, fe, NULL);
    for (int a = 0; a < NDOF; ++a) {
      const int32_t q = m->eq[(int64_t)a * m->padded + e];
      if (q >= 0) f[q] += fe[a];
    }
  }
  if (m->nodal_alpha_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) f[q] += m->nodal_alpha_mass[q] * v[q];
}

/* InternalForce::mass_times_ground (internal_force.cpp:601-626): y = M r_dir with the unit
 * translation at every element DOF (fixed ones included), plus the free nodal masses. */
void fxo_mass_times_ground(const fxo_mesh* m, int dir, double* y) {
  const double k[3] = {0.0, 0.0, 1.0};
  for (int32_t q = 0; q < m->num_equations; ++q) y[q] = 0.0;
  for (int32_t e = 0; e < m->count; ++e) {
    double xe[24], ve[24], ye[24];
    element_coords(m, e, xe);
    for (int a = 0; a < NDOF; ++a) ve[a] = (a % 3) == dir ? 1.0 : 0.0;
    fxo_brick_operator(&m->params[m->param[e]], k, xe, ve, ye);
    for (int a = 0; a < NDOF; ++a) {
      const int32_t q = m->eq[(int64_t)a * m->padded + e];
      if (q >= 0) y[q] += ye[a];
    }
  }
  if (m->nodal_mass) {
    /* the free nodal masses in direction dir (ground_nodal_mass, internal_force.cpp:621-625);
     * an equation's DOF is its local DOF index mod 3 in any element that has it */
    int8_t* dof = (int8_t*)malloc((size_t)(m->num_equations > 0 ? m->num_equations : 1));
    for (int32_t q = 0; q < m->num_equations; ++q) dof[q] = -1;
    for (int32_t e = 0; e < m->count; ++e)
      for (int a = 0; a < NDOF; ++a) {
        const int32_t q = m->eq[(int64_t)a * m->padded + e];
        if (q >= 0) dof[q] = (int8_t)(a % 3);
      }
    for (int32_t q = 0; q < m->num_equations; ++q)
      if (dof[q] == dir) y[q] += m->nodal_mass[q];
    free(dof);
  }
}

/* ---------------------------------------------------------------- vector kernels */
/* VectorOps::dot's documented order (src/solvers/vector_ops.hpp:5-14, vector_ops.cpp:19-43):
 * chunks of 2048 entries; lane l of `lanes` sums entries l, l+lanes, ... of a chunk; lane 0 adds
 * the lane sums in lane order; levels of chunk sums until one value is left. */
#define KCHUNK 2048
static double* reduce_level(const double* x, const double* y, int64_t n, int lanes, int fused, int64_t* nout) {
  const int64_t nc = (n + KCHUNK - 1) / KCHUNK;
  double* out = (double*)malloc(sizeof(double) * (size_t)(nc > 0 ? nc : 1));
  double* lane = (double*)malloc(sizeof(double) * (size_t)lanes);
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t begin = c * KCHUNK;
    const int64_t len = n - begin < KCHUNK ? n - begin : KCHUNK;
    for (int l = 0; l < lanes; ++l) {
      double s = 0.0;
      for (int64_t k = l; k < len; k += lanes) {
        if (y) s = fused ? fma(x[begin + k], y[begin + k], s) : s + x[begin + k] * y[begin + k];
        else s += x[begin + k];
      }
      lane[l] = s;
    }
    double total = 0.0;
    for (int l = 0; l < lanes; ++l) total += lane[l];
    out[c] = total;
  }
  free(lane);
  *nout = nc;
  return out;
}
double fxo_dot(const double* x, const double* y, int64_t n, int lanes, int fused) {
  if (n == 0) return 0.0;
  int64_t np;
  double* p = reduce_level(x, y, n, lanes, fused, &np);
  while (np > 1) {
    int64_t nn;
    double* q = reduce_level(p, NULL, np, lanes, fused, &nn);
    free(p);
    p = q;
    np = nn;
  }
  const double r = p[0];
  free(p);
  return r;
}

/* ---------------------------------------------------------------- solvers */
/* Jacobi (src/solvers/jacobi.cpp:10-26): inverse of the operator diagonal. */
static double* jacobi_inverse(const fxo_mesh* m, const double* k) {
  const int32_t n = m->num_equations;
  double* d = (double*)malloc(sizeof(double) * (size_t)n);
  fxo_operator_diagonal(m, k, d);
  for (int32_t i = 0; i < n; ++i) d[i] = 1.0 / d[i];
  return d;
}

/* ConjugateGradient::solve, src/solvers/cg.cpp:24-71, with the Jacobi preconditioner. */
void fxo_cg(const fxo_mesh* m, const double* k, const double* b, double* x, double rtol, double atol, int max_it,
            int lanes, double* result) {
  const int32_t n = m->num_equations;
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* z = (double*)malloc(sizeof(double) * (size_t)n);
  double* pd = (double*)malloc(sizeof(double) * (size_t)n);
  double* ap = (double*)malloc(sizeof(double) * (size_t)n);
  double* inv = jacobi_inverse(m, k);
  double conv = 0, iters = 0, indef = 0;
  const double rhs = sqrt(fxo_dot(b, b, n, lanes, 0));
  fxo_apply_operator(m, k, x, ap);
  for (int32_t i = 0; i < n; ++i) r[i] = b[i];
  for (int32_t i = 0; i < n; ++i) r[i] += -1.0 * ap[i];
  double rnorm = sqrt(fxo_dot(r, r, n, lanes, 0));
  const double r0 = rnorm;
  const double tol = rtol * rhs > atol ? rtol * rhs : atol;
  if (rnorm <= tol) {
    conv = 1;
    goto done;
  }
  for (int32_t i = 0; i < n; ++i) z[i] = inv[i] * r[i];
  for (int32_t i = 0; i < n; ++i) pd[i] = z[i];
  double rz = fxo_dot(r, z, n, lanes, 0);
  for (int it = 1; it <= max_it; ++it) {
    fxo_apply_operator(m, k, pd, ap);
    const double pap = fxo_dot(pd, ap, n, lanes, 0);
    if (!(pap > 0.0)) {
      indef = 1;
      iters = it - 1;
      goto done;
    }
    const double alpha = rz / pap;
    for (int32_t i = 0; i < n; ++i) x[i] += alpha * pd[i];
    for (int32_t i = 0; i < n; ++i) r[i] += -alpha * ap[i];
    rnorm = sqrt(fxo_dot(r, r, n, lanes, 0));
    iters = it;
    if (rnorm <= tol) {
      conv = 1;
      goto done;
    }
    for (int32_t i = 0; i < n; ++i) z[i] = inv[i] * r[i];
    const double rz_new = fxo_dot(r, z, n, lanes, 0);
    const double beta = rz_new / rz;
    rz = rz_new;
    for (int32_t i = 0; i < n; ++i) pd[i] = z[i] + beta * pd[i];
  }
done:
  result[0] = conv;
  result[1] = iters;
  result[2] = rhs;
  result[3] = r0;
  result[4] = rnorm;
  result[5] = indef;
  free(r);
  free(z);
  free(pd);
  free(ap);
  free(inv);
}

/* Gmres::solve, src/solvers/gmres.cpp:32-123: FGMRES(m) with Jacobi, CGS2 through the block
 * kernels (BlockOps::dots in the dot order above, BlockOps::combine w += sum_c (a y_c) V_c,
 * src/solvers/block_ops.cpp:59-90), Givens rotations on the host, true residual at every
 * restart and at convergence. */
static void block_dots(const double* V, int64_t n, int k, const double* w, int lanes, double* h) {
  for (int c = 0; c < k; ++c) h[c] = fxo_dot(V + (int64_t)c * n, w, n, lanes, 0);
}
static void block_combine(const double* V, int64_t n, int k, const double* y, double a, double* w) {
  double coef[64];
  for (int c = 0; c < k; ++c) coef[c] = a * y[c];
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int c = 0; c < k; ++c) s += coef[c] * V[(int64_t)c * n + i];
    w[i] += s;
  }
}
void fxo_gmres(const fxo_mesh* m, const double* k, const double* b, double* x, double rtol, double atol, int max_it,
               int lanes, int restart, double* result) {
  const int64_t n = m->num_equations;
  const int M = restart < 1 ? 1 : (restart > 63 ? 63 : restart);
  double* V = (double*)calloc((size_t)(n * (M + 1)), sizeof(double));
  double* Z = (double*)calloc((size_t)(n * M), sizeof(double));
  double* w = (double*)malloc(sizeof(double) * (size_t)n);
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* inv = jacobi_inverse(m, k);
  double H[64 * 65], cs[64], sn[64], g[65], h[64], h2[64], y[64];
#define HIJ(i, j) H[(j) * (M + 1) + (i)]
  int iterations = 0, first = 1, converged = 0;
  double initial = 0.0, final_res = 0.0;
  const double rhs = sqrt(fxo_dot(b, b, n, lanes, 0));
  const double tol = rtol * rhs > atol ? rtol * rhs : atol;
  for (;;) {
    fxo_apply_operator(m, k, x, w);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i];
    for (int64_t i = 0; i < n; ++i) r[i] += -1.0 * w[i];
    const double beta = sqrt(fxo_dot(r, r, n, lanes, 0));
    if (first) initial = beta;
    first = 0;
    final_res = beta;
    if (beta <= tol) {
      converged = 1;
      break;
    }
    if (iterations >= max_it) break;
    for (int64_t i = 0; i < n; ++i) V[i] = 0.0;
    for (int64_t i = 0; i < n; ++i) V[i] += (1.0 / beta) * r[i];
    for (int i = 0; i <= M; ++i) g[i] = 0.0;
    g[0] = beta;
    int j = 0;
    for (; j < M && iterations < max_it; ++j) {
      double* vj = V + (int64_t)j * n;
      double* zj = Z + (int64_t)j * n;
      for (int64_t i = 0; i < n; ++i) zj[i] = inv[i] * vj[i];
      fxo_apply_operator(m, k, zj, w);
      block_dots(V, n, j + 1, w, lanes, h);
      block_combine(V, n, j + 1, h, -1.0, w);
      block_dots(V, n, j + 1, w, lanes, h2);
      block_combine(V, n, j + 1, h2, -1.0, w);
      for (int i = 0; i <= j; ++i) HIJ(i, j) = h[i] + h2[i];
      const double hn = sqrt(fxo_dot(w, w, n, lanes, 0));
      HIJ(j + 1, j) = hn;
      if (hn > 0.0) {
        double* vn = V + (int64_t)(j + 1) * n;
        for (int64_t i = 0; i < n; ++i) vn[i] = 0.0;
        for (int64_t i = 0; i < n; ++i) vn[i] += (1.0 / hn) * w[i];
      }
      for (int i = 0; i < j; ++i) {
        const double a = HIJ(i, j), c = HIJ(i + 1, j);
        HIJ(i, j) = cs[i] * a + sn[i] * c;
        HIJ(i + 1, j) = -sn[i] * a + cs[i] * c;
      }
      const double a = HIJ(j, j), c = HIJ(j + 1, j);
      const double d = hypot(a, c);
      cs[j] = d > 0.0 ? a / d : 1.0;
      sn[j] = d > 0.0 ? c / d : 0.0;
      HIJ(j, j) = d;
      HIJ(j + 1, j) = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      ++iterations;
      final_res = fabs(g[j + 1]);
      if (final_res <= tol || hn == 0.0) {
        ++j;
        break;
      }
    }
    for (int i = j - 1; i >= 0; --i) {
      double s = g[i];
      for (int kk = i + 1; kk < j; ++kk) s -= HIJ(i, kk) * y[kk];
      y[i] = s / HIJ(i, i);
    }
    block_combine(Z, n, j, y, 1.0, x);
    if (final_res <= tol) {
      fxo_apply_operator(m, k, x, w);
      for (int64_t i = 0; i < n; ++i) r[i] = b[i];
      for (int64_t i = 0; i < n; ++i) r[i] += -1.0 * w[i];
      final_res = sqrt(fxo_dot(r, r, n, lanes, 0));
      if (final_res <= tol) {
        converged = 1;
        break;
      }
    }
    if (iterations >= max_it) break;
  }
#undef HIJ
  result[0] = converged;
  result[1] = iterations;
  result[2] = rhs;
  result[3] = initial;
  result[4] = final_res;
  result[5] = 0;
  free(V);
  free(Z);
  free(w);
  free(r);
  free(inv);
}

/* ---------------------------------------------------------------- time stepping */
/* One ExplicitDifference step: ed_predict (explicit_analysis.cpp:62-69), the force at
 * (u, vh), ed_correct (:72-84) with the UniformExcitation load ground_load (:52-58): the
 * pattern acting along equation q's DOF loads it with -m_q ag. */
void fxo_ed_step(const fxo_mesh* m, const double* mass, const int8_t* eq_dof, const double* ag, double dt, double* u,
                 double* vh, double* a, double* v_rec, double* f) {
  const int32_t n = m->num_equations;
  for (int32_t q = 0; q < n; ++q) {
    vh[q] += a[q] * dt;
    u[q] += vh[q] * dt;
  }
  fxo_force(m, u, vh, f);
  const double halfT = dt * 0.125;
  for (int32_t q = 0; q < n; ++q) {
    double gl = 0.0;
    for (int p = 0; p < 3; ++p)
      if (ag && ag[p] != 0.0 && eq_dof[q] == p) gl -= mass[q] * ag[p];
    const double R = -f[q] + gl;
    const double a_new = R / mass[q];
    const double t = 3.0 * a_new + a[q];
    v_rec[q] = vh[q] + t * halfT;
    a[q] = a_new;
  }
}

/* ---------------------------------------------------------------- ground motions and stages */
/* PathSeries::getFactor, uniform spacing (src/exec/ground_motion.cpp:21-39): 0 before the start,
 * linear between samples floor(incr) and floor(incr) + 1, the last value (useLast) or 0 after. */
double fxo_path_uniform(const double* values, int64_t n, double dt, double factor, double start, int use_last,
                        double t) {
  if (t < start) return 0.0;
  const double incr = (t - start) / dt;
  const long long i1 = (long long)floor(incr);
  const long long i2 = i1 + 1;
  if (i2 >= n) return use_last ? factor * values[n - 1] : 0.0;
  const double v1 = values[i1], v2 = values[i2];
  return factor * (v1 + (v2 - v1) * (incr - (double)i1));
}

/* PathTimeSeries::getFactor (ground_motion.cpp:41-77): the interval walk from *loc, forwards or
 * backwards, kept for the next call; 0 outside the times. */
double fxo_path_time(const double* values, const double* times, int64_t n, double factor, int* loc, double t) {
  int l = *loc;
  double t1 = times[l];
  if (t < t1 && l == 0) return 0.0;
  if (t == t1) return factor * values[l];
  const int last = (int)n - 1;
  if (t > t1 && l == last) return 0.0;
  double t2 = times[l + 1];
  if (t > t2) {
    while (t > t2 && l < last - 1) {
      ++l;
      t1 = t2;
      t2 = times[l + 1];
    }
    *loc = l;
    if (t > t2) return 0.0;
  } else if (t < t1) {
    while (t < t1 && l > 0) {
      --l;
      t2 = t1;
      t1 = times[l];
    }
    *loc = l;
    if (t < t1) return 0.0;
  }
  const double v1 = values[l], v2 = values[l + 1];
  return factor * (v1 + (v2 - v1) * (t - t1) / (t2 - t1));
}

/* ground_load (explicit_analysis.cpp:51-58): -m accel(p) for every pattern acting in the DOF */
static double ground_load(double mq, int dof_q, const double* accel, const int32_t* gdof, int npat) {
  double r = 0.0;
  for (int p = 0; p < npat; ++p)
    if (gdof[p] == dof_q) r -= mq * accel[p];
  return r;
}

/* ed_predict, force, ed_correct (explicit_analysis.cpp:62-84 in the order of :700-711) */
void fxo_ed_stage_step(const fxo_mesh* m, const double* mass, const int8_t* eq_dof, const double* accel,
                       const int32_t* gdof, int npat, double dt, double* u, double* vh, double* a, double* v_rec,
                       double* f) {
  const int32_t n = m->num_equations;
  for (int32_t q = 0; q < n; ++q) {
    vh[q] += a[q] * dt;
    u[q] += vh[q] * dt;
  }
  fxo_force(m, u, vh, f);
  const double halfT = dt * 0.125;
  for (int32_t q = 0; q < n; ++q) {
    const double R = -f[q] + ground_load(mass[q], eq_dof[q], accel, gdof, npat);
    const double a_new = R / mass[q];
    const double t = 3.0 * a_new + a[q];
    v_rec[q] = vh[q] + t * halfT;
    a[q] = a_new;
  }
}

/* cd_garbage_velocity, force, cd_solve (explicit_analysis.cpp:86-117 in the order of :712-721),
 * c2 = 0.5 / dt, c3 = 1 / dt^2 (:673) */
void fxo_cd_stage_step(const fxo_mesh* m, const double* mass, const double* cm, const int8_t* eq_dof,
                       const double* accel, const int32_t* gdof, int npat, double dt, double* u, double* um,
                       double* v_elem, double* a, double* v_rec, double* f) {
  const int32_t n = m->num_equations;
  const double c2 = 0.5 / dt, c3 = 1.0 / (dt * dt);
  for (int32_t q = 0; q < n; ++q) v_elem[q] = um[q] * -c2;
  fxo_force(m, u, v_elem, f);
  for (int32_t q = 0; q < n; ++q) {
    const double ag = u[q] * (-2.0 * c3) + um[q] * c3;
    const double R = -f[q] - mass[q] * ag + ground_load(mass[q], eq_dof[q], accel, gdof, npat);
    const double A = mass[q] * c3 + cm[q] * c2;
    const double U = R / A;
    double Ud = U * 3.0;
    Ud += u[q] * -4.0;
    Ud += um[q];
    Ud *= c2;
    const double Udd = (Ud - v_rec[q]) / dt;
    um[q] = u[q];
    u[q] = U;
    v_rec[q] = Ud;
    a[q] = Udd;
  }
}

void fxo_newmark_predict(int64_t n, double* u, double* v, double* a, double* ut, double* vt, double* at, double a1,
                         double a2, double a3, double a4) {
  for (int64_t q = 0; q < n; ++q) {
    ut[q] = u[q];
    vt[q] = v[q];
    at[q] = a[q];
    v[q] = v[q] * a1 + at[q] * a2;
    a[q] = a[q] * a4 + vt[q] * a3;
  }
}

void fxo_newmark_update(int64_t n, const double* du, double* u, double* v, double* a, double c2, double c3) {
  for (int64_t q = 0; q < n; ++q) {
    u[q] += du[q];
    v[q] += du[q] * c2;
    a[q] += du[q] * c3;
  }
}

/* ---------------------------------------------------------------- J2 */
int fxo_j2_update(double E, double nu, double sigma_y, double H, double hk, const double* committed, double* trial,
                  const double* eps, double* sigma, double* D) {
  const double K = E / (3.0 * (1.0 - 2.0 * nu));
  const double G = E / (2.0 * (1.0 + nu));
  const double Hkin = hk * H, Hiso = (1.0 - hk) * H;
  /* tensor components (shear halved) of the elastic strain */
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
  const double f = nxi - r23 * (sigma_y + Hiso * alpha);
  for (int i = 0; i < 13; ++i) trial[i] = committed[i];
  for (int i = 0; i < 36; ++i) D[i] = 0.0;
  const double p = K * tr;
  if (f <= 0.0 || nxi == 0.0) {
    for (int i = 0; i < 6; ++i) sigma[i] = s_tr[i] + (i < 3 ? p : 0.0);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) D[i * 6 + j] = K + 2.0 * G * ((i == j ? 1.0 : 0.0) - 1.0 / 3.0);
    for (int i = 3; i < 6; ++i) D[i * 6 + i] = G;
    return 0;
  }
  const double dg = f / (2.0 * G + (2.0 / 3.0) * H);
  double n[6];
  for (int i = 0; i < 6; ++i) n[i] = xi[i] / nxi;
  for (int i = 0; i < 6; ++i) sigma[i] = s_tr[i] - 2.0 * G * dg * n[i] + (i < 3 ? p : 0.0);
  for (int i = 0; i < 6; ++i) trial[i] = committed[i] + (i < 3 ? 1.0 : 2.0) * dg * n[i];
  trial[6] = alpha + r23 * dg;
  for (int i = 0; i < 6; ++i) trial[7 + i] = back[i] + (2.0 / 3.0) * Hkin * dg * n[i];
  const double theta = 1.0 - 2.0 * G * dg / nxi;
  const double thetab = 1.0 / (1.0 + H / (3.0 * G)) - (1.0 - theta);
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double idev;
      if (i < 3 && j < 3) idev = (i == j ? 1.0 : 0.0) - 1.0 / 3.0;
      else idev = (i == j) ? 0.5 : 0.0;
      const double vol = (i < 3 && j < 3) ? K : 0.0;
      D[i * 6 + j] = vol + 2.0 * G * theta * idev - 2.0 * G * thetab * n[i] * n[j];
    }
  return 1;
}

/* ---------------------------------------------------------------- J2 system level
 * No counterpart in the reference. j2[4 * s] = {kind (0 elastic, 1 J2), sigma_y, H, hk} of
 * parameter set s. Per element and Gauss point, component c of point gp of element e is at
 * [(c * 8 + gp) * padded + e]: the committed and trial states (13 components) and the point's
 * consistent tangent of the last force evaluation (36 components, row-major). Elastic sets use the
 * elastic element routines above. */
static int is_j2(const double* j2, int32_t s) { return j2[4 * s] == 1.0; }

/* The J2 element force: fxo_brick_compute's sums with the return-mapped stress (no stiffness-
 * proportional damping on J2 sets). */
static int brick_force_j2(const fxo_param* p, const double* j2p, const double* xe, const double* ue,
                          const double* ve, const double* committed, double* trial, double* Dpts, int64_t stride,
                          double* fe) {
  double xl[3][8];
  local_coords(xe, xl);
  double resid[NDOF], fdamp[NDOF];
  for (int a = 0; a < NDOF; ++a) resid[a] = fdamp[a] = 0.0;
  int plastic = 0;
  for (int i = 0; i < NGP; i++) {
    point_shape s;
    point_geometry(xl, i, &s);
    double strain[NS], stress[NS], D[NS * NS], cst[13], tst[13], v_gp[3];
    point_strain(&s, ue, strain);
    for (int c = 0; c < 13; ++c) cst[c] = committed[(c * 8 + i) * stride];
    plastic += fxo_j2_update(p->E, p->nu, j2p[1], j2p[2], j2p[3], cst, tst, strain, stress, D);
    for (int c = 0; c < 13; ++c) trial[(c * 8 + i) * stride] = tst[c];
    for (int c = 0; c < 36; ++c) Dpts[(c * 8 + i) * stride] = D[c];
    v_gp[0] = v_gp[1] = v_gp[2] = 0.0;
    if (p->alphaM != 0.0 && p->mass_type == 0)
      for (int j = 0; j < NNODE; j++)
        for (int q = 0; q < 3; q++) v_gp[q] += s.shp[3][j] * ve[3 * j + q];
    for (int j = 0; j < NNODE; j++) {
      double residJ[3], body[3], dampJ[3];
      point_node_force(&s, stress, j, residJ);
      for (int q = 0; q < 3; q++) body[q] = s.dvol * p->b[q] * s.shp[3][j];
      dampJ[0] = dampJ[1] = dampJ[2] = 0.0;
      if (p->alphaM != 0.0) {
        const double temp = s.shp[3][j] * s.dvol * p->rho;
        for (int q = 0; q < 3; q++) {
          const double vq = p->mass_type == 0 ? v_gp[q] : ve[3 * j + q];
          dampJ[q] += p->alphaM * temp * vq;
        }
      }
      for (int q = 0; q < 3; q++) {
        resid[3 * j + q] += residJ[q];
        resid[3 * j + q] -= body[q];
        fdamp[3 * j + q] += dampJ[q];
      }
    }
  }
  for (int a = 0; a < NDOF; ++a) fe[a] = resid[a] + fdamp[a];
  return plastic;
}

void fxo_force_j2(const fxo_mesh* m, const double* j2, const double* committed, double* trial, double* Dpts,
                  const double* u, const double* v, double* f, int* plastic) {
  int np = 0;
  for (int32_t q = 0; q < m->num_equations; ++q) f[q] = 0.0;
  for (int32_t e = 0; e < m->count; ++e) {
    double xe[24], ue[24], ve[24], fe[24];
    element_coords(m, e, xe);
    for (int a = 0; a < NDOF; ++a) {
      const int32_t q = m->eq[(int64_t)a * m->padded + e];
      ue[a] = q >= 0 ? u[q] : 0.0;
      ve[a] = q >= 0 ? v[q] : 0.0;
    }
    const int32_t ps = m->param[e];
    if (is_j2(j2, ps))
      np += brick_force_j2(&m->params[ps], j2 + 4 * ps, xe, ue, ve, committed + e, trial + e, Dpts + e, m->padded, fe);
    else
      fxo_brick_compute(&m->params[ps], xe, ue, ve, fe, NULL);
    for (int a = 0; a < NDOF; ++a) {
      const int32_t q = m->eq[(int64_t)a * m->padded + e];
      if (q >= 0) f[q] += fe[a];
    }
  }
  if (m->nodal_alpha_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) f[q] += m->nodal_alpha_mass[q] * v[q];
  *plastic = np;
}

/* Effective matrices of a J2 element's points: cK D_t (or cK D_elastic with `initial`). */
static void j2_point_matrices(const fxo_param* p, const double* j2p, const factors* f, const double* Dpts,
                              int64_t stride, int initial, double Dp[NGP][NS][NS]) {
  double De[NS * NS], sig[NS], cst[13] = {0}, tst[13];
  const double zero[NS] = {0, 0, 0, 0, 0, 0};
  if (initial) fxo_j2_update(p->E, p->nu, j2p[1], j2p[2], j2p[3], cst, tst, zero, sig, De);
  for (int gp = 0; gp < NGP; ++gp)
    for (int a = 0; a < NS; ++a)
      for (int c = 0; c < NS; ++c) {
        const double D = initial ? De[a * NS + c] : Dpts[((a * NS + c) * 8 + gp) * stride];
        Dp[gp][a][c] = f->cK * D;
      }
}

void fxo_apply_j2(const fxo_mesh* m, const double* j2, const double* Dpts, const double* k, int initial,
                  const double* x, double* y) {
  for (int32_t q = 0; q < m->num_equations; ++q) y[q] = 0.0;
  for (int32_t e = 0; e < m->count; ++e) {
    double xe[24], ve[24], ye[24];
    element_coords(m, e, xe);
    for (int a = 0; a < NDOF; ++a) {
      const int32_t q = m->eq[(int64_t)a * m->padded + e];
      ve[a] = q >= 0 ? x[q] : 0.0;
    }
    const int32_t ps = m->param[e];
    const fxo_param* p = &m->params[ps];
    if (is_j2(j2, ps)) {
      const factors f = make_factors(p, k);
      double Dp[NGP][NS][NS];
      j2_point_matrices(p, j2 + 4 * ps, &f, Dpts + e, m->padded, initial, Dp);
      brick_operator_pts(p, &f, xe, ve, Dp, ye);
    } else {
      fxo_brick_operator(p, k, xe, ve, ye);
    }
    for (int a = 0; a < NDOF; ++a) {
      const int32_t q = m->eq[(int64_t)a * m->padded + e];
      if (q >= 0) y[q] += ye[a];
    }
  }
  if (k[2] != 0.0 && m->nodal_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) y[q] += k[2] * m->nodal_mass[q] * x[q];
  if (k[1] != 0.0 && m->nodal_alpha_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) y[q] += k[1] * m->nodal_alpha_mass[q] * x[q];
}

void fxo_diagonal_j2(const fxo_mesh* m, const double* j2, const double* Dpts, const double* k, int initial,
                     double* d) {
  for (int32_t q = 0; q < m->num_equations; ++q) d[q] = 0.0;
  for (int32_t e = 0; e < m->count; ++e) {
    double xe[24], de[24];
    int32_t eqe[24];
    element_coords(m, e, xe);
    for (int a = 0; a < NDOF; ++a) eqe[a] = m->eq[(int64_t)a * m->padded + e];
    const int32_t ps = m->param[e];
    const fxo_param* p = &m->params[ps];
    if (is_j2(j2, ps)) {
      const factors f = make_factors(p, k);
      double Dp[NGP][NS][NS];
      j2_point_matrices(p, j2 + 4 * ps, &f, Dpts + e, m->padded, initial, Dp);
      brick_diagonal_pts(p, &f, xe, eqe, Dp, de);
    } else {
      fxo_brick_diagonal(p, k, xe, eqe, de);
    }
    for (int a = 0; a < NDOF; ++a)
      if (eqe[a] >= 0) d[eqe[a]] += de[a];
  }
  if (k[2] != 0.0 && m->nodal_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) d[q] += k[2] * m->nodal_mass[q] * 1.0;
  if (k[1] != 0.0 && m->nodal_alpha_mass)
    for (int32_t q = 0; q < m->num_equations; ++q) d[q] += k[1] * m->nodal_alpha_mass[q] * 1.0;
}

void fxo_libm_eval(int fn, const double* x, const double* y, double* out, int64_t n) {
  for (int64_t i = 0; i < n; ++i)
    out[i] = fn == 0 ? exp(x[i]) : fn == 1 ? log(x[i]) : fn == 2 ? pow(x[i], y[i]) : cos(x[i]);
}
