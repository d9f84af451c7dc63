// SSPbrick: the 8-node brick with one integration point and physical hourglass stabilization
// (McGann, Arduino and Mackenzie-Helnwein's stabilized single-point brick; OpenSees' SSPbrick), as
// the reference runs it (src/physics/elements/ssp_brick.hpp). One `__host__ __device__` definition
// used by the Gauss-point path's kernels, the element-constant setup kernel and the compile step.
//
// Per element (small strain: the reference geometry never changes), computed once:
//   geometry  dNmod (the rows of Bnot: modified shape-function derivatives), the volume mVol and
//             each node's volume weight (the integral of N_i, 2 x 2 x 2 Gauss: mass and body
//             force), kGeo values;
//   constants the four hourglass vectors gamma_g (Mben's rows) and the upper triangle of the
//             12 x 12 matrix interior = FCF - KuT FeCFe^-1 FeCFhg from the material's initial
//             tangent (C1 = lambda + 2 mu, C2 = lambda, C3 = mu), kCon values.
// Per evaluation: strain = Bnot u at the one point, node force mVol Bnot^T stress, and the
// stabilization Kstab u = Mben^T (interior (Mben u)) without forming the 24 x 24 matrix.
//
// How the stabilization matrix is built here. Every entry of FCF, FeCFe and FeCFhg is an
// isotropic contraction of a 3 x 3 "moment" matrix Q(X, Y) = sum of w * Jinv[m][X] Jinv[n][Y]
// (the Jacobian inverse's rows m, n; w a combination of the Jacobian determinant's polynomial
// coefficients J[0..19]). Each family of moments is a short list of (w, m, n, symmetric) terms,
// and the blocks follow from three index rules:
//   full      (i == k) C1 Q(i, i) + C3 (Q(j, j) + Q(l, l)),  (i != k) C2 Q(i, k) + C3 Q(k, i)
//             (C4 Q(i, k) for a symmetric family, C4 = C2 + C3),
//   shear     (i == k) C3 (Q(j, j) + Q(l, l)),                (i != k) C3 Q(i, k),
// with {j, l} the other two indices; the enhanced-strain coefficients C_mn are the full rule on
// Q = Jinv[m][.] Jinv[n][.]. The term lists, the evaluation order of every sum and product, and
// the LU inverses are those of the reference (which follows OpenSees' GetStab), so the constants
// are the reference's bit for bit.
#pragma once

#include <cmath>

#include "brick_gp.cuh"

namespace fx {
namespace ssp {

constexpr int kGeo = 24 + 1 + 8;  // dNmod (node-major), mVol, nodeVol
constexpr int kCon = 32 + 78;     // gamma vectors (8 each: st, ut, us, stu), interior's upper triangle

// Corner signs of node i in stdBrick order: (-,-,-) (+,-,-) (+,+,-) (-,+,-), then z = +.
FX_HD double corner_sign(int i, int axis) {
  if (axis == 0) return (i == 1 || i == 2 || i == 5 || i == 6) ? 1.0 : -1.0;
  if (axis == 1) return (i == 2 || i == 3 || i == 6 || i == 7) ? 1.0 : -1.0;
  return i >= 4 ? 1.0 : -1.0;
}

// The natural-coordinate and hourglass vectors, value at node i (all +-1/8):
// v = 0 xi, 1 eta, 2 zeta, 3 hut (eta zeta), 4 hus (xi zeta), 5 hst (xi eta), 6 hstu (xi eta zeta).
FX_HD double basis(int v, int i) {
  const double sx = corner_sign(i, 0), sy = corner_sign(i, 1), sz = corner_sign(i, 2);
  double s;
  switch (v) {
    case 0: s = sx; break;
    case 1: s = sy; break;
    case 2: s = sz; break;
    case 3: s = sy * sz; break;
    case 4: s = sx * sz; break;
    case 5: s = sx * sy; break;
    default: s = sx * sy * sz; break;
  }
  return 0.125 * s;
}

FX_HD double dot8v(const double* x, int v) {
  double r = 0.0;
  for (int i = 0; i < 8; i++) r += x[i] * basis(v, i);
  return r;
}

// f a . (b x c), the scaled first vector formed first (f = 1, -1 or 2: exact).
FX_HD double triple(double f, const double a[3], const double b[3], const double c[3]) {
  const double fa[3] = {f * a[0], f * a[1], f * a[2]};
  const double t[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
  double r = 0.0;
  for (int k = 0; k < 3; k++) r += fa[k] * t[k];
  return r;
}

// The Jacobian determinant's polynomial coefficients as sums of triple products of the seven
// coefficient vectors e1..e7 (e_v = (x, y, z) . basis v): J[k] = sum f e_a . (e_b x e_c).
struct TripleTerm {
  signed char f, a, b, c;
};
struct TripleSum {
  int n;
  TripleTerm t[3];
};
// (vectors 1..7: 1 xi, 2 eta, 3 zeta, 4 hut, 5 hus, 6 hst, 7 hstu)
FX_HD TripleSum jacobian_term(int k) {
  switch (k) {
    case 0: return {1, {{1, 1, 2, 3}}};
    case 4: return {3, {{1, 7, 2, 3}, {1, 4, 5, 2}, {1, 4, 3, 6}}};
    case 5: return {3, {{1, 1, 7, 3}, {1, 4, 5, 1}, {1, 3, 5, 6}}};
    case 6: return {3, {{1, 1, 2, 7}, {1, 4, 1, 6}, {1, 2, 5, 6}}};
    case 7: return {1, {{-1, 1, 5, 6}}};
    case 8: return {1, {{-1, 4, 2, 6}}};
    case 9: return {1, {{-1, 4, 5, 3}}};
    case 10: return {1, {{1, 2, 4, 7}}};
    case 11: return {1, {{-1, 3, 4, 7}}};
    case 12: return {1, {{1, 3, 5, 7}}};
    case 13: return {1, {{-1, 1, 5, 7}}};
    case 14: return {1, {{1, 1, 6, 7}}};
    case 15: return {1, {{-1, 2, 6, 7}}};
    case 16: return {1, {{2, 4, 5, 6}}};
    case 17: return {1, {{1, 7, 5, 6}}};
    case 18: return {1, {{1, 4, 7, 6}}};
    case 19: return {1, {{1, 4, 5, 7}}};
    default: return {0, {}};  // J[1..3] are zero (OpenSees sets them so)
  }
}

// Square matrix inverse by LU with partial pivoting (Doolittle, rows swapped on the largest
// pivot), then one forward and one backward substitution per column of the identity. Returns
// false on a zero pivot.
template <int N>
FX_HD bool lu_inverse(const double (&A)[N][N], double (&Ai)[N][N]) {
  double L[N][N];
  int piv[N];
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) L[i][j] = A[i][j];
  for (int k = 0; k < N; ++k) {
    int p = k;
    double big = fabs(L[k][k]);
    for (int i = k + 1; i < N; ++i)
      if (fabs(L[i][k]) > big) {
        big = fabs(L[i][k]);
        p = i;
      }
    piv[k] = p;
    if (big == 0.0) return false;
    if (p != k)
      for (int j = 0; j < N; ++j) {
        const double t = L[k][j];
        L[k][j] = L[p][j];
        L[p][j] = t;
      }
    const double r = 1.0 / L[k][k];
    for (int i = k + 1; i < N; ++i) {
      L[i][k] *= r;
      const double m = L[i][k];
      for (int j = k + 1; j < N; ++j) L[i][j] -= m * L[k][j];
    }
  }
  for (int c = 0; c < N; ++c) {
    double x[N];
    for (int i = 0; i < N; ++i) x[i] = (i == c) ? 1.0 : 0.0;
    for (int k = 0; k < N; ++k)
      if (piv[k] != k) {
        const double t = x[k];
        x[k] = x[piv[k]];
        x[piv[k]] = t;
      }
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < i; ++j) x[i] -= L[i][j] * x[j];
    for (int i = N - 1; i >= 0; --i) {
      for (int j = i + 1; j < N; ++j) x[i] -= L[i][j] * x[j];
      x[i] /= L[i][i];
    }
    for (int i = 0; i < N; ++i) Ai[i][c] = x[i];
  }
  return true;
}

struct Frame {
  double J[20];
  double vol;
  double dN[8][3];
  double Jinv[3][3];
  double gamma[4][8];  // hourglass vectors: st, ut, us, stu
};

// One component of Bnot's row vector at every node, from the coefficient arrays P, Q of the two
// other axes (x: P = y-coefficients, Q = z-coefficients; y: z, x; z: x, y), index 1..7.
FX_HD void bnot_component(const double* P, const double* Q, double vol, double out[8]) {
  const double u1 = P[2] * Q[3] - Q[2] * P[3], u2 = P[3] * Q[1] - Q[3] * P[1], u3 = P[1] * Q[2] - Q[1] * P[2];
  const double w1 = P[6] * Q[5] - Q[6] * P[5], w2 = P[4] * Q[6] - Q[4] * P[6], w3 = P[5] * Q[4] - Q[5] * P[4];
  for (int i = 0; i < 8; i++) {
    const double xi = basis(0, i), et = basis(1, i), ze = basis(2, i);
    const double hst = basis(5, i), hut = basis(3, i), hus = basis(4, i);
    out[i] = (8.0 * (u1 * xi + u2 * et + u3 * ze) +
              (8.0 / 3.0) * (w1 * xi + w2 * et + w3 * ze + (P[5] * Q[1] - Q[5] * P[1] + P[2] * Q[4] - Q[2] * P[4]) * hst +
                             (P[6] * Q[2] - Q[6] * P[2] + P[3] * Q[5] - Q[3] * P[5]) * hut +
                             (P[1] * Q[6] - Q[1] * P[6] + P[4] * Q[3] - Q[4] * P[3]) * hus)) /
             vol;
  }
}

// GetStab's geometry (no material): J[], mVol, dNmod and, with `hourglass`, Jinv and the gamma
// vectors (G = I - dNmod X, gamma_g = G h_g).
FX_HD void frame(const double xl[3][8], Frame& f, bool hourglass) {
  double co[3][8];  // co[d][v], v = 1..7
  for (int d = 0; d < 3; ++d) {
    co[d][0] = 0.0;
    for (int v = 1; v <= 7; ++v) co[d][v] = dot8v(xl[d], v - 1);
  }
  for (int k = 0; k < 20; ++k) {
    const TripleSum s = jacobian_term(k);
    double r = 0.0;
    for (int q = 0; q < s.n; ++q) {
      const TripleTerm& t = s.t[q];
      const double a[3] = {co[0][t.a], co[1][t.a], co[2][t.a]};
      const double b[3] = {co[0][t.b], co[1][t.b], co[2][t.b]};
      const double c[3] = {co[0][t.c], co[1][t.c], co[2][t.c]};
      const double v = triple(static_cast<double>(t.f), a, b, c);
      r = q == 0 ? v : r + v;
    }
    f.J[k] = s.n ? r : 0.0;
  }
  f.vol = 8.0 * (f.J[0] + (f.J[7] + f.J[8] + f.J[9]) / 3.0);
  double bx[8], by[8], bz[8];
  bnot_component(co[1], co[2], f.vol, bx);
  bnot_component(co[2], co[0], f.vol, by);
  bnot_component(co[0], co[1], f.vol, bz);
  for (int i = 0; i < 8; ++i) {
    f.dN[i][0] = bx[i];
    f.dN[i][1] = by[i];
    f.dN[i][2] = bz[i];
  }
  if (!hourglass) return;
  double Jm[3][3];
  for (int d = 0; d < 3; ++d)
    for (int v = 0; v < 3; ++v) {
      double s = 0.0;
      for (int i = 0; i < 8; ++i) s += xl[d][i] * basis(v, i);
      Jm[d][v] = s;
    }
  if (!lu_inverse<3>(Jm, f.Jinv))
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) f.Jinv[a][c] = 0.0;
  double G[8][8];
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += f.dN[i][k] * xl[k][j];
      G[i][j] = (i == j ? 1.0 : 0.0) - s;
    }
  const int hv[4] = {5, 3, 4, 6};  // st, ut, us, stu
  for (int i = 0; i < 8; ++i)
    for (int g = 0; g < 4; ++g) {
      double s = 0.0;
      for (int j = 0; j < 8; ++j) s += G[i][j] * basis(hv[g], j);
      f.gamma[g][i] = s;
    }
}

// ---- the stabilization matrix
// Weights of the moments, combinations of J[] (index into the array from weights()).
enum Weight : int {
  W0789, W0879, W0978, W417, W518, W619, W11215, W11512, W21114, W21411, W31013, W31310, W789, W897, W798,
  W174, W185, W196, W16, kWeights
};
FX_HD void weights(const double* J, double* w) {
  w[W0789] = 8.0 * (J[0] / 3.0 + J[7] / 5.0 + J[8] / 9.0 + J[9] / 9.0);
  w[W0879] = 8.0 * (J[0] / 3.0 + J[8] / 5.0 + J[7] / 9.0 + J[9] / 9.0);
  w[W0978] = 8.0 * (J[0] / 3.0 + J[9] / 5.0 + J[7] / 9.0 + J[8] / 9.0);
  w[W417] = 8.0 * (J[4] / 9.0 + J[17] / 27.0);
  w[W518] = 8.0 * (J[5] / 9.0 + J[18] / 27.0);
  w[W619] = 8.0 * (J[6] / 9.0 + J[19] / 27.0);
  w[W11215] = 8.0 * (J[1] / 9.0 + J[12] / 15.0 + J[15] / 27.0);
  w[W11512] = 8.0 * (J[1] / 9.0 + J[15] / 15.0 + J[12] / 27.0);
  w[W21114] = 8.0 * (J[2] / 9.0 + J[11] / 15.0 + J[14] / 27.0);
  w[W21411] = 8.0 * (J[2] / 9.0 + J[14] / 15.0 + J[11] / 27.0);
  w[W31013] = 8.0 * (J[3] / 9.0 + J[10] / 15.0 + J[13] / 27.0);
  w[W31310] = 8.0 * (J[3] / 9.0 + J[13] / 15.0 + J[10] / 27.0);
  w[W789] = 8.0 * (J[0] / 9.0 + J[7] / 15.0 + J[8] / 15.0 + J[9] / 27.0);
  w[W897] = 8.0 * (J[0] / 9.0 + J[8] / 15.0 + J[9] / 15.0 + J[7] / 27.0);
  w[W798] = 8.0 * (J[0] / 9.0 + J[7] / 15.0 + J[9] / 15.0 + J[8] / 27.0);
  w[W174] = 8.0 * (J[4] / 27.0 + 64.0 * J[17] / 45.0);
  w[W185] = 8.0 * (J[5] / 27.0 + 64.0 * J[18] / 45.0);
  w[W196] = 8.0 * (J[6] / 27.0 + 64.0 * J[19] / 45.0);
  w[W16] = 8.0 * J[16] / 27.0;
}

// A moment family: terms w Jinv[m][X] Jinv[n][Y], or, symmetric, w (Jinv[m][X] Jinv[n][Y] +
// Jinv[n][X] Jinv[m][Y]), summed in list order.
struct MomentTerm {
  signed char w, m, n, sym;
};
struct Moment {
  int n;
  MomentTerm t[6];
};
// Families: 0 Hst, 1 Hut, 2 Hus (st, ut, us with themselves), 3 Itt (st-ut), 4 Iss (st-us),
// 5 Iuu (ut-us), 6 Ist (st-stu), 7 Iut (ut-stu), 8 Ius (us-stu), 9 Hstu (stu with itself).
FX_HD Moment moment(int family) {
  switch (family) {
    case 0: return {3, {{W0879, 0, 0, 0}, {W0789, 1, 1, 0}, {W619, 0, 1, 1}}};
    case 1: return {3, {{W0978, 1, 1, 0}, {W0879, 2, 2, 0}, {W417, 1, 2, 1}}};
    case 2: return {3, {{W0978, 0, 0, 0}, {W0789, 2, 2, 0}, {W518, 0, 2, 1}}};
    case 3: return {4, {{W0879, 0, 2, 0}, {W417, 0, 1, 0}, {W518, 1, 1, 0}, {W619, 1, 2, 0}}};
    case 4: return {4, {{W0789, 1, 2, 0}, {W417, 0, 0, 0}, {W518, 1, 0, 0}, {W619, 0, 2, 0}}};
    case 5: return {4, {{W0978, 1, 0, 0}, {W417, 2, 0, 0}, {W518, 1, 2, 0}, {W619, 2, 2, 0}}};
    case 6: return {5, {{W31013, 0, 0, 0}, {W31310, 1, 1, 0}, {W21411, 2, 1, 0}, {W11512, 2, 0, 0}, {W16, 0, 1, 1}}};
    case 7: return {5, {{W21114, 0, 1, 0}, {W31013, 0, 2, 0}, {W11215, 1, 1, 0}, {W11512, 2, 2, 0}, {W16, 1, 2, 1}}};
    case 8: return {5, {{W21114, 0, 0, 0}, {W11215, 1, 0, 0}, {W31310, 1, 2, 0}, {W21411, 2, 2, 0}, {W16, 0, 2, 1}}};
    default:
      return {6, {{W897, 0, 0, 0}, {W798, 1, 1, 0}, {W789, 2, 2, 0}, {W185, 0, 2, 1}, {W196, 0, 1, 1}, {W174, 1, 2, 1}}};
  }
}

FX_HD void moment_matrix(int family, const double* w, const double Ji[3][3], double Q[3][3]) {
  const Moment M = moment(family);
  for (int X = 0; X < 3; ++X)
    for (int Y = 0; Y < 3; ++Y) {
      double s = 0.0;
      for (int q = 0; q < M.n; ++q) {
        const MomentTerm& t = M.t[q];
        const double v = t.sym ? w[t.w] * (Ji[t.m][X] * Ji[t.n][Y] + Ji[t.n][X] * Ji[t.m][Y])
                               : w[t.w] * Ji[t.m][X] * Ji[t.n][Y];
        s = q == 0 ? v : s + v;
      }
      Q[X][Y] = s;
    }
}

// The two other indices of i, in the order the diagonal sums take them.
FX_HD void others(int i, int& j, int& l) {
  j = i == 1 ? 0 : 1;
  l = i == 2 ? 1 : 2;
  if (i == 2) {
    j = 1;
    l = 0;
  }
}

// The full isotropic rule on a moment (symmetric families with C4 off the diagonal).
FX_HD double full_rule(const double Q[3][3], int i, int k, double C1, double C2, double C3, bool sym) {
  if (i == k) {
    int j, l;
    others(i, j, l);
    return C1 * Q[i][i] + C3 * (Q[j][j] + Q[l][l]);
  }
  return sym ? (C2 + C3) * Q[i][k] : C2 * Q[i][k] + C3 * Q[k][i];
}
// The shear rule (the blocks coupling the stu mode).
FX_HD double shear_rule(const double Q[3][3], int i, int k, double C3) {
  if (i == k) {
    int j, l;
    others(i, j, l);
    return C3 * (Q[j][j] + Q[l][l]);
  }
  return C3 * Q[i][k];
}

// interior = FCF - KuT FeCFe^-1 FeCFhg (12 x 12, hourglass modes st ut us stu, 3 components each).
FX_HD void interior_matrix(const Frame& f, double C1, double C2, double C3, double out[12][12]) {
  double w[kWeights];
  weights(f.J, w);
  const double(&Ji)[3][3] = f.Jinv;
  const double C4 = C2 + C3;
  // FCF by blocks: (g, h) g <= h; the lower blocks transpose the upper ones, and a diagonal block
  // is computed on and above its diagonal and mirrored
  double FCF[12][12];
  const int fam[4][4] = {{0, 3, 4, 6}, {3, 1, 5, 7}, {4, 5, 2, 8}, {6, 7, 8, 9}};
  for (int g = 0; g < 4; ++g)
    for (int h = g; h < 4; ++h) {
      double Q[3][3];
      moment_matrix(fam[g][h], w, Ji, Q);
      for (int i = 0; i < 3; ++i)
        for (int k = g == h ? i : 0; k < 3; ++k) {
          double v;
          if (h == 3) v = shear_rule(Q, i, k, C3);
          else v = full_rule(Q, i, k, C1, C2, C3, g == h);
          FCF[3 * g + i][3 * h + k] = v;
          FCF[3 * h + k][3 * g + i] = v;
        }
    }
  (void)C4;
  // enhanced-strain coefficients C_mn (m <= n: ss st su tt tu uu), the full rule on Jinv rows
  double Cc[3][3][3][3];  // [m][n][X][Y]
  for (int m = 0; m < 3; ++m)
    for (int n = m; n < 3; ++n)
      for (int X = 0; X < 3; ++X)
        for (int Y = 0; Y < 3; ++Y) {
          double v;
          if (X == Y) {
            int j, l;
            others(X, j, l);
            v = C1 * Ji[m][X] * Ji[n][X] + C3 * (Ji[m][j] * Ji[n][j] + Ji[m][l] * Ji[n][l]);
          } else if (m == n) {
            v = C4 * Ji[m][X] * Ji[m][Y];
          } else {
            v = C2 * Ji[m][X] * Ji[n][Y] + C3 * Ji[m][Y] * Ji[n][X];
          }
          Cc[m][n][X][Y] = v;
        }
  // for the symmetric C_mm the reference reads one triangle: entry (X, Y) and (Y, X) alike
  auto C = [&](int m, int n, int X, int Y) {
    if (m == n && X > Y) return Cc[m][n][Y][X];
    return Cc[m][n][X][Y];
  };
  // FeCFe: block (a, b) of the enhanced modes s t u is C_ab times its weight; below the diagonal
  // the transposed block
  const int fe_w[3][3] = {{W0789, W619, W518}, {W619, W0879, W417}, {W518, W417, W0978}};
  double FeCFe[9][9];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k)
          FeCFe[3 * a + i][3 * b + k] = a <= b ? C(a, b, i, k) * w[fe_w[a][b]] : C(b, a, k, i) * w[fe_w[a][b]];
  double FeCFeInv[9][9];
  if (!lu_inverse<9>(FeCFe, FeCFeInv))
    for (int a = 0; a < 9; ++a)
      for (int c = 0; c < 9; ++c) FeCFeInv[a][c] = 0.0;
  // FeCFhg (9 x 12, the stu columns zero): entry = C(first) w1 + C(second) w2 by block
  double FeCFhg[9][12];
  for (int a = 0; a < 9; ++a)
    for (int c = 0; c < 12; ++c) FeCFhg[a][c] = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) {
      // rows s
      FeCFhg[i][k] = C(0, 1, i, k) * w[W0789] + C(0, 0, i, k) * w[W619];
      FeCFhg[i][3 + k] = C(0, 2, i, k) * w[W619] + C(0, 1, i, k) * w[W518];
      FeCFhg[i][6 + k] = C(0, 2, i, k) * w[W0789] + C(0, 0, i, k) * w[W518];
      // rows t
      FeCFhg[3 + i][k] = C(0, 1, k, i) * w[W0879] + C(1, 1, i, k) * w[W619];
      FeCFhg[3 + i][3 + k] = C(1, 2, i, k) * w[W0879] + C(1, 1, i, k) * w[W417];
      FeCFhg[3 + i][6 + k] = C(1, 2, i, k) * w[W619] + C(0, 1, k, i) * w[W417];
      // rows u
      FeCFhg[6 + i][k] = C(1, 2, k, i) * w[W518] + C(0, 2, k, i) * w[W417];
      FeCFhg[6 + i][3 + k] = C(1, 2, k, i) * w[W0978] + C(2, 2, i, k) * w[W417];
      FeCFhg[6 + i][6 + k] = C(0, 2, k, i) * w[W0978] + C(2, 2, i, k) * w[W518];
    }
  double KuTinv[12][9];
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 9; ++j) {
      double s = 0.0;
      for (int k = 0; k < 9; ++k) s += FeCFhg[k][i] * FeCFeInv[k][j];
      KuTinv[i][j] = s;
    }
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j) {
      double s = 0.0;
      for (int k = 0; k < 9; ++k) s += KuTinv[i][k] * FeCFhg[k][j];
      out[i][j] = FCF[i][j] - s;
    }
}

// Each node's volume weight: the integral of N_i over the element (2 x 2 x 2 Gauss, exact for
// the trilinear map; the points in stdBrick's order).
FX_HD void node_volumes(const double xl[3][8], double w[8]) {
  for (int j = 0; j < 8; ++j) w[j] = 0.0;
  for (int gp = 0; gp < 8; ++gp) {
    PointShape s;
    point_shape(xl, gp, s);
    for (int j = 0; j < 8; ++j) w[j] += s.N[j] * s.dvol;
  }
}

// The element's geometry record (kGeo values, value k at g[k * ld]) and constants (kCon values,
// c[k * ld]) for initial tangent moduli C1, C2, C3.
template <class V>
FX_HD void element_setup(const double xl[3][8], double C1, double C2, double C3, V g, V c) {
  Frame f;
  frame(xl, f, true);
  for (int k = 0; k < 24; ++k) g[k] = f.dN[k / 3][k % 3];
  g[24] = f.vol;
  double nv[8];
  node_volumes(xl, nv);
  for (int i = 0; i < 8; ++i) g[25 + i] = nv[i];
  double K[12][12];
  interior_matrix(f, C1, C2, C3, K);
  for (int gi = 0; gi < 4; ++gi)
    for (int i = 0; i < 8; ++i) c[8 * gi + i] = f.gamma[gi][i];
  int k = 32;
  for (int r = 0; r < 12; ++r)
    for (int q = r; q < 12; ++q) c[k++] = K[r][q];
}

// interior(r, q) from the packed upper triangle.
template <class V>
FX_HD double interior_at(const V& c, int r, int q) {
  if (r > q) {
    const int t = r;
    r = q;
    q = t;
  }
  return c[32 + 12 * r - r * (r - 1) / 2 + (q - r)];
}

// z = interior (Mben v): 12 values (Mben v: the four hourglass modes of each component).
template <class V>
FX_HD void stab_reduce(const V& c, const double* v, double z[12]) {
  double m[12];
  for (int gi = 0; gi < 4; ++gi)
    for (int d = 0; d < 3; ++d) {
      double s = 0.0;
      for (int i = 0; i < 8; ++i) s += c[8 * gi + i] * v[3 * i + d];
      m[3 * gi + d] = s;
    }
  for (int r = 0; r < 12; ++r) {
    double s = 0.0;
    for (int q = 0; q < 12; ++q) s += interior_at(c, r, q) * m[q];
    z[r] = s;
  }
}
// (Kstab v) at node j: Mben_j^T z.
template <class V>
FX_HD void stab_node(const V& c, const double z[12], int j, double out[3]) {
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    for (int gi = 0; gi < 4; ++gi) s += c[8 * gi + j] * z[3 * gi + d];
    out[d] = s;
  }
}
// Kstab(a, b), summed in the order of (min, max) so that it is exactly symmetric.
template <class V>
FX_HD double stab_entry(const V& c, int a, int b) {
  if (a > b) {
    const int t = a;
    a = b;
    b = t;
  }
  const int i = a / 3, d = a % 3, k = b / 3, e = b % 3;
  double s = 0.0;
  for (int gi = 0; gi < 4; ++gi)
    for (int hi = 0; hi < 4; ++hi) s += c[8 * gi + i] * interior_at(c, 3 * gi + d, 3 * hi + e) * c[8 * hi + k];
  return s;
}

// The one point's strain, Bnot u, accumulated node by node in column order.
template <class V>
FX_HD void strain_of(const V& g, const double* u, double e[6]) {
  for (int c = 0; c < 6; ++c) e[c] = 0.0;
  for (int i = 0; i < 8; i++) {
    const double bx = g[3 * i], by = g[3 * i + 1], bz = g[3 * i + 2];
    const double u0 = u[3 * i], u1 = u[3 * i + 1], u2 = u[3 * i + 2];
    e[0] += bx * u0;
    e[3] += by * u0;
    e[5] += bz * u0;
    e[1] += by * u1;
    e[3] += bx * u1;
    e[4] += bz * u1;
    e[2] += bz * u2;
    e[4] += by * u2;
    e[5] += bx * u2;
  }
}
// mVol Bnot_j^T s (column sums, then times mVol).
template <class V>
FX_HD void node_force(const V& g, const double s[6], int j, double f[3]) {
  const double bx = g[3 * j], by = g[3 * j + 1], bz = g[3 * j + 2], vol = g[24];
  f[0] = (bx * s[0] + by * s[3] + bz * s[5]) * vol;
  f[1] = (by * s[1] + bx * s[3] + bz * s[4]) * vol;
  f[2] = (bz * s[2] + by * s[4] + bx * s[5]) * vol;
}
// The point's 3 x 3 block (J, K) of mVol Bnot^T D Bnot, in the reference's two-stage form.
template <class V>
FX_HD void block(const V& g, const double D[6][6], int J, int K, double out[3][3]) {
  double BJ[6][3] = {}, BK[6][3] = {};
  const int nd[2] = {J, K};
  for (int w = 0; w < 2; ++w) {
    double(*B)[3] = w ? BK : BJ;
    const int n = nd[w];
    B[0][0] = g[3 * n];
    B[1][1] = g[3 * n + 1];
    B[2][2] = g[3 * n + 2];
    B[3][0] = g[3 * n + 1];
    B[3][1] = g[3 * n];
    B[4][1] = g[3 * n + 2];
    B[4][2] = g[3 * n + 1];
    B[5][0] = g[3 * n + 2];
    B[5][2] = g[3 * n];
  }
  const double vol = g[24];
  double BD[3][6];
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 6; q++) {
      double s = 0.0;
      for (int r = 0; r < 6; r++) s += BJ[r][p] * (D[r][q] * vol);
      BD[p][q] = s;
    }
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 3; q++) {
      double s = 0.0;
      for (int r = 0; r < 6; r++) s += BD[p][r] * BK[r][q];
      out[p][q] = s;
    }
}

// ---- element routines on the cached geometry g (kGeo values) and constants c (kCon values)
// Operator factors of an element whose initial stiffness is its tangent (element_operator.hpp:
// 45-56 with initial_stiffness_is_tangent): the stiffness term and betaK, betaKinit damping on the
// current tangent, betaKcomm on the committed one, alphaM and the mass term on the lumped mass;
// the stabilization Kstab is part of every stiffness, so its factor adds all three betas.
struct Factors {
  double cK, cc, cM, cE;
};
FX_HD Factors factors(const ParamGP& p, double ks, double kd, double km) {
  Factors f;
  f.cK = ks + kd * p.betaK + kd * p.betaKinit;
  f.cc = kd * p.betaKcomm;
  f.cM = km + kd * p.alphaM;
  f.cE = ks + kd * (p.betaK + p.betaKinit + p.betaKcomm);
  return f;
}

// D_eff = cK D + cc D of the elastic material (its current and committed tangents are D).
FX_HD void effective(const ParamGP& p, const Factors& f, double De[6][6]) {
  double D[6][6];
  elastic_D(p, D);
  for (int a = 0; a < 6; ++a)
    for (int c = 0; c < 6; ++c) {
      double v = f.cK * D[a][c];
      if (f.cc != 0.0) v += f.cc * D[a][c];
      De[a][c] = v;
    }
}

// y_e = K_eff,e x_e (element_operator_apply, element_operator.hpp:82-130): the point's
// mVol Bnot^T D_eff Bnot x and lumped mass, then cE Kstab x.
template <class V>
FX_HD void element_apply(const ParamGP& p, const Factors& f, const V& g, const V& c, const double* xe, double* ye) {
  for (int a = 0; a < 24; ++a) ye[a] = 0.0;
  double De[6][6], e[6], sg[6];
  effective(p, f, De);
  strain_of(g, xe, e);
  for (int a = 0; a < 6; ++a) {
    double sum = 0.0;
    for (int q = 0; q < 6; ++q) sum += De[a][q] * e[q];
    sg[a] = sum;
  }
  for (int j = 0; j < 8; ++j) {
    double fj[3];
    node_force(g, sg, j, fj);
    for (int q = 0; q < 3; ++q) ye[3 * j + q] += fj[q];
    if (f.cM != 0.0) {
      const double m = p.rho * g[25 + j];
      for (int q = 0; q < 3; ++q) ye[3 * j + q] += f.cM * (m * xe[3 * j + q]);
    }
  }
  if (f.cE != 0.0) {
    double z[12];
    stab_reduce(c, xe, z);
    for (int j = 0; j < 8; ++j) {
      double kj[3];
      stab_node(c, z, j, kj);
      for (int q = 0; q < 3; ++q) ye[3 * j + q] += f.cE * kj[q];
    }
  }
}

// diag(K_eff) by element with the merged-equation cross terms (element_operator_diagonal,
// element_operator.hpp:138-209).
template <class V>
FX_HD void element_diagonal(const ParamGP& p, const Factors& f, const V& g, const V& c, const int* eq, double* de) {
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
  double De[6][6];
  effective(p, f, De);
  for (int j = 0; j < 8; ++j) {
    double blk[3][3];
    block(g, De, j, j, blk);
    const double m = f.cM != 0.0 ? f.cM * (p.rho * g[25 + j]) : 0.0;
    for (int q = 0; q < 3; ++q) de[3 * j + q] += blk[q][q] + m;
  }
  if (merged)
    for (int J = 0; J < 8; ++J)
      for (int K = 0; K < 8; ++K) {
        bool any = false;
        for (int a = 0; a < 3 && !any; ++a)
          for (int q = 0; q < 3; ++q) {
            const int ia = 3 * J + a, ic = 3 * K + q;
            if (ia != ic && eq[ia] >= 0 && eq[ia] == eq[ic]) any = true;
          }
        if (!any) continue;
        double blk[3][3];
        block(g, De, J, K, blk);
        const double m = (f.cM != 0.0 && J != K) ? f.cM * 0.0 : 0.0;  // the lumped mass off its diagonal
        for (int a = 0; a < 3; ++a)
          for (int q = 0; q < 3; ++q) {
            const int ia = 3 * J + a, ic = 3 * K + q;
            if (ia == ic || eq[ia] < 0 || eq[ia] != eq[ic]) continue;
            de[first[ia]] += blk[a][q] + (a == q ? m : 0.0);
          }
      }
  if (f.cE != 0.0) {
    for (int a = 0; a < 24; ++a) de[a] += f.cE * stab_entry(c, a, a);
    if (merged)
      for (int a = 0; a < 24; ++a)
        for (int b = 0; b < 24; ++b) {
          if (a == b || eq[a] < 0 || eq[a] != eq[b]) continue;
          de[first[a]] += f.cE * stab_entry(c, a, b);
        }
  }
}

// Internal force plus the Rayleigh damping forces of an elastic element (SSPbrick::compute_with,
// ssp_brick.hpp: Kstab u first, with (betaK + betaKinit + betaKcomm) Kstab v in the damping
// force, then the point's stress, body force (b times the node's volume weight), damping stress
// and alphaM lumped mass): fe = resid + fdamp.
template <class V>
FX_HD void element_force(const ParamGP& p, const V& g, const V& c, const double* ue, const double* ve, double* fe) {
  double resid[24], fdamp[24];
  double zu[12], zv[12];
  stab_reduce(c, ue, zu);
  stab_reduce(c, ve, zv);
  const double beta = p.betaK + p.betaKinit + p.betaKcomm;
  for (int j = 0; j < 8; ++j) {
    stab_node(c, zu, j, resid + 3 * j);
    if (beta != 0.0) {
      double kv[3];
      stab_node(c, zv, j, kv);
      for (int q = 0; q < 3; ++q) fdamp[3 * j + q] = beta * kv[q];
    } else {
      for (int q = 0; q < 3; ++q) fdamp[3 * j + q] = 0.0;
    }
  }
  double e[6], sg[6], ds[6];
  strain_of(g, ue, e);
  elastic_stress(p, e, sg);
  const bool stiff = p.betaK != 0.0 || p.betaKinit != 0.0 || p.betaKcomm != 0.0;
  for (int a = 0; a < 6; ++a) ds[a] = 0.0;
  if (stiff) {
    double D[6][6], rate[6];
    elastic_D(p, D);
    strain_of(g, ve, rate);
    for (int a = 0; a < 6; ++a) {
      double sum = 0.0;
      for (int q = 0; q < 6; ++q) {
        double d = p.betaK * D[a][q];
        if (p.betaKinit != 0.0) d += p.betaKinit * D[a][q];
        if (p.betaKcomm != 0.0) d += p.betaKcomm * D[a][q];
        sum += d * rate[q];
      }
      ds[a] = sum;
    }
  }
  for (int j = 0; j < 8; ++j) {
    double rj[3], dj[3] = {0.0, 0.0, 0.0};
    node_force(g, sg, j, rj);
    if (stiff) node_force(g, ds, j, dj);
    if (p.alphaM != 0.0) {
      const double m = p.rho * g[25 + j];
      for (int q = 0; q < 3; ++q) dj[q] += p.alphaM * m * ve[3 * j + q];
    }
    for (int q = 0; q < 3; ++q) {
      resid[3 * j + q] += rj[q];
      resid[3 * j + q] -= p.b[q] * g[25 + j];
      fdamp[3 * j + q] += dj[q];
    }
  }
  for (int a = 0; a < 24; ++a) fe[a] = resid[a] + fdamp[a];
}

}  // namespace ssp
}  // namespace fx
