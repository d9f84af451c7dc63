// PressureIndependMultiYield at one material point, for the device and the host: multi-yield-surface
// von Mises plasticity with kinematic (Mroz) hardening of nested surfaces (Elgamal, Yang and Parra's
// soil model, OpenSees nDMaterial PressureIndependMultiYield, three-dimensional form). The
// reference's material is src/physics/materials/pressure_independ_multi_yield.hpp (setup :102-139,
// setUpSurfaces :282-388, getStress :478-541, finish :544-575, elast2Plast :578-609, the surface
// functions :611-849, getTangent :853-885) over src/physics/common/t2_vector.hpp. The published
// algorithm's steps are followed in the same arithmetic order (no contracted multiply-adds: the
// translation units that include this file build with --fmad=false), so that a point gives
// OpenSees' bits wherever the math library agrees (sqrt is exact; pow, used at the switch to the
// plastic stage with a friction angle, may differ in the last place on the device).
//
// State of a point, `nstate(ns)` values, read and written through a strided view (a point's values
// `ld` apart, so that consecutive points are consecutive in memory for every value):
//   0..12   stress: components (11 22 33 12 23 31, tensor shear), deviator, mean
//   13..25  strain at the last commit, the same 13 values
//   26      active surface, 27 switched to plastic (0/1), 28 shear modulus G, 29 bulk modulus K
//   30      the update changed the surfaces (a trial state's surfaces are valid only then, when the
//           update ran copy-on-write; the full form writes them always and sets 1)
//   31 + 8 (i - 1) + {0, 1, 2..7}: surface i (1..ns): size, plastic modulus, center (6)
// The moduli and surfaces start at the material's values and are scaled by the confinement at the
// switch to the plastic stage (when the friction angle is positive).
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define FX_PIMY_HD __host__ __device__
#else
#define FX_PIMY_HD
#endif

namespace fx {
namespace pimy {

constexpr int kMaxSurfaces = 40;
constexpr double kLow = 20. * DBL_EPSILON;  // OpenSees LOW_LIMIT
constexpr double kUp = 1.0e+30;             // OpenSees UP_LIMIT
constexpr double kVeryLarge = 1.0e200;      // a Vector divided by zero
constexpr double kPi = 3.14159265358979;    // OpenSees' value

enum : int { S_STRESS = 0, S_STRAIN = 13, S_ACTIVE = 26, S_E2P = 27, S_G = 28, S_K = 29, S_CHANGED = 30, S_SURF = 31 };
FX_PIMY_HD constexpr int nstate(int ns) { return S_SURF + 8 * ns; }

// The material after setup: constructor values and the surfaces of setUpSurfaces ([0] unused).
struct Params {
  int ns;  // yield surfaces
  double rho, G0, K0, phi, gamma_peak;
  double pref;  // reference pressure, negative (compression)
  double cohesion, n_press, p_res;
  double size[kMaxSurfaces + 1], modulus[kMaxSurfaces + 1];
};

// setup failures (the reference's Setup codes)
enum : int { kOk = 0, kTooManySurfaces = 1, kBadFriction = 2, kBadModulus = 3, kTooFewPairs = 4, kBadInput = 5 };

// ---- six-component vectors in OpenSees' Vector arithmetic
FX_PIMY_HD inline double dd(const double* a, const double* b) {  // tensor double-dot in vector form
  double r = 0.;
  for (int i = 0; i < 3; i++) r += a[i] * b[i] + 2 * a[i + 3] * b[i + 3];
  return r;
}
FX_PIMY_HD inline void vset(double* a, const double* b) {
  for (int i = 0; i < 6; i++) a[i] = b[i];
}
FX_PIMY_HD inline void vsub(double* a, const double* b) {
  for (int i = 0; i < 6; i++) a[i] -= b[i];
}
FX_PIMY_HD inline void vadd(double* a, const double* b) {
  for (int i = 0; i < 6; i++) a[i] += b[i];
}
FX_PIMY_HD inline void vscale(double* a, double f) {
  for (int i = 0; i < 6; i++) a[i] *= f;
}
FX_PIMY_HD inline void vdiv(double* a, double f) {
  if (f == 0.0) {
    for (int i = 0; i < 6; i++) a[i] = kVeryLarge;
  } else {
    for (int i = 0; i < 6; i++) a[i] /= f;
  }
}
FX_PIMY_HD inline void vaxpy(double* a, const double* b, double f) {  // a += b f
  for (int i = 0; i < 6; i++) a[i] += b[i] * f;
}
FX_PIMY_HD inline void vmul(double* a, const double* b, double f) {  // a = b f
  for (int i = 0; i < 6; i++) a[i] = b[i] * f;
}

// A second-order tensor as OpenSees' T2Vector keeps it: components, deviator and mean, each
// derived in the order of the setter that made it (so all 13 are kept, not recomputed).
struct Ten {
  double t[6], d[6], m;
  FX_PIMY_HD void from_full(const double* v, bool engineering) {  // setData(vector, isEngrgStrain)
    vset(t, v);
    m = (t[0] + t[1] + t[2]) / 3.0;
    for (int i = 0; i < 3; i++) {
      d[i] = t[i] - m;
      d[i + 3] = t[i + 3];
      if (engineering) {
        d[i + 3] /= 2.;
        t[i + 3] /= 2.;
      }
    }
  }
  FX_PIMY_HD void from_dev(const double* dv, double mean) {  // setData(deviator, volume)
    m = mean;
    const double dm = (dv[0] + dv[1] + dv[2]) / 3.;
    for (int i = 0; i < 3; i++) {
      d[i] = dv[i] - dm;
      d[i + 3] = dv[i + 3];
      t[i] = d[i] + m;
      t[i + 3] = d[i + 3];
    }
  }
  FX_PIMY_HD void engineering(double* out) const {  // t2Vector(1)
    vset(out, t);
    for (int i = 0; i < 3; i++) out[i + 3] *= 2.;
  }
  FX_PIMY_HD double dev_length() const { return sqrt(dd(d, d)); }
  FX_PIMY_HD double oct_shear() const { return sqrt(1. / 3.) * dev_length(); }
  FX_PIMY_HD double oct_shear_engr() const { return 2. * sqrt(1. / 3.) * dev_length(); }  // of a strain
  FX_PIMY_HD double dev_ratio(double p_res) const {  // deviatorRatio
    return sqrt(3. / 2. * dd(d, d)) / (fabs(m) + fabs(p_res));
  }
  FX_PIMY_HD void unit(double* out) const {  // unitT2: the components over their length
    vset(out, t);
    const double len = sqrt(dd(t, t));
    if (len <= kLow) vdiv(out, kLow);
    else vdiv(out, len);
  }
  FX_PIMY_HD bool zero() const {
    for (int i = 0; i < 6; i++)
      if (t[i] != 0.0) return false;
    return true;
  }
  template <class V>
  FX_PIMY_HD void load(const V& s, int k) {
    for (int i = 0; i < 6; i++) t[i] = s[k + i];
    for (int i = 0; i < 6; i++) d[i] = s[k + 6 + i];
    m = s[k + 12];
  }
  template <class V>
  FX_PIMY_HD void store(const V& s, int k) const {
    for (int i = 0; i < 6; i++) s[k + i] = t[i];
    for (int i = 0; i < 6; i++) s[k + 6 + i] = d[i];
    s[k + 12] = m;
  }
};

// One point's values, `ld` apart.
template <class T>
struct Slab {
  T* p;
  int64_t ld;
  FX_PIMY_HD T& operator[](int k) const { return p[k * ld]; }
};

// MultiYieldSurface's secondOrderEqn: the smaller non-negative root of A x^2 + B x + C; `ok` false
// (and NaN) where OpenSees stops the program.
FX_PIMY_HD inline double quad_root(double A, double B, double C, bool& ok) {
  const double nan = static_cast<double>(NAN);
  if (A == 0) {
    ok = false;
    return nan;
  }
  if (C == 0) return 0;
  if (B == 0) {
    if (C / A > 0) {
      ok = false;
      return nan;
    }
    return sqrt(-C / A);
  }
  const double det = B * B - 4. * A * C;
  if (det < 0) {
    ok = false;
    return nan;
  }
  double r1 = B > 0 ? (-B - sqrt(det)) / (2. * A) : (-B + sqrt(det)) / (2. * A);
  double r2 = C / (A * r1);
  if (r1 < 0 && r2 < 0) {
    if (fabs(r1) < kLow) r1 = 0.;
    else if (fabs(r2) < kLow) r2 = 0.;
  }
  if (r1 < 0 && r2 < 0) {
    ok = false;
    return nan;
  }
  if (r1 < 0) return r2;
  if (r2 < 0) return r1;
  return r1 > r2 ? r2 : r1;
}

FX_PIMY_HD inline void elastic_D(double G, double K, double* D) {  // D[6 i + j]
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double v = 0.;
      if (i == j) v += G;
      if (i < 3 && j < 3 && i == j) v += G;
      if (i < 3 && j < 3) v += (K - 2. * G / 3.);
      D[6 * i + j] = v;
    }
}

// Constructor checks and setUpSurfaces: in9 = rho, refShearModul, refBulkModul, cohesi,
// peakShearStra, frictionAng, refPress, pressDependCoe, noYieldSurf; pairs = noYieldSurf (gamma,
// G/Gmax) pairs of a user backbone, or NULL for the hyperbolic one. Values OpenSees resets with a
// warning are reset the same way; the ones it treats as fatal return an error code.
inline int setup(const double* in9, const double* pairs, Params& p) {
  double rho = in9[0], phi = in9[5], c = in9[3], n_press = in9[7];
  const double G0 = in9[1], K0 = in9[2], gpeak = in9[4], pr = in9[6];
  int ns = static_cast<int>(in9[8]);
  if (G0 <= 0 || K0 <= 0) return kBadInput;
  if (phi < 0.) phi = 0.;
  if (phi == 0. && c <= 0.) return kBadInput;
  if (c <= 0) c = 0.;
  if (gpeak <= 0 || pr <= 0) return kBadInput;
  if (n_press < 0) n_press = 0.;
  if (n_press > 0 && phi == 0) n_press = 0.;
  if (ns <= 0) ns = 10;
  if (ns > 100) ns = 100;
  if (rho < 0) rho = 0.;
  if (ns > kMaxSurfaces) return kTooManySurfaces;
  if (pairs != nullptr && ns < 2) return kTooFewPairs;
  p.ns = ns;
  p.rho = rho;
  p.G0 = G0;
  p.K0 = K0;
  p.gamma_peak = gpeak;
  p.pref = -pr;
  p.n_press = n_press;
  for (int i = 0; i <= kMaxSurfaces; ++i) p.size[i] = p.modulus[i] = 0.0;
  double p_res = 0.;
  double cone = 0.;
  // plastic modulus of the segment between two backbone points (stress, strain) (OpenSees'
  // H' = 2 G H / (2 G - H) of the segment's elasto-plastic modulus H, capped)
  auto segment = [&](double s1, double e1, double s2, double e2) {
    const double ep = 2. * (s2 - s1) / (e2 - e1);
    return (2. * G0 - ep) <= 0 ? kUp : (2. * G0 * ep) / (2. * G0 - ep);
  };
  if (pairs == nullptr) {  // hyperbolic backbone, ns equal stress steps up to the peak
    double peak = 0., gref = 0.;
    if (phi > 0) {
      const double sinphi = std::sin(phi * kPi / 180.);
      const double M = 6. * sinphi / (3. - sinphi);
      p_res = 3. * c / (std::sqrt(2.) * M);
      cone = -(p.pref - p_res);
      peak = std::sqrt(2.) * cone * M / 3.;
    } else {  // the cohesion is the peak shear strength
      peak = 2 * std::sqrt(2.) * c / 3;
      p_res = 0.;
    }
    gref = (gpeak * peak) / (G0 * gpeak - peak);
    const double step = peak / ns;
    for (int i = 1; i <= ns; i++) {
      const double s1 = i * step, s2 = s1 + step;
      const double e1 = s1 * gref / (G0 * gref - s1), e2 = s2 * gref / (G0 * gref - s2);
      const double sz = phi > 0. ? 3. * s1 / std::sqrt(2.) / cone : 3. * s1 / std::sqrt(2.);
      double h = segment(s1, e1, s2, e2);
      if (h < 0) h = 0;
      if (h > kUp) h = kUp;
      if (i == ns) h = 0;
      p.size[i] = sz;
      p.modulus[i] = h;
    }
  } else {  // user backbone: the cone from the last pair's strength
    const int last = 2 * (ns - 1);
    const double tmax = G0 * pairs[last] * pairs[last + 1];
    if (phi > 0) {
      const double M = -(std::sqrt(3.) * tmax - 2. * c) / p.pref;
      if (M <= 0) {  // no cone: a von Mises cylinder, the given cohesion dropped
        c = std::sqrt(3.) / 2 * tmax;
        phi = 0.;
        cone = 1.;
        p_res = 0.;
      } else {
        const double sinphi = 3 * M / (6 + M);
        if (sinphi < 0. || sinphi > 1.) return kBadFriction;
        p_res = 2. * c / M;
        if (p_res < 0.01 * p.pref) p_res = 0.01 * p.pref;
        cone = -(p.pref - p_res);
        phi = std::asin(sinphi) * 180 / kPi;
      }
    } else {
      c = std::sqrt(3.) / 2 * tmax;
      cone = 1.;
      p_res = 0.;
    }
    for (int i = 1; i < ns; i++) {
      const int k = 2 * (i - 1);
      const double e1 = pairs[k], s1 = G0 * pairs[k + 1] * e1;
      const double e2 = pairs[k + 2], s2 = G0 * pairs[k + 3] * e2;
      double h = segment(s1, e1, s2, e2);
      if (h <= 0) return kBadModulus;
      if (h > kUp) h = kUp;
      p.size[i] = std::sqrt(3.) * s1 / cone;
      p.modulus[i] = h;
      if (i == ns - 1) {
        p.size[i + 1] = std::sqrt(3.) * s2 / cone;
        p.modulus[i + 1] = 0;
      }
    }
  }
  p.p_res = p_res;
  p.phi = phi;
  p.cohesion = c;
  return kOk;
}

template <class V>
FX_PIMY_HD inline void initial_state(const Params& p, const V& s) {
  for (int k = 0; k < nstate(p.ns); ++k) s[k] = 0.0;
  s[S_G] = p.G0;
  s[S_K] = p.K0;
  for (int i = 1; i <= p.ns; ++i) {
    s[S_SURF + 8 * (i - 1)] = p.size[i];
    s[S_SURF + 8 * (i - 1) + 1] = p.modulus[i];
  }
}

// The tangent D[6 i + j] of a compact form t[kTan] (Point::compact): the elastic tangent of the
// point's moduli in the elastic stage; in the plastic stage OpenSees' expression, elastic minus
// coeff dv (x) dv (which is what it gives, signed zeros included, at an inactive point).
constexpr int kTan = 10;
FX_PIMY_HD inline void compact_D(const double* t, double* D) {
  const double G = t[1], K = t[2];
  if (t[0] != 1.0) {
    elastic_D(G, K, D);
    return;
  }
  const double coeff = t[3];
  const double* dv = t + 4;
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double v = -coeff * dv[i] * dv[j];
      if (i == j) v += G;
      if (i < 3 && j < 3 && i == j) v += G;
      if (i < 3 && j < 3) v += (K - 2. * G / 3.);
      D[6 * i + j] = v;
    }
}

FX_PIMY_HD inline int to_int(double x) {  // C++ truncation, NaN 0 and clamped outside int
  if (!(x == x)) return 0;
  if (x >= 2147483647.0) return 2147483647;
  if (x <= -2147483648.0) return -2147483647 - 1;
  return static_cast<int>(x);
}

// One point's update from its committed state C to the trial state T at the total strain eps
// (engineering shear): OpenSees' setTrialStrain + getStress + getTangent, the instance's members as
// locals. The surfaces are read from the committed state until the update first changes one; then
// all of them are copied to the trial state, which holds them from there on (copy on write: most
// updates change no surface). `full`: the trial state's surfaces are written in any case.
template <class CV, class TV>
struct Point {
  const Params& P;
  int stage;  // 0 elastic, 1 plastic (updateMaterialStage)
  CV C;
  TV T;
  bool full = true;
  bool dirty = false;  // the trial state holds the surfaces
  bool ok = true;  // false after a state OpenSees stops the program for
  Ten cur, strain, trial, rate, sub;  // currentStress, currentStrain, trialStress, strainRate, subStrainRate
  int active_c = 0, active = 0, e2p = 0;
  double G = 0., K = 0.;

  FX_PIMY_HD Point(const Params& p, int st, CV c, TV t) : P(p), stage(st), C(c), T(t) {}

  FX_PIMY_HD int at(int i) const { return S_SURF + 8 * (i - 1); }
  FX_PIMY_HD double sv(int k) const { return dirty ? T[k] : C[k]; }
  FX_PIMY_HD void touch() {  // the first change: the surfaces into the trial state
    if (dirty) return;
    for (int k = S_SURF; k < nstate(P.ns); ++k) T[k] = C[k];
    dirty = true;
  }
  FX_PIMY_HD double size(int i) const { return i == 0 ? 0. : sv(at(i)); }
  FX_PIMY_HD double hmod(int i) const { return i == 0 ? 0. : sv(at(i) + 1); }
  FX_PIMY_HD void center(int i, double* c) const {
    for (int k = 0; k < 6; ++k) c[k] = i == 0 ? 0. : sv(at(i) + 2 + k);
  }
  FX_PIMY_HD void set_center(int i, const double* c) {
    touch();
    for (int k = 0; k < 6; ++k) T[at(i) + 2 + k] = c[k];
  }

  FX_PIMY_HD double yield(const Ten& s, int i) const {  // yieldFunc
    double x[6], c[6];
    vset(x, s.d);
    center(i, c);
    vsub(x, c);
    const double sz = size(i);
    return 3. / 2. * dd(x, x) - sz * sz;
  }

  FX_PIMY_HD void scale_deviator(Ten& s, int i) {  // deviatorScaling, its recursion as a loop
    for (int it = 0; it < 100000; ++it) {
      const double diff = yield(s, i);
      if (i < P.ns && diff < 0.) {
        const double sz = size(i), dsz = sqrt(sz * sz + diff);
        double dv[6], x[6], c[6];
        vset(dv, s.d);
        center(i, c);
        for (int k = 0; k < 6; ++k) x[k] = dv[k] - c[k];
        double f = (sz - dsz) / dsz;
        if (f < 1.e-13) f = 1.e-13;
        vaxpy(dv, x, f);
        s.from_dev(dv, s.m);
        continue;
      }
      if (i == P.ns && fabs(diff) > kLow) {
        const double sz = size(i);
        double nd[6];
        vmul(nd, s.d, sz / sqrt(diff + sz * sz));
        s.from_dev(nd, s.m);
      }
      return;
    }
    ok = false;
  }

  FX_PIMY_HD void init_surfaces() {  // initSurfaceUpdate
    if (active_c == 0) return;
    double dv[6];
    vset(dv, cur.d);
    const double Ms = sqrt(3. / 2. * dd(dv, dv));
    if (active_c < P.ns) {  // the outermost surface does not move
      double nc[6];
      vmul(nc, dv, 1.0 - size(active_c) / Ms);
      set_center(active_c, nc);
    }
    for (int i = 1; i < active_c; ++i) {
      double nc[6];
      const double f = 1. - size(i) / Ms;
      for (int k = 0; k < 6; ++k) nc[k] = dv[k] * f;
      set_center(i, nc);
    }
  }

  FX_PIMY_HD void scale_to_confinement() {  // paramScaling
    if (P.phi == 0.) return;
    const double h = -(cur.m - P.p_res);
    double f = -h / (P.pref - P.p_res);
    f = pow(f, P.n_press);
    G *= f;
    K *= f;
    touch();
    for (int i = 1; i <= P.ns; ++i) {
      const double hm = hmod(i) * f, sz = size(i) * h;
      T[at(i)] = sz;
      T[at(i) + 1] = hm;
      const double zero[6] = {0., 0., 0., 0., 0., 0.};
      set_center(i, zero);
    }
  }

  FX_PIMY_HD void elastic_to_plastic() {  // elast2Plast
    e2p = 1;
    if (cur.m > 0. && P.phi > 0.) {  // tension dropped
      double dv[6];
      vset(dv, cur.d);
      cur.from_full(dv, false);
    }
    scale_to_confinement();
    if (cur.dev_length() == 0.) return;
    while (yield(cur, ++active_c) > 0) {
      if (active_c == P.ns) {
        scale_deviator(cur, P.ns);
        init_surfaces();
        return;
      }
    }
    active_c--;
    init_surfaces();
  }

  FX_PIMY_HD void set_trial_stress(const Ten& in) {  // setTrialStress (in may be `trial` itself)
    const Ten s = in;
    double dv[6];
    vset(dv, s.d);
    vaxpy(dv, sub.d, 2. * G);
    trial.from_dev(dv, s.m);
  }

  FX_PIMY_HD int set_sub_rate() {  // setSubStrainRate
    if (rate.zero()) return 0;
    double epm;
    if (active == 0) epm = 2 * G;
    else {
      const double h = hmod(active);
      epm = 2 * G * h / (2 * G + h);
    }
    double inc[6];
    vmul(inc, rate.d, epm);
    Ten st;
    st.from_full(inc, false);
    const double single = size(P.ns) / P.ns;
    const double total = 3. * st.oct_shear() / sqrt(2.);
    int n = to_int(total / single + 1);
    if (n > P.ns) n = P.ns;
    vset(inc, rate.t);
    vdiv(inc, n);
    sub.from_full(inc, false);
    return n;
  }

  FX_PIMY_HD void normal_at(const Ten& s, double* n) const {  // getSurfaceNormal
    double c[6];
    vset(n, s.d);
    center(active, c);
    vsub(n, c);
    vdiv(n, sqrt(dd(n, n)));
  }

  FX_PIMY_HD void contact_stress(Ten& out) const {  // getContactStress
    double c[6], dv[6];
    center(active, c);
    vset(dv, trial.d);
    vsub(dv, c);
    const double Ms = sqrt(3. / 2. * dd(dv, dv));
    vscale(dv, size(active) / Ms);
    vadd(dv, c);
    out.from_dev(dv, trial.m);
  }

  FX_PIMY_HD bool reversal() const {  // isLoadReversal
    if (active == 0) return false;
    double n[6], a[6];
    normal_at(cur, n);
    vset(a, trial.d);
    vsub(a, cur.d);
    return dd(a, n) < 0;
  }

  FX_PIMY_HD double loading(const Ten& contact, const double* n, int crossed) const {  // getLoadingFunc
    const double t1 = 2. * G, t2 = hmod(active);
    const double t = t1 + t2;
    double x[6];
    vset(x, trial.d);
    vsub(x, contact.d);
    double lf = dd(n, x) / t;
    if (crossed) {
      const double t3 = hmod(active - 1);
      lf *= (t3 - t2) / t3;
    }
    return lf;
  }

  FX_PIMY_HD bool crossing_next() const {  // isCrossingNextSurface
    if (active == P.ns) return false;
    return yield(trial, active + 1) > 0;
  }

  FX_PIMY_HD void correct(int crossed) {  // stressCorrection, its recursion as a loop
    for (;;) {
      Ten contact;
      contact_stress(contact);
      double n[6], dv[6];
      normal_at(contact, n);
      const double lf = loading(contact, n, crossed);
      vmul(dv, n, -2 * G * lf);
      vadd(dv, trial.d);
      trial.from_dev(dv, trial.m);
      scale_deviator(trial, active);
      if (crossing_next()) {
        active++;
        crossed = 1;
        continue;
      }
      return;
    }
  }

  FX_PIMY_HD void move_active_surface() {  // updateActiveSurface
    if (active == P.ns) return;
    double t1[6], t2[6], x[6], c[6], oc[6];
    center(active, c);
    const double sz = size(active);
    center(active + 1, oc);
    const double osz = size(active + 1);
    vset(t1, trial.d);
    vsub(t1, c);
    vset(t2, c);
    vsub(t2, oc);
    double A = dd(t1, t1);
    double B = 2. * dd(t1, t2);
    double Cc = dd(t2, t2) - 2. / 3. * osz * osz;
    double X = quad_root(A, B, Cc, ok);
    if (fabs(X - 1.) < kLow) X = 1.;
    if (X < 1.) {  // the surface would move the wrong way
      ok = false;
      return;
    }
    vset(x, c);
    vaxpy(x, t1, X);
    vscale(x, (1.0 - sz / osz));
    vset(t2, c);
    vaxpy(t2, oc, -sz / osz);
    vsub(x, t2);
    Ten dir;
    dir.from_full(x, false);
    if (dir.dev_length() < kLow) return;
    vset(x, dir.d);
    A = dd(x, x);
    B = -2 * dd(t1, x);
    if (fabs(B) < kLow) B = 0.;
    Cc = dd(t1, t1) - 2. / 3. * sz * sz;
    if (fabs(Cc) < kLow || fabs(Cc) / dd(t1, t1) < kLow) return;
    if ((fabs(B) < 1.0e-10) && (fabs(Cc) < 1.0e-10)) return;  // tiny coefficients: no motion
    if (B > 0. || Cc < 0.) {
      ok = false;
      return;
    }
    X = quad_root(A, B, Cc, ok);
    vaxpy(c, x, X);
    set_center(active, c);
  }

  FX_PIMY_HD void move_inner_surfaces() {  // updateInnerSurface
    if (active <= 1) return;
    double dv[6], c[6];
    vset(dv, cur.d);
    center(active, c);
    const double sz = size(active);
    for (int i = 1; i < active; ++i) {
      double nc[6];
      vset(nc, c);
      vsub(nc, dv);
      vscale(nc, size(i) / sz);
      vadd(nc, dv);
      set_center(i, nc);
    }
  }

  // getTangent in compact form (kTan values): stage, G, K, the rank-one coefficient and the
  // deviator about the active surface's center; compact_D expands it to the 6 x 6 tangent.
  FX_PIMY_HD void compact(double* t) const {
    t[0] = stage;
    t[1] = G;
    t[2] = K;
    double coeff = 0., dv[6] = {0., 0., 0., 0., 0., 0.};
    if (stage == 1 && active > 0) {
      double c[6];
      vset(dv, trial.d);
      center(active, c);
      vsub(dv, c);
      const double sz = size(active), h = hmod(active);
      coeff = 6. * G * G / (2. * G + h) / sz / sz;
    }
    t[3] = coeff;
    for (int i = 0; i < 6; ++i) t[4 + i] = dv[i];
  }
  FX_PIMY_HD void tangent(double* D) const {  // getTangent, D[6 i + j]
    double t[10];
    compact(t);
    compact_D(t, D);
  }

  // setTrialStrain + getStress; with `stop`, the compacted corrector's predictor: returns true at the
  // first stress correction (the trial state then is partial: update_compact redoes the update)
  FX_PIMY_HD bool run(const double* eps, bool stop = false) {
    cur.load(C, S_STRESS);
    strain.load(C, S_STRAIN);
    active_c = static_cast<int>(C[S_ACTIVE]);
    active = active_c;
    e2p = static_cast<int>(C[S_E2P]);
    G = C[S_G];
    K = C[S_K];
    double w[6], cs[6];
    vset(w, eps);
    strain.engineering(cs);
    vsub(w, cs);
    rate.from_full(w, true);
    if (stage == 1 && e2p == 0) elastic_to_plastic();
    if (stage != 1) {  // linear elastic: sigma += D rate, column by column
      double D[36], a[6], r[6];
      tangent(D);
      vset(a, cur.t);
      rate.engineering(r);
      for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) a[j] += D[6 * j + i] * r[i];
      trial.from_full(a, false);
      return false;
    }
    active = active_c;
    sub = rate;
    set_trial_stress(cur);
    if (reversal()) {
      move_inner_surfaces();
      active = 0;
    }
    const int nsub = set_sub_rate();
    for (int i = 0; i < nsub; i++) {
      if (i == 0) set_trial_stress(cur);
      else set_trial_stress(trial);
      if (active == 0 && !crossing_next()) continue;
      if (stop) return true;
      if (active == 0) active++;
      correct(0);
      move_active_surface();
    }
    double vol = K * (rate.m * 3.);
    vol += cur.m;
    double dv[6];
    vset(dv, trial.d);
    trial.from_dev(dv, vol);
    return false;
  }

  FX_PIMY_HD void finish(double* sig, double* D) {  // the tangent (D may be NULL), the outputs, the trial state
    if (D) tangent(D);
    for (int i = 0; i < 6; ++i) sig[i] = ok ? trial.t[i] : static_cast<double>(NAN);
    double w[6];
    vset(w, strain.t);
    vadd(w, rate.t);
    Ten at_commit;
    at_commit.from_full(w, false);
    trial.store(T, S_STRESS);
    at_commit.store(T, S_STRAIN);
    T[S_E2P] = e2p;
    T[S_G] = G;
    T[S_K] = K;
    T[S_ACTIVE] = stage == 1 ? active : active_c;
    if (full) touch();
    T[S_CHANGED] = dirty ? 1.0 : 0.0;
  }
};

// The update of one point: trial state, stress and tangent (D[6 i + j]) at total strain eps.
template <class CV, class TV>
FX_PIMY_HD inline bool update(const Params& p, int stage, CV C, TV T, const double* eps, double* sig, double* D) {
  Point<CV, TV> pt(p, stage, C, T);
  pt.run(eps);
  pt.finish(sig, D);
  return pt.ok;
}

// The same with the tangent in compact form t[kTan]; *plastic: an active yield surface. Copy on
// write: the trial state's surfaces are written only if the update changed them (value S_CHANGED),
// so a commit copies the surfaces of those points only.
template <class CV, class TV>
FX_PIMY_HD inline bool update_compact(const Params& p, int stage, CV C, TV T, const double* eps, double* sig, double* t,
                                 bool* plastic) {
  Point<CV, TV> pt(p, stage, C, T);
  pt.full = false;
  pt.run(eps);
  pt.finish(sig, nullptr);
  pt.compact(t);
  *plastic = stage == 1 && pt.active > 0;
  return pt.ok;
}

// The compacted corrector's predictor (the reference's PressureIndependMultiYield::predict,
// pressure_independ_multi_yield.hpp:243-253): the update up to its first stress correction. A point
// that needs none is finished as update_compact finishes it (stress, compact tangent, trial state)
// and false returned; otherwise true, and update_compact redoes the whole update (the same
// function: the same bits as the fused path).
template <class CV, class TV>
FX_PIMY_HD inline bool predict_compact(const Params& p, int stage, CV C, TV T, const double* eps, double* sig,
                                       double* t, bool* ok) {
  Point<CV, TV> pt(p, stage, C, T);
  pt.full = false;
  if (pt.run(eps, true)) return true;
  pt.finish(sig, nullptr);
  pt.compact(t);
  *ok = pt.ok;
  return false;
}

// The tangent at the committed state in compact form t[kTan] (betaKcomm damping; the reference's
// PressureIndependMultiYield::committed_tangent, src/physics/materials/
// pressure_independ_multi_yield.hpp:160-168): getTangent after commitState, the trial stress,
// active surface, moduli and surfaces all the committed ones. C holds every surface.
template <class CV>
FX_PIMY_HD inline void committed_compact(const Params& p, int stage, CV C, double* t) {
  Point<CV, CV> pt(p, stage, C, C);
  pt.cur.load(C, S_STRESS);
  pt.trial = pt.cur;
  pt.active = static_cast<int>(C[S_ACTIVE]);
  pt.G = C[S_G];
  pt.K = C[S_K];
  pt.compact(t);
}

}  // namespace pimy
}  // namespace fx
