// PressureDependMultiYield at one material point, for the device and the host: multi-yield-surface
// plasticity with conical (Drucker-Prager type) surfaces, dilatancy, contraction and the
// phase-transformation zone of cyclic mobility (Yang, Elgamal and Parra's model for sands, OpenSees
// nDMaterial PressureDependMultiYield, three-dimensional form). The reference's material is
// src/physics/materials/pressure_depend_multi_yield.hpp (setup :122-170, setUpSurfaces :298-428,
// predict/correct :490-561, finish :563-607, elast2Plast :609-631 and the surface, potential and PPZ
// functions :633-1185, getTangent :1197-1239). The published algorithm's steps are followed in the
// same arithmetic order (built with --fmad=false), so that on the host a point gives OpenSees' bits.
// On the device the update's pow, exp, log and cos are fx_math.h's, built from IEEE-exact operations:
// the same bits as a host build of those functions, within 0.54 ulp, and the host C library's result
// on 99.6-100 % of arguments (one ulp apart otherwise). So the device update is, bit for bit, the
// reference's material linked to fx_math.h's functions (oracle/_ref/libfxref_fxmath.so), and differs
// from the C library's update only where a last-place difference turns a decision of the model.
//
// State of a point, nstate(ns) values through a strided view (as pimy.cuh): 0..12 stress, 13..25
// strain at the last commit, 26..38 reversal stress, 39..51 PPZ pivot, 52..64 PPZ center, 65..77
// lock stress (each: components, deviator, mean), then active surface, pressureD, onPPZ, PPZ size,
// cumulated dilative strain, its maximum, cumulated translation strain, the PPZ strain before and
// on the opposite side, the largest compression, switched to plastic; from 89 the ns surface centers.
// Sizes and plastic moduli are the material's (the same for every point).
#pragma once

#include <cmath>

#include "fx_math.h"
#include "pimy.cuh"

namespace fx {
namespace pdmy {

using pimy::dd;
using pimy::kLow;
using pimy::kMaxSurfaces;
using pimy::kPi;
using pimy::kUp;
using pimy::Slab;
using pimy::Ten;
using pimy::to_int;
using pimy::vadd;
using pimy::vaxpy;
using pimy::vdiv;
using pimy::vmul;
using pimy::vscale;
using pimy::vset;
using pimy::vsub;

// The update's elementary functions (unqualified calls below find these): the C library's on the
// host, fx_math.h's on the device.
FX_HD double pow(double x, double y) {
#ifdef __CUDA_ARCH__
  return fxm_pow(x, y);
#else
  return std::pow(x, y);
#endif
}
FX_HD double exp(double x) {
#ifdef __CUDA_ARCH__
  return fxm_exp(x);
#else
  return std::exp(x);
#endif
}
FX_HD double log(double x) {
#ifdef __CUDA_ARCH__
  return fxm_log(x);
#else
  return std::log(x);
#endif
}
FX_HD double cos(double x) {
#ifdef __CUDA_ARCH__
  return fxm_cos(x);
#else
  return std::cos(x);
#endif
}

constexpr double kLock = 1.0e+30;  // MultiYieldSurface's LOCK_VALUE

enum : int {
  S_STRESS = 0, S_STRAIN = 13, S_REV = 26, S_PIVOT = 39, S_PPZC = 52, S_LOCK = 65, S_ACTIVE = 78, S_PD = 79,
  S_ONPPZ = 80, S_PPZSIZE = 81, S_CUMD = 82, S_MAXCUMD = 83, S_CUMT = 84, S_PREPPZ = 85, S_OPPO = 86, S_MAXP = 87,
  S_E2P = 88, S_CENTERS = 89
};
FX_PIMY_HD constexpr int nstate(int ns) { return S_CENTERS + 6 * ns; }

struct Params {
  int ns;
  double rho, G0, K0, phi, gamma_peak, pref, c, n_press, phi_pt, contrac, dilat1, dilat2, liq1, liq2, liq4, e0,
      cs1, cs2, cs3, pa, hv, pv;
  double p_res, ratio_pt, strain_pt;  // from the surfaces' set-up
  double size[kMaxSurfaces + 1], modulus[kMaxSurfaces + 1];
};

// Constructor checks and setUpSurfaces: in23 = rho, refShearModul, refBulkModul, frictionAng,
// peakShearStra, refPress, pressDependCoe, PTAng, contrac, dilat1, dilat2, liquefac1, liquefac2,
// liquefac3, noYieldSurf, e, cs1, cs2, cs3, pa, c, hv, pv; pairs = noYieldSurf (gamma, G/Gmax) pairs
// or NULL. Error codes as pimy::setup.
inline int setup(const double* in, const double* pairs, Params& p) {
  double phi = in[3], phi_pt = in[7], c = in[20], n_press = in[6], cs1 = in[16];
  int ns = static_cast<int>(in[14]);
  const double G0 = in[1], K0 = in[2], gpeak = in[4], pr = in[5];
  if (G0 <= 0 || K0 <= 0 || phi <= 0. || phi >= 90. || phi_pt <= 0. || gpeak <= 0 || pr <= 0 || in[0] < 0 ||
      in[15] < 0)
    return pimy::kBadInput;
  if (phi_pt > phi) phi_pt = phi;
  if (c < 0) c = 0.;
  if (n_press < 0) n_press = 0.;
  if (ns <= 0) ns = 10;
  if (ns > 40) ns = 40;
  if (cs1 < 0) cs1 = 0.8;
  if (ns > kMaxSurfaces) return pimy::kTooManySurfaces;
  if (pairs != nullptr && ns < 2) return pimy::kTooFewPairs;
  p.ns = ns;
  p.rho = in[0];
  p.G0 = G0;
  p.K0 = K0;
  p.gamma_peak = gpeak;
  p.pref = -pr;
  p.c = c;
  p.n_press = n_press;
  p.contrac = in[8];
  p.dilat1 = in[9];
  p.dilat2 = in[10];
  p.liq1 = in[11];
  p.liq2 = in[12];
  p.liq4 = in[13];
  p.e0 = in[15];
  p.cs1 = cs1;
  p.cs2 = in[17];
  p.cs3 = in[18];
  p.pa = in[19];
  p.hv = in[21];
  p.pv = in[22];
  p.strain_pt = 0.;  // stays 0 if no surface pair brackets the phase-transformation ratio
  for (int i = 0; i <= kMaxSurfaces; ++i) p.size[i] = p.modulus[i] = 0.0;
  double p_res = 0.0, ratio_pt = 0.0, cone;
  auto segment = [&](double s1, double e1, double s2, double e2) {
    const double ep = 2. * (s2 - s1) / (e2 - e1);
    return (2. * G0 - ep) <= 0 ? kUp : (2. * G0 * ep) / (2. * G0 - ep);
  };
  if (pairs == nullptr) {  // hyperbolic backbone
    const double sinphi = std::sin(phi * kPi / 180.);
    const double M = 6. * sinphi / (3. - sinphi);
    const double sinpt = std::sin(phi_pt * kPi / 180.);
    ratio_pt = 6. * sinpt / (3. - sinpt);
    p_res = 2 * c / M;
    if (p_res < 0.0001 * p.pa) p_res = 0.0001 * p.pa;
    cone = -(p.pref - p_res);
    const double peak = std::sqrt(2.) * cone * M / 3.;
    const double gref = (gpeak * peak) / (G0 * gpeak - peak);
    const double step = peak / ns;
    for (int i = 1; i <= ns; i++) {
      const double s1 = i * step, s2 = s1 + step;
      const double r1 = 3. * s1 / std::sqrt(2.) / cone, r2 = 3. * s2 / std::sqrt(2.) / cone;
      const double e1 = s1 * gref / (G0 * gref - s1), e2 = s2 * gref / (G0 * gref - s2);
      if (r1 <= ratio_pt && r2 >= ratio_pt) {
        const double f = (r2 - ratio_pt) / (r2 - r1);
        p.strain_pt = e2 - f * (e2 - e1);
      }
      double h = segment(s1, e1, s2, e2);
      if (h < 0) h = 0;
      if (h > kUp) h = kUp;
      if (i == ns) h = 0;
      p.size[i] = r1;
      p.modulus[i] = h;
    }
  } else {  // user backbone: the cone from the last pair's strength
    const int last = 2 * (ns - 1);
    const double tmax = G0 * pairs[last] * pairs[last + 1];
    const double M = -(std::sqrt(3.) * tmax - 2. * c) / p.pref;
    p_res = 2 * c / M;
    if (p_res < 0.0001 * p.pa) p_res = 0.0001 * p.pa;
    cone = -(p.pref - p_res);
    const double sinphi = 3 * M / (6 + M);
    if (sinphi < 0. || sinphi > 1.) return pimy::kBadFriction;
    phi = std::asin(sinphi) * 180 / kPi;
    if (phi_pt > phi) phi_pt = phi;
    const double sinpt = std::sin(phi_pt * kPi / 180.);
    ratio_pt = 6. * sinpt / (3. - sinpt);
    for (int i = 1; i < ns; i++) {
      const int k = 2 * (i - 1);
      const double e1 = pairs[k], s1 = G0 * pairs[k + 1] * e1;
      const double e2 = pairs[k + 2], s2 = G0 * pairs[k + 3] * e2;
      const double r1 = std::sqrt(3.) * s1 / cone, r2 = std::sqrt(3.) * s2 / cone;
      if (r1 <= ratio_pt && r2 >= ratio_pt) {
        const double f = (r2 - ratio_pt) / (r2 - r1);
        p.strain_pt = std::sqrt(6.) / 3 * (e2 - f * (e2 - e1));  // octahedral: sqrt(6)/3 gamma_12
      }
      double h = segment(s1, e1, s2, e2);
      if (h <= 0) return pimy::kBadModulus;
      if (h > kUp) h = kUp;
      p.size[i] = r1;
      p.modulus[i] = h;
      if (i == ns - 1) {
        p.size[i + 1] = r2;
        p.modulus[i + 1] = 0;
      }
    }
  }
  p.p_res = p_res;
  p.phi = phi;
  p.phi_pt = phi_pt;
  p.ratio_pt = ratio_pt;
  return pimy::kOk;
}

template <class V>
FX_PIMY_HD inline void initial_state(const Params& p, const V& s) {
  for (int k = 0; k < nstate(p.ns); ++k) s[k] = 0.0;
  s[S_ONPPZ] = -1;
}

FX_PIMY_HD inline void elastic_D(const Params& p, double factor, double* D) {  // elastic_tangent, D[6 i + j]
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double v = 0.;
      if (i == j) v += p.G0 * factor;
      if (i < 3 && j < 3 && i == j) v += p.G0 * factor;
      if (i < 3 && j < 3) v += (p.K0 - 2. * p.G0 / 3.) * factor;
      D[6 * i + j] = v;
    }
}

// The tangent D[6 i + j] of a compact form t[kTan] (Point::compact): the reference elastic tangent in
// the elastic stage; in the plastic stage getTangent's expression from the point's moduli G, K, its
// coefficients c1 (volumetric) and c2 and the normal's deviator w.
constexpr int kTan = 11;
FX_PIMY_HD inline void compact_D(const Params& p, const double* t, double* D) {
  if (t[0] != 1.0) {
    elastic_D(p, 1.0, D);
    return;
  }
  const double G = t[1], Kb = t[2], c1 = t[3], c2 = t[4];
  const double* w = t + 5;
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double v = -c2 * w[i] * w[j];
      if (i == j) v += G;
      if (i < 3 && j < 3 && i == j) v += G;
      if (i < 3 && j < 3) v += (Kb - 2. * G / 3. - c1);
      D[6 * i + j] = v;
    }
}

// One point's update from the committed state C to the trial state T at total strain eps
// (engineering shear): OpenSees' setTrialStrain + getStress + getTangent, the instance's members as
// locals, the trial buffer holding the surface centers being worked on.
template <class CV, class TV>
struct Point {
  const Params& P;
  int stage;
  CV C;
  TV T;
  bool ok = true;
  Ten cur, strain, trial, rev, pivot, ppzc, lock, rate, sub, tstrain;
  int active_c = 0, active = 0, e2p = 0, onppz = -1;
  double max_press = 0., pd = 0., ppz_size = 0., cumd = 0., maxcumd = 0., cumt = 0., preppz = 0., oppo = 0.;
  double mfac = 0.;  // modulusFactor of the last trial stress

  FX_PIMY_HD Point(const Params& p, int st, CV c, TV t) : P(p), stage(st), C(c), T(t) {}

  FX_PIMY_HD void center(int i, double* c) const {
    for (int k = 0; k < 6; ++k) c[k] = i == 0 ? 0. : T[S_CENTERS + 6 * (i - 1) + k];
  }
  FX_PIMY_HD void set_center(int i, const double* c) {
    for (int k = 0; k < 6; ++k) T[S_CENTERS + 6 * (i - 1) + k] = c[k];
  }

  FX_PIMY_HD void load() {
    cur.load(C, S_STRESS);
    strain.load(C, S_STRAIN);
    active_c = static_cast<int>(C[S_ACTIVE]);
    e2p = static_cast<int>(C[S_E2P]);
    max_press = C[S_MAXP];
    rev.load(C, S_REV);
    pivot.load(C, S_PIVOT);
    ppzc.load(C, S_PPZC);
    lock.load(C, S_LOCK);
    active = active_c;
    pd = C[S_PD];
    onppz = static_cast<int>(C[S_ONPPZ]);
    ppz_size = C[S_PPZSIZE];
    cumd = C[S_CUMD];
    maxcumd = C[S_MAXCUMD];
    cumt = C[S_CUMT];
    preppz = C[S_PREPPZ];
    oppo = C[S_OPPO];
  }

  FX_PIMY_HD double yield(const Ten& s, int i) const {  // yieldFunc
    const double h = s.m - P.p_res;
    double w[6], c[6];
    vset(w, s.d);
    center(i, c);
    vaxpy(w, c, -h);
    const double sz = P.size[i] * h;
    return 3. / 2. * dd(w, w) - sz * sz;
  }

  FX_PIMY_HD void scale_deviator(Ten& s, int i) {  // deviatorScaling, its recursion as a loop
    for (int it = 0; it < 100000; ++it) {
      const double diff = yield(s, i);
      const double h = s.m - P.p_res;
      if (i < P.ns && diff < 0.) {
        const double sz = -P.size[i] * h, dsz = sqrt(sz * sz + diff);
        double dv[6], w[6], c[6];
        vset(dv, s.d);
        vset(w, dv);
        center(i, c);
        vaxpy(w, c, -h);
        double f = (sz - dsz) / dsz;
        if (f < 1.e-13) f = 1.e-13;
        vaxpy(dv, w, f);
        s.from_dev(dv, s.m);
        continue;
      }
      if (i == P.ns && fabs(diff) > kLow) {
        const double sz = -P.size[i] * h;
        double w[6];
        vset(w, s.d);
        vscale(w, sz / sqrt(diff + sz * sz));
        s.from_dev(w, s.m);
      }
      return;
    }
    ok = false;
  }

  FX_PIMY_HD void init_surfaces() {  // initSurfaceUpdate
    if (active_c == 0) return;
    const double h = -(cur.m - P.p_res);
    double dv[6];
    vset(dv, cur.d);
    const double Ms = sqrt(3. / 2. * dd(dv, dv));
    if (active_c < P.ns) {
      double w[6];
      vmul(w, dv, (1. - P.size[active_c] * h / Ms));
      vdiv(w, -h);
      set_center(active_c, w);
    }
    for (int i = 1; i < active_c; ++i) {
      double w[6];
      vmul(w, dv, (1. - P.size[i] * h / Ms));
      vdiv(w, -h);
      set_center(i, w);
    }
    active = active_c;
  }

  FX_PIMY_HD void elastic_to_plastic() {  // elast2Plast
    e2p = 1;
    if (cur.m > 0.) {
      double dv[6];
      vset(dv, cur.d);
      cur.from_full(dv, false);
    }
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

  FX_PIMY_HD double modulus_factor(const Ten& s) const {  // getModulusFactor
    const double h = s.m - P.p_res;
    double f = h / (P.pref - P.p_res);
    f = pow(f, P.n_press);
    return (1.e-10 > f) ? 1.e-10 : f;
  }

  FX_PIMY_HD void set_trial_stress(const Ten& in) {  // setTrialStress (in may be `trial`)
    const Ten s = in;
    mfac = modulus_factor(s);
    double w[6];
    vset(w, s.d);
    vaxpy(w, sub.d, 2 * P.G0 * mfac);
    double B = P.K0 * mfac;
    if (P.hv != 0. && trial.m <= max_press && sub.m < 0.) {
      const double tp = fabs(trial.m - P.p_res);
      B = (B * P.hv * pow(tp, P.pv)) / (B + P.hv * pow(tp, P.pv));
    }
    double vol = s.m + sub.m * 3. * B;
    if (vol > 0.) vol = 0.;
    trial.from_dev(w, vol);
  }

  FX_PIMY_HD int set_sub_rate() {  // setSubStrainRate
    if (active == P.ns) return 1;
    if (rate.zero()) return 0;
    const double h = -(cur.m - P.p_res);
    const double f = modulus_factor(cur);
    double epm;
    if (active == 0) epm = 2 * P.G0 * f;
    else {
      const double pm = P.modulus[active] * f;
      epm = 2 * P.G0 * f * pm / (2 * P.G0 * f + pm);
    }
    double w[6];
    vmul(w, rate.d, epm);
    Ten st;
    st.from_full(w, false);
    const double single = P.size[P.ns] * h / P.ns;
    const double total = 3. * st.oct_shear() / sqrt(2.);
    int n = to_int(total / single + 1);
    if (n > P.ns) n = P.ns;
    const int n1 = to_int(rate.oct_shear_engr() / 1.0e-4);
    const int n2 = to_int(rate.m / 1.e-5);
    if (n1 > n) n = n1;
    if (n2 > n) n = n2;
    vmul(w, rate.t, 1.0 / n);
    sub.from_full(w, false);
    return n;
  }

  FX_PIMY_HD void contact_stress(Ten& out) const {  // getContactStress
    const double h = trial.m - P.p_res;
    double c[6], w[6];
    center(active, c);
    vset(w, trial.d);
    vaxpy(w, c, -h);
    const double Ms = sqrt(3. / 2. * dd(w, w));
    const double f = P.size[active] * (-h) / Ms;
    for (int k = 0; k < 6; ++k) w[k] = w[k] * f + c[k] * h;
    out.from_dev(w, trial.m);
  }

  FX_PIMY_HD void normal_at(const Ten& s, Ten& out) const {  // getSurfaceNormal
    const double h = s.m - P.p_res;
    double w[6], c[6], u[6];
    vset(w, s.d);
    center(active, c);
    const double sz = P.size[active];
    const double vol = h * (dd(c, c) - 2. / 3. * sz * sz) - dd(w, c);
    vaxpy(w, c, -h);
    vscale(w, 3.0);
    Ten n;
    n.from_dev(w, vol);
    n.unit(u);
    out.from_full(u, false);
  }

  FX_PIMY_HD int reversal(const Ten& s) const {  // isLoadReversal
    if (active == 0) return 0;
    Ten n;
    normal_at(s, n);
    double w[6];
    vset(w, trial.t);
    vsub(w, cur.t);
    return dd(w, n.t) < 0 ? 1 : 0;
  }

  FX_PIMY_HD int critical(const Ten& s) const {  // isCriticalState
    double vol = tstrain.m * 3.0;
    const double etr = P.e0 + vol + vol * P.e0;
    vol = strain.m * 3.0;
    const double ecu = P.e0 + vol + vol * P.e0;
    double ecr1, ecr2;
    if (P.cs3 != 0.) {
      ecr1 = P.cs1 - P.cs2 * pow(fabs(-s.m / P.pa), P.cs3);
      ecr2 = P.cs1 - P.cs2 * pow(fabs(-cur.m / P.pa), P.cs3);
    } else {
      ecr1 = P.cs1 - P.cs2 * log(fabs(-s.m / P.pa));
      ecr2 = P.cs1 - P.cs2 * log(fabs(-cur.m / P.pa));
    }
    if (ecu < ecr2 && etr < ecr1) return 0;
    if (ecu > ecr2 && etr > ecr1) return 0;
    return 1;
  }

  FX_PIMY_HD double ppz_limit(int which, const Ten& contact) const {  // getPPZLimits
    const double vol = -contact.m;
    double lim;
    if (vol >= P.liq1) lim = 0.;
    else {
      const double t = vol * kPi / P.liq1 / 2.;
      lim = P.liq2 * pow(cos(t), 3.);
    }
    return which == 1 ? lim : P.liq4 * lim;
  }

  FX_PIMY_HD void ppz_translation(const Ten& contact) {  // PPZTranslation
    if (P.liq1 == 0.) return;
    const double lim = ppz_limit(1, contact);
    if (lim == 0.) return;
    const double tlim = ppz_limit(2, contact);
    double w[6];
    vset(w, tstrain.d);
    vsub(w, pivot.d);
    Ten wt;
    wt.from_full(w, false);
    double t = wt.oct_shear_engr();
    if (cumt < t) cumt = t;
    if (maxcumd == 0.) t = tlim;
    else t = tlim * cumd / maxcumd;
    if (cumt > t) cumt = t;
  }

  FX_PIMY_HD void update_ppz(const Ten& contact) {  // updatePPZ
    Ten wt;
    double w[6];
    if (P.liq1 == 0.) {  // no PPZ
      if (onppz == 2) {
        for (int i = 0; i < 6; ++i) w[i] = tstrain.t[i] - pivot.t[i];
        wt.from_full(w, false);
        cumd = wt.oct_shear_engr();
      } else {
        onppz = 2;
        pivot = tstrain;
        cumd = 0.;
      }
      return;
    }
    if (onppz == 2) {  // dilating: the cumulated dilative strain
      pivot = tstrain;
      cumd += sub.oct_shear_engr();
      if (cumd > maxcumd) maxcumd = cumd;
      return;
    }
    const double lim = ppz_limit(1, contact), tlim = ppz_limit(2, contact);
    if (onppz == -1 || onppz == 0) {
      vset(w, tstrain.t);
      vsub(w, pivot.t);
      wt.from_full(w, false);
      if (wt.oct_shear_engr() > cumd) {
        const double vol = -contact.m;
        oppo = preppz;
        double r = (vol + P.p_res) / (-P.pref + P.p_res);
        r = pow(r, 1. - P.n_press);
        preppz = r * P.strain_pt;
        if (oppo == 0.) oppo = preppz;
      }
    }
    if (onppz > -1) ppz_size = lim + (preppz + oppo + tlim + maxcumd) / 2.;
    else ppz_size = lim + (preppz + oppo + maxcumd) / 2.;
    if (onppz == 0 || onppz == 1) {  // the new PPZ center
      vset(w, pivot.t);
      vsub(w, ppzc.t);
      wt.from_full(w, false);
      const double f = (ppz_size - cumt) / wt.oct_shear_engr();
      vset(w, pivot.t);
      vaxpy(w, wt.t, -f);
      ppzc.from_full(w, false);
    }
    vset(w, tstrain.t);
    vsub(w, ppzc.t);
    wt.from_full(w, false);
    const double t = dd(sub.t, w);
    if ((wt.oct_shear_engr() > ppz_size && t > 0.) || lim == 0.) {  // outside the PPZ
      vset(w, tstrain.t);
      vsub(w, pivot.t);
      wt.from_full(w, false);
      if (wt.oct_shear_engr() > cumd) {
        cumd = 0.;
        if (lim == 0.) maxcumd = 0.;
      }
      onppz = 2;
      pivot = tstrain;
      cumt = 0.;
    } else {  // inside
      if (onppz == 0 || onppz == 1) ppz_translation(contact);
      if (onppz == -1 || onppz == 0) lock = contact;
      if (onppz == 0) onppz = 1;
    }
  }

  FX_PIMY_HD double potential(const Ten& contact, const Ten& n) {  // getPlasticPotential
    const double cr_c = contact.dev_ratio(P.p_res);
    double t = cr_c / P.ratio_pt;
    const double fpt = (t * t - 1) / (t * t + 1) / 3.;
    double contract = fpt * P.contrac;
    if (contract > 0.) contract = -contract;
    if (contract < -5.0e4) contract = -5.0e4;
    double unload;
    t = cur.m - pd;
    if (t >= 0.) unload = 0.;
    else {
      const double hd = pd - P.p_res;
      double t1 = sqrt(3. / 2.) * cur.dev_length() + P.ratio_pt * hd;
      t = t1 / (-t);
      if (t < P.size[P.ns]) t = P.size[P.ns];
      t1 = (rev.m - P.p_res) / hd;
      unload = -sqrt(3. / 2.) * n.dev_length() * t1 / t;
    }
    const double cr = cur.dev_ratio(P.p_res), tr = trial.dev_ratio(P.p_res);
    const double shear = dd(cur.d, trial.d);
    double pp;
    if (fpt < 0.) {  // below the phase transformation
      if (pd == 0.) pp = contract;
      else if (trial.m >= pd) {
        pd = 0.;
        pp = contract;
      } else if (tr > cr && shear >= 0.)
        pp = contract;
      else
        pp = unload;
    } else {  // above
      if (tr > cr && shear >= 0.) {  // dilation
        if (pd == 0.) pd = cur.m;
        rev = cur;
        update_ppz(contact);
        if (onppz == -1 || onppz == 1) return kLock;
        double dil = critical(contact) ? 0 : fpt * P.dilat1 * exp(P.dilat2 * cumd);
        if (dil > 5.0e4) dil = 5.0e4;
        return dil;
      } else if (pd == 0.)
        pp = contract;
      else if (trial.m >= pd) {
        pd = 0.;
        pp = contract;
      } else
        pp = unload;
    }
    if (onppz > 0) onppz = 0;
    if (onppz != -1) ppz_translation(contact);
    if (critical(contact)) return 0.;
    return pp;
  }

  FX_PIMY_HD double loading(const Ten& contact, const Ten& n, double pp, int crossed) const {  // getLoadingFunc
    const double modul = P.modulus[active];
    const double t1 = 2. * P.G0 * mfac * dd(n.d, n.d);
    const double t2 = 9. * P.K0 * mfac * n.m * pp;
    double t = t1 + t2 + modul * mfac;
    const double limit = active == P.ns ? P.modulus[active - 1] * mfac / 2. : modul * mfac / 2.;
    if (t < limit) t = limit;
    double w[6];
    vset(w, trial.d);
    vsub(w, contact.d);
    double lf = dd(n.t, w) / t;
    if (lf < 0.) lf = 0;
    if (crossed) {
      t = (P.modulus[active - 1] - modul) / P.modulus[active - 1];
      lf *= t;
    }
    return lf;
  }

  FX_PIMY_HD bool crossing_next() const {  // isCrossingNextSurface
    if (active == P.ns) return false;
    return yield(trial, active + 1) > 0;
  }

  FX_PIMY_HD int correction(int crossed) {  // stressCorrection, its recursion as a loop; 1: locked
    for (;;) {
      Ten contact, n;
      contact_stress(contact);
      normal_at(contact, n);
      const double pp = potential(contact, n);
      if (pp == kLock && (onppz == -1 || onppz == 1)) {
        trial = lock;
        return 1;
      }
      const double tv = trial.m;
      const double lf = loading(contact, n, pp, crossed);
      double vol = tv - pp * 3 * P.K0 * mfac * lf;
      double w[6];
      vset(w, trial.d);
      if (vol > 0. && vol != tv) {
        double f = tv / (tv - vol);
        f *= -2 * P.G0 * mfac * lf;
        vaxpy(w, n.d, f);
        vol = 0.;
      } else if (vol > 0.) {
        vol = 0.;
      } else {
        const double f = -2 * P.G0 * mfac * lf;
        vaxpy(w, n.d, f);
      }
      trial.from_dev(w, vol);
      scale_deviator(trial, active);
      if (crossing_next()) {
        active++;
        crossed = 1;
        continue;
      }
      return 0;
    }
  }

  FX_PIMY_HD void move_active() {  // updateActiveSurface
    if (active == P.ns) return;
    const double h = trial.m - P.p_res;
    double t1[6], t2[6], c[6], oc[6], w[6];
    center(active, c);
    const double sz = P.size[active];
    center(active + 1, oc);
    const double osz = P.size[active + 1];
    vset(t1, trial.d);
    vaxpy(t1, c, -h);
    vset(t2, c);
    vsub(t2, oc);
    vscale(t2, h);
    double A = dd(t1, t1);
    double B = 2. * dd(t1, t2);
    double Cc = dd(t2, t2) - 2. / 3. * osz * osz * h * h;
    double X = pimy::quad_root(A, B, Cc, ok);
    if (fabs(X - 1.) < kLow) X = 1.;
    if (X < 1.) return;
    vmul(w, t1, X);
    vaxpy(w, c, h);
    vscale(w, (1.0 - sz / osz));
    vset(t2, c);
    vaxpy(t2, oc, -sz / osz);
    vscale(t2, h);
    vsub(w, t2);
    Ten dir;
    dir.from_full(w, false);
    if (dir.dev_length() < kLow) return;
    vset(w, dir.d);
    A = h * h * dd(w, w);
    B = 2 * h * dd(t1, w);
    if (fabs(B) < kLow) B = 0.;
    Cc = dd(t1, t1) - 2. / 3. * sz * sz * h * h;
    if (fabs(Cc) < kLow || fabs(Cc) / dd(t1, t1) < kLow) return;
    if (B > 0. || Cc < 0.) {
      ok = false;
      return;
    }
    X = pimy::quad_root(A, B, Cc, ok);
    vaxpy(c, w, -X);
    set_center(active, c);
  }

  FX_PIMY_HD void move_inner() {  // updateInnerSurface
    if (active <= 1) return;
    const double h = cur.m - P.p_res;
    double dv[6], c[6];
    vset(dv, cur.d);
    center(active, c);
    const double sz = P.size[active];
    for (int i = 1; i < active; ++i) {
      double w[6];
      vmul(w, c, h);
      vsub(w, dv);
      vscale(w, P.size[i] / sz);
      vadd(w, dv);
      vdiv(w, h);
      set_center(i, w);
    }
  }

  // getTangent in compact form (kTan values): stage, G, K, the two rank-one coefficients and the
  // normal's deviator; compact_D expands it.
  FX_PIMY_HD void compact(double* t) const {
    t[0] = stage;
    for (int k = 1; k < kTan; ++k) t[k] = 0.;
    if (stage != 1) return;
    const double f = modulus_factor(cur);
    const double G = f * P.G0;
    double Kb = f * P.K0;
    if (P.hv != 0. && trial.m <= max_press && rate.m < 0.) {
      const double tp = fabs(trial.m - P.p_res);
      Kb = (Kb * P.hv * pow(tp, P.pv)) / (Kb + P.hv * pow(tp, P.pv));
    }
    double w[6] = {0., 0., 0., 0., 0., 0.}, c1 = 0., c2 = 0.;
    if (active_c > 0) {  // the normal at the committed stress, to the trial active surface
      Ten n;
      normal_at(cur, n);
      vset(w, n.d);
      const double vol = n.m;
      const double Ho = 9. * Kb * vol * vol + 2. * G * dd(w, w);
      const double pm = f * P.modulus[active_c];
      c1 = 9. * Kb * Kb * vol * vol / (Ho + pm);
      c2 = 4. * G * G / (Ho + pm);
    }
    t[1] = G;
    t[2] = Kb;
    t[3] = c1;
    t[4] = c2;
    for (int k = 0; k < 6; ++k) t[5 + k] = w[k];
  }
  FX_PIMY_HD void tangent(double* D) const {  // getTangent, D[6 i + j]
    double t[kTan];
    compact(t);
    compact_D(P, t, D);
  }

  FX_PIMY_HD bool predict(const double* eps) {  // getStress up to the elastic-or-plastic decision
    load();
    double w[6], cs[6];
    vset(w, eps);
    strain.engineering(cs);
    vsub(w, cs);
    rate.from_full(w, true);
    for (int k = S_CENTERS; k < nstate(P.ns); ++k) T[k] = C[k];
    if (stage == 1 && e2p == 0) elastic_to_plastic();
    if (stage != 1) {  // linear elastic: sigma += D rate, column by column
      double D[36], r[6];
      elastic_D(P, 1.0, D);
      vset(w, cur.t);
      rate.engineering(r);
      for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) w[j] += D[6 * j + i] * r[i];
      trial.from_full(w, false);
      return false;
    }
    active = active_c;
    sub = rate;
    set_trial_stress(cur);
    if (active > 0 && reversal(cur)) {
      move_inner();
      active = 0;
    }
    if (active == 0 && !crossing_next()) {
      vset(w, strain.t);
      vadd(w, rate.t);
      tstrain.from_full(w, false);
      return false;
    }
    return true;
  }

  FX_PIMY_HD void correct() {  // the sub-increment loop of getStress
    const int nsub = set_sub_rate();
    for (int i = 0; i < nsub; i++) {
      double w[6];
      vset(w, strain.t);
      vaxpy(w, sub.t, (i + 1));
      tstrain.from_full(w, false);
      int is;
      if (i == 0) {
        set_trial_stress(cur);
        is = reversal(cur);
      } else {
        Ten prev;
        prev.from_full(trial.t, false);
        set_trial_stress(trial);
        is = reversal(prev);
      }
      if (active > 0 && is) {
        move_inner();
        active = 0;
      }
      if (active == 0 && !crossing_next()) continue;
      if (active == 0) active++;
      if (correction(0) == 0) move_active();
    }
  }

  FX_PIMY_HD void finish(double* sig, double* D) {  // the tangent, the outputs, the trial state
    if (D) tangent(D);
    for (int i = 0; i < 6; ++i) sig[i] = ok ? trial.t[i] : static_cast<double>(NAN);
    double w[6];
    vset(w, strain.t);
    vadd(w, rate.t);
    Ten at_commit;
    at_commit.from_full(w, false);
    trial.store(T, S_STRESS);
    at_commit.store(T, S_STRAIN);
    if (stage == 1) {
      rev.store(T, S_REV);
      pivot.store(T, S_PIVOT);
      ppzc.store(T, S_PPZC);
      lock.store(T, S_LOCK);
      T[S_ACTIVE] = active;
      T[S_PD] = pd;
      T[S_ONPPZ] = onppz;
      T[S_PPZSIZE] = ppz_size;
      T[S_CUMD] = cumd;
      T[S_MAXCUMD] = maxcumd;
      T[S_CUMT] = cumt;
      T[S_PREPPZ] = preppz;
      T[S_OPPO] = oppo;
      double mp = max_press;
      if (trial.m < mp) mp = trial.m;
      T[S_MAXP] = mp;
      T[S_E2P] = e2p;
    } else {  // the plastic values stay the committed ones
      for (int k = S_REV; k < S_CENTERS; ++k) T[k] = C[k];
    }
  }
};

// The update of one point: trial state, stress and tangent (D[6 i + j], NULL: not formed) at total
// strain eps.
template <class CV, class TV>
FX_PIMY_HD inline bool update(const Params& p, int stage, CV C, TV T, const double* eps, double* sig, double* D) {
  Point<CV, TV> pt(p, stage, C, T);
  if (pt.predict(eps)) pt.correct();
  pt.finish(sig, D);
  return pt.ok;
}

// The same with the tangent in compact form t[kTan]; *plastic: an active yield surface.
template <class CV, class TV>
FX_PIMY_HD inline bool update_compact(const Params& p, int stage, CV C, TV T, const double* eps, double* sig, double* t,
                                      bool* plastic) {
  Point<CV, TV> pt(p, stage, C, T);
  if (pt.predict(eps)) pt.correct();
  pt.finish(sig, nullptr);
  pt.compact(t);
  *plastic = stage == 1 && pt.active > 0;
  return pt.ok;
}

// The compacted corrector's predictor (the reference's PressureDependMultiYield::predict,
// pressure_depend_multi_yield.hpp:260-283): the elastic predictor; a point that stays elastic is
// finished as update_compact finishes it and false returned; otherwise true, and update_compact
// redoes the update (predictor and corrector: the same bits as the fused path).
template <class CV, class TV>
FX_PIMY_HD inline bool predict_compact(const Params& p, int stage, CV C, TV T, const double* eps, double* sig,
                                       double* t, bool* ok) {
  Point<CV, TV> pt(p, stage, C, T);
  if (pt.predict(eps)) return true;
  pt.finish(sig, nullptr);
  pt.compact(t);
  *ok = pt.ok;
  return false;
}

// The tangent at the committed state in compact form t[kTan] (betaKcomm damping; the reference's
// PressureDependMultiYield::committed_tangent, src/physics/materials/
// pressure_depend_multi_yield.hpp:186-200): the reference elastic tangent in the elastic stage or
// before the switch to plastic; otherwise getTangent after commitState, the trial stress and the
// surface centers the committed ones and no strain rate (so no volumetric softening).
template <class CV>
FX_PIMY_HD inline void committed_compact(const Params& p, int stage, CV C, double* t) {
  if (stage != 1 || C[S_E2P] == 0.0) {
    t[0] = 0.;
    for (int k = 1; k < kTan; ++k) t[k] = 0.;
    return;
  }
  Point<CV, CV> pt(p, stage, C, C);  // the centers read from C
  pt.load();
  pt.trial = pt.cur;
  double z[6] = {0., 0., 0., 0., 0., 0.};
  pt.rate.from_full(z, true);
  pt.compact(t);
}

}  // namespace pdmy
}  // namespace fx
