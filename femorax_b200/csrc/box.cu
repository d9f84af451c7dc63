// Box execution path, host side: the plan (grid detection, node -> equation words, coefficient
// modes), the coefficient tables, the autotuner and the batched entry points. The kernels and
// their launch shapes are in box_kernels.cuh.
#include <algorithm>
#include <cstring>
#include <cmath>

#include "box_kernels.cuh"

namespace fx {
namespace boxk {
// instantiated in box_f64_apply.cu, box_f64_force.cu, box_f64_forcew.cu and their FP32 twins
extern template void launch<double, 0>(const BoxPlan&, const BoxArgs<double>&, cudaStream_t);
extern template void launch<double, 1>(const BoxPlan&, const BoxArgs<double>&, cudaStream_t);
extern template void launch<float, 0>(const BoxPlan&, const BoxArgs<float>&, cudaStream_t);
extern template void launch<float, 1>(const BoxPlan&, const BoxArgs<float>&, cudaStream_t);
extern template void launch<double, 2>(const BoxPlan&, const BoxArgs<double>&, cudaStream_t);
extern template void launch<float, 2>(const BoxPlan&, const BoxArgs<float>&, cudaStream_t);
}  // namespace boxk
using namespace boxk;

namespace {

// ------------------------------------------------------------------ coefficients
// Exact element operator on a box with sides h. With J = hx hy hz / 8, rho_d = 2 / h_d, and
// w(0) = 2, w(1) = 2/3 (integrals of 1 and xi^2 over [-1, 1]), for mode m of component c:
//   diag = 2 J [ (lambda + mu) [m_c] rho_c^2 prod_{e != c} w(m_e)
//                + mu sum_{d: m_d} rho_d^2 prod_{e != d} w(m_e) ] (stiffness)
//          + rho J prod_e w(m_e) (consistent mass) or 8 rho J (lumped mass, H^T H = 8 I),
// couplings 4 J rho_c0 rho_c1 w(r) lambda (resp. mu); all scaled by 1/64 for the two
// unnormalised transforms. Apply: stiffness factor cK + c0 + cc (the elastic tangents are one
// matrix), mass factor cM'. Force: stiffness factor 1 (on u + beta v), no mass (the lumped
// alphaM masses act in nodal space), body force b J on mode 0.
void build_coef(ForceState& s, int mode, const double k[3]) {
  BoxPlan& p = s.box;
  const double J = p.h[0] * p.h[1] * p.h[2] / 8.0;
  const double rd[3] = {2.0 / p.h[0], 2.0 / p.h[1], 2.0 / p.h[2]};
  auto w = [](int bit) { return bit ? 2.0 / 3.0 : 2.0; };
  std::vector<BoxCoef> h(static_cast<size_t>(s.nparams));
  std::vector<BoxCoef32> h32(static_cast<size_t>(s.nparams));
  BoxScaled sc0{};  // scaled grids: set 0's stiffness (per element times E_e / E_0) and its mass
  const int32_t nbuild = p.scaled ? 1 : s.nparams;  // a scaled grid needs set 0 only
  for (int32_t i = 0; i < nbuild; ++i) {
    const ParamGP& q = s.params_h[i];
    double l2m, lam, mu;
    lame(q, l2m, lam, mu);
    double sk = 1.0, sm = 0.0;
    if (mode != 1) {  // the operator (0) or the mass product (2): factors of the coefficients k
      const OpFactors f = op_factors(q, k[0], k[1], k[2]);
      sk = f.cK + f.c0 + f.cc;
      sm = f.cM;
    }
    const bool cons = q.mass_type == 0;
    BoxCoef c{};
    for (int comp = 0; comp < 3; ++comp)
      for (int m = 0; m < 8; ++m) {
        auto bit = [&](int d) { return (m >> d) & 1; };
        double dk = 0.0;
        if (bit(comp)) {
          double pw = 1.0;
          for (int e = 0; e < 3; ++e)
            if (e != comp) pw *= w(bit(e));
          dk += (lam + mu) * rd[comp] * rd[comp] * pw;
        }
        for (int d = 0; d < 3; ++d) {
          if (!bit(d)) continue;
          double pw = 1.0;
          for (int e = 0; e < 3; ++e)
            if (e != d) pw *= w(bit(e));
          dk += mu * rd[d] * rd[d] * pw;
        }
        dk *= 2.0 * J * sk;
        const double dm = cons ? sm * q.rho * J * w(bit(0)) * w(bit(1)) * w(bit(2)) : 8.0 * sm * q.rho * J;
        c.grp[m ^ (1 << comp)][comp] = (dk + dm) / 64.0;
        if (i == 0) {
          sc0.grp[m ^ (1 << comp)][comp] = dk / 64.0;
          sc0.dmm[m] = dm / 64.0;
        }
      }
    // couplings of axis pair pr (components pr, pr + 1 mod 3; third axis e): lambda part for
    // r = 0 in group 0 and for r = 1 in group 2^e; mu part for r = 0 in group 2^c0 + 2^c1 and
    // for r = 1 in group 7
    for (int pr = 0; pr < 3; ++pr) {
      const int c0 = pr, c1 = (pr + 1) % 3, e = (pr + 2) % 3;
      const double base0 = 4.0 * J * rd[c0] * rd[c1] * w(0) * sk / 64.0;
      const double base1 = 4.0 * J * rd[c0] * rd[c1] * w(1) * sk / 64.0;
      if (pr == 0) c.grp[0][3] = base0 * lam;
      else c.more[pr - 1] = base0 * lam;
      c.grp[1 << e][3] = base1 * lam;
      c.grp[(1 << c0) | (1 << c1)][3] = base0 * mu;
      if (pr == 0) c.grp[7][3] = base1 * mu;
      else c.more[2 + pr - 1] = base1 * mu;
    }
    for (int d = 0; d < 3; ++d) c.body[d] = mode == 1 ? q.b[d] * J : 0.0;
    h[i] = c;
    BoxCoef32& f = h32[i];
    for (int g = 0; g < 8; ++g)
      for (int j = 0; j < 4; ++j) f.grp[g][j] = static_cast<float>(c.grp[g][j]);
    for (int j = 0; j < 4; ++j) f.more[j] = static_cast<float>(c.more[j]);
    for (int d = 0; d < 3; ++d) f.body[d] = static_cast<float>(c.body[d]);
    f.pad_ = 0.f;
  }
  BoxPlan::CoefSet& cs = p.cset[mode];
  if (p.layered)
    for (int32_t i = 0; i < s.nparams; ++i) {
      cs.tab.c[i] = h[i];
      cs.tab32.c[i] = h32[i];
    }
  if (p.scaled) {
    BoxScaled32 c32{};
    for (int g = 0; g < 8; ++g) sc0.grp[g][3] = h[0].grp[g][3];
    for (int j = 0; j < 4; ++j) sc0.more[j] = h[0].more[j];
    for (int d = 0; d < 3; ++d) sc0.body[d] = h[0].body[d];
    for (int g = 0; g < 8; ++g)
      for (int j = 0; j < 4; ++j) c32.grp[g][j] = static_cast<float>(sc0.grp[g][j]);
    for (int j = 0; j < 4; ++j) c32.more[j] = static_cast<float>(sc0.more[j]);
    for (int m = 0; m < 8; ++m) c32.dmm[m] = static_cast<float>(sc0.dmm[m]);
    for (int d = 0; d < 3; ++d) c32.body[d] = static_cast<float>(sc0.body[d]);
    if (cs.scoef.n != 1) cs.scoef.alloc(1);
    if (cs.scoef32.n != 1) cs.scoef32.alloc(1);
    FX_CUDA(cudaMemcpy(cs.scoef.ptr, &sc0, sizeof(sc0), cudaMemcpyHostToDevice));
    FX_CUDA(cudaMemcpy(cs.scoef32.ptr, &c32, sizeof(c32), cudaMemcpyHostToDevice));
  }
  if (!p.scaled) {  // (a scaled grid reads its one table only)
    if (cs.coef.n != h.size()) cs.coef.alloc(h.size());
    if (cs.coef32.n != h32.size()) cs.coef32.alloc(h32.size());
    FX_CUDA(cudaMemcpy(cs.coef.ptr, h.data(), h.size() * sizeof(BoxCoef), cudaMemcpyHostToDevice));
    FX_CUDA(cudaMemcpy(cs.coef32.ptr, h32.data(), h32.size() * sizeof(BoxCoef32), cudaMemcpyHostToDevice));
  }
  for (int j = 0; j < 3; ++j) cs.k[j] = k[j];
  cs.built = true;
}

void ensure_coef(ForceState& s, int mode, const double k[3]) {
  const BoxPlan& p = s.box;
  const BoxPlan::CoefSet& cs = p.cset[mode];
  if (cs.built && cs.k[0] == k[0] && cs.k[1] == k[1] && cs.k[2] == k[2]) return;
  build_coef(s, mode, k);
}

}  // namespace

int box_num_variants() { return kNumVariants; }

void box_prepare(ForceState& s, const double k[3]) { ensure_coef(s, 0, k); }

void box_set_launch(ForceState& s, int variant, int kz) {
  if (variant < 0 || variant >= kNumVariants) throw Error(FX_E_INVALID, "box launch variant out of range");
  if (kz == 0) throw Error(FX_E_INVALID, "kz must not be 0");
  for (auto& per_mode : s.box.shape)
    for (auto& sh : per_mode) {
      sh.variant = variant;
      sh.kz = kz > 0 ? kz : -kz;
      sh.persistent = kz < 0;
    }
  s.box.tuned = true;
}

// ------------------------------------------------------------------ plan
void box_build_plan(ForceState& s) {
  BoxPlan& p = s.box;
  p.qualifies = false;
  auto no = [&](const std::string& why) { p.why_not = why; };
  if (s.count == 0) return no("no elements");
  bool all_lumped = true;
  for (const auto& q : s.params_h) {
    if (q.kind != 0) return no("a parameter set is not elastic");
    if (q.element != 0) return no("a parameter set is not stdBrick");
    if (q.mass_type == 0) all_lumped = false;
  }
  const int32_t N = s.N, P = s.P;
  auto X = [&](int32_t n, int d) { return s.coords_h[static_cast<size_t>(d) * N + n]; };
  double h[3];
  {
    const int32_t n0 = s.node_h[0], n1 = s.node_h[static_cast<size_t>(1) * P], n3 = s.node_h[static_cast<size_t>(3) * P],
                  n4 = s.node_h[static_cast<size_t>(4) * P];
    h[0] = X(n1, 0) - X(n0, 0);
    h[1] = X(n3, 1) - X(n0, 1);
    h[2] = X(n4, 2) - X(n0, 2);
  }
  if (!(h[0] > 0 && h[1] > 0 && h[2] > 0)) return no("element 0 is not an axis-aligned box in stdBrick order");
  double lo[3] = {1e300, 1e300, 1e300};
  for (int32_t n = 0; n < N; ++n)
    for (int d = 0; d < 3; ++d) lo[d] = std::min(lo[d], X(n, d));
  const double tol = 1e-9;
  static const int ci[8] = {0, 1, 1, 0, 0, 1, 1, 0}, cj[8] = {0, 0, 1, 1, 0, 0, 1, 1}, ck[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  std::vector<int32_t> eidx(static_cast<size_t>(s.count) * 3);
  int mx[3] = {0, 0, 0};
  for (int32_t e = 0; e < s.count; ++e) {
    const int32_t n0 = s.node_h[e];
    int g[3];
    for (int d = 0; d < 3; ++d) {
      const double f = (X(n0, d) - lo[d]) / h[d];
      g[d] = static_cast<int>(std::lround(f));
      if (std::fabs(f - g[d]) > 1e-6) return no("element corner off the grid");
    }
    for (int a = 0; a < 8; ++a) {
      const int32_t n = s.node_h[static_cast<size_t>(a) * P + e];
      const int off[3] = {ci[a], cj[a], ck[a]};
      for (int d = 0; d < 3; ++d) {
        const double want = X(n0, d) + off[d] * h[d];
        if (std::fabs(X(n, d) - want) > tol * h[d] * (1.0 + std::fabs(g[d] + off[d])))
          return no("element is not a box of the common spacing");
      }
    }
    for (int d = 0; d < 3; ++d) {
      eidx[static_cast<size_t>(e) * 3 + d] = g[d];
      mx[d] = std::max(mx[d], g[d] + 1);
    }
  }
  const int nx = mx[0], ny = mx[1], nz = mx[2];
  if (static_cast<int64_t>(nx) * ny * nz != s.count) return no("elements do not fill a full grid");
  const int64_t NXn = nx + 1, NYn = ny + 1, NZn = nz + 1;
  std::vector<int32_t> cell(static_cast<size_t>(s.count), -1);
  std::vector<int32_t> gnode(static_cast<size_t>(NXn * NYn * NZn), -1);
  for (int32_t e = 0; e < s.count; ++e) {
    const int gi = eidx[static_cast<size_t>(e) * 3], gj = eidx[static_cast<size_t>(e) * 3 + 1],
              gk = eidx[static_cast<size_t>(e) * 3 + 2];
    int32_t& c = cell[(static_cast<size_t>(gk) * ny + gj) * nx + gi];
    if (c >= 0) return no("two elements in one grid cell");
    c = e;
    for (int a = 0; a < 8; ++a) {
      const int32_t n = s.node_h[static_cast<size_t>(a) * P + e];
      int32_t& gn = gnode[(static_cast<size_t>(gk + ck[a]) * NYn + gj + cj[a]) * NXn + gi + ci[a]];
      if (gn >= 0 && gn != n) return no("two nodes at one grid point");
      gn = n;
    }
  }
  // node -> equations: free DOFs must be consecutive equations; no equation shared by two nodes
  std::vector<int32_t> eq_of_node(static_cast<size_t>(N) * 3, -2);
  for (int32_t e = 0; e < s.count; ++e)
    for (int a = 0; a < 8; ++a) {
      const int32_t n = s.node_h[static_cast<size_t>(a) * P + e];
      for (int d = 0; d < 3; ++d) eq_of_node[static_cast<size_t>(n) * 3 + d] = s.eq_h[static_cast<size_t>(3 * a + d) * P + e];
    }
  std::vector<int32_t> packed(gnode.size(), 0);
  std::vector<char> eq_seen(static_cast<size_t>(s.neq), 0);
  bool full = true;
  for (size_t g = 0; g < gnode.size(); ++g) {
    const int32_t n = gnode[g];
    if (n < 0) return no("a grid point has no node");
    uint32_t mask = 0;
    int32_t base = -1, expect = -1;
    for (int d = 0; d < 3; ++d) {
      const int32_t q = eq_of_node[static_cast<size_t>(n) * 3 + d];
      if (q < 0) continue;
      if (q >= s.neq || eq_seen[q]) return no("equations shared between nodes (ties)");
      eq_seen[q] = 1;
      if (base < 0) {
        base = q;
        expect = q;
      }
      if (q != expect) return no("a node's equations are not consecutive");
      ++expect;
      mask |= 1u << d;
    }
    if (base >= (1 << 29)) return no("more than 2^29 equations");
    full = full && (mask == 0u || mask == 7u);
    packed[g] = static_cast<int32_t>((mask << 29) | static_cast<uint32_t>(base < 0 ? 0 : base));
  }
  std::vector<int32_t> eparam(static_cast<size_t>(s.count));
  for (size_t c = 0; c < cell.size(); ++c) eparam[c] = s.param_h[cell[c]];
  // layered: one parameter set per element plane, few sets and planes (kernel-parameter tables)
  p.layered = s.nparams <= kTableParams && nz <= kTableLayers;
  for (int k = 0; k < nz && p.layered; ++k) {
    const int32_t first = eparam[static_cast<size_t>(k) * nx * ny];
    for (int64_t c = 0; c < static_cast<int64_t>(nx) * ny; ++c)
      if (eparam[static_cast<size_t>(k) * nx * ny + c] != first) {
        p.layered = false;
        break;
      }
    for (auto& cs : p.cset) cs.tab.layer[k] = cs.tab32.layer[k] = static_cast<uint8_t>(first);
  }
  // scaled: many sets that differ only in E (per-element moduli): one table, per-element scales
  p.scaled = false;
  if (!p.layered && s.nparams > kParamsInShared) {
    const ParamGP& q0 = s.params_h[0];
    bool same = q0.E > 0.0;
    for (const auto& q : s.params_h)
      same = same && q.kind == 0 && q.E > 0.0 && q.nu == q0.nu && q.rho == q0.rho && q.b[0] == q0.b[0] &&
             q.b[1] == q0.b[1] && q.b[2] == q0.b[2] && q.alphaM == q0.alphaM && q.betaK == q0.betaK &&
             q.betaKinit == q0.betaKinit && q.betaKcomm == q0.betaKcomm && q.mass_type == q0.mass_type;
    if (same) {
      std::vector<double> es(eparam.size());
      std::vector<float> es32(eparam.size());
      for (size_t c = 0; c < eparam.size(); ++c) {
        es[c] = s.params_h[eparam[c]].E / q0.E;
        es32[c] = static_cast<float>(es[c]);
      }
      p.escale.upload(es);
      p.escale32.upload(es32);
      p.scaled = true;
    }
  }
  // force form: one beta, and lumped masses or no mass-proportional damping (then f_int has no
  // mass term and the mass type does not matter)
  const double beta0 = s.params_h[0].betaK + s.params_h[0].betaKinit + s.params_h[0].betaKcomm;
  bool one_beta = true;
  for (const auto& q : s.params_h) one_beta = one_beta && (q.betaK + q.betaKinit + q.betaKcomm) == beta0;
  bool no_alpha = s.nodal_alpha_h.empty() || std::all_of(s.nodal_alpha_h.begin(), s.nodal_alpha_h.end(),
                                                           [](double m) { return m == 0.0; });
  for (const auto& q : s.params_h) no_alpha = no_alpha && q.alphaM == 0.0;
  p.force_ok = one_beta && (all_lumped || no_alpha);
  p.beta = beta0;
  if (p.force_ok) {
    // lumped alphaM masses per equation: alphaM_e rho_e J per element corner, then the nodal ones
    const double J = h[0] * h[1] * h[2] / 8.0;
    std::vector<double> la(static_cast<size_t>(s.neq), 0.0);
    for (int32_t e = 0; e < s.count; ++e) {
      const ParamGP& q = s.params_h[s.param_h[e]];
      const double m = q.alphaM * q.rho * J;
      for (int k = 0; k < 24; ++k) {
        const int32_t eq = s.eq_h[static_cast<size_t>(k) * P + e];
        if (eq >= 0) la[eq] += m;
      }
    }
    for (size_t i = 0; i < s.nodal_alpha_h.size(); ++i) la[i] += s.nodal_alpha_h[i];
    p.la.upload(la);
  }
  p.full = full && s.neq >= 3;  // (the FULL gather addresses equation d < 3 of a fixed node)
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  for (int d = 0; d < 3; ++d) p.h[d] = h[d];
  p.node_eq.upload(packed);
  p.node_eq_h = std::move(packed);
  p.pipe.variant = -1;
  p.queue.upload(std::vector<int>(2, 0));
  p.elem_param.upload(eparam);
  p.grid_node_h = std::move(gnode);
  p.qualifies = true;
  p.why_not.clear();
  for (auto& cs : p.cset) cs.built = false;
}

// ------------------------------------------------------------------ operator entry points
template <class T>
static BoxArgs<T> args(const ForceState& s, int mode, const T* x, const T* v, T* y) {
  const BoxPlan::CoefSet& cs = s.box.cset[mode];
  const void* coef = sizeof(T) == 8 ? static_cast<const void*>(cs.coef.ptr) : static_cast<const void*>(cs.coef32.ptr);
  BoxArgs<T> a{};
  a.cset = mode;
  a.nx = s.box.nx;
  a.ny = s.box.ny;
  a.nz = s.box.nz;
  a.kz = s.box.shape[sizeof(T) == 4 ? 1 : 0][mode == 1 ? 1 : 0].kz;
  a.nparams = s.nparams;
  a.node_eq = s.box.node_eq.ptr;
  a.elem_param = s.box.elem_param.ptr;
  a.coef = coef;
  if (s.box.scaled) {
    if constexpr (sizeof(T) == 8) {
      a.coef = cs.scoef.ptr;
      a.escale = s.box.escale.ptr;
    } else {
      a.coef = cs.scoef32.ptr;
      a.escale = s.box.escale32.ptr;
    }
  }
  a.x = x;
  a.v = v;
  a.y = y;
  return a;
}

template <class T>
static void apply_t(ForceState& s, const double k[3], const T* x, T* y, cudaStream_t st, const int* skip) {
  ensure_coef(s, 0, k);
  BoxArgs<T> a = args<T>(s, 0, x, nullptr, y);
  a.skip = skip;
  if (k[2] != 0.0 && s.has_nodal_mass) {
    a.nm1 = s.nodal_mass.ptr;
    a.c1 = k[2];
  }
  if (k[1] != 0.0 && s.has_nodal_alpha) {
    a.nm2 = s.nodal_alpha_mass.ptr;
    a.c2 = k[1];
  }
  launch<T, 0>(s.box, a, st);
}

template <class T>
static void force_t(ForceState& s, const T* u, const T* v, T* f, cudaStream_t st) {
  const double k1[3] = {1.0, 0.0, 0.0};
  ensure_coef(s, 1, k1);
  BoxArgs<T> a = args<T>(s, 1, u, v, f);
  a.beta = static_cast<T>(s.box.beta);
  a.nm2 = s.box.la.ptr;
  launch<T, 1>(s.box, a, st);
}

// the force from w = u + beta v, formed by the caller (v: the velocity of the la v term)
template <class T>
static void force_w_t(ForceState& s, const T* w, const T* v, T* f, cudaStream_t st) {
  if (!s.box.force_ok) throw Error(FX_E_UNSUPPORTED, "box force form needs one beta, and lumped masses or no mass-proportional damping");
  const double k1[3] = {1.0, 0.0, 0.0};
  ensure_coef(s, 1, k1);
  BoxArgs<T> a = args<T>(s, 1, w, v, f);
  a.kz = s.box.shape[sizeof(T) == 4 ? 1 : 0][0].kz;  // one staged vector: the apply's shape
  a.nm2 = s.box.la.ptr;
  launch<T, 2>(s.box, a, st);
}

void box_mass_apply(ForceState& s, const double* x, double* y, cudaStream_t st) {
  const double k[3] = {0.0, 0.0, 1.0};
  ensure_coef(s, 2, k);
  BoxArgs<double> a = args<double>(s, 2, x, nullptr, y);
  if (s.has_nodal_mass) {
    a.nm1 = s.nodal_mass.ptr;
    a.c1 = 1.0;
  }
  launch<double, 0>(s.box, a, st);
}

void box_force_w(ForceState& s, const double* w, const double* v, double* f, cudaStream_t st) {
  force_w_t<double>(s, w, v, f, st);
}
void box_force_w_f32(ForceState& s, const float* w, const float* v, float* f, cudaStream_t st) {
  force_w_t<float>(s, w, v, f, st);
}

void box_apply(ForceState& s, const double k[3], const double* x, double* y, cudaStream_t st, const int* skip) {
  apply_t<double>(s, k, x, y, st, skip);
}
void box_apply_f32(ForceState& s, const double k[3], const float* x, float* y, cudaStream_t st, const int* skip) {
  apply_t<float>(s, k, x, y, st, skip);
}
void box_force(ForceState& s, const double* u, const double* v, double* f, cudaStream_t st) {
  if (!s.box.force_ok) throw Error(FX_E_UNSUPPORTED, "box force form needs one beta, and lumped masses or no mass-proportional damping");
  force_t<double>(s, u, v, f, st);
}
void box_force_f32(ForceState& s, const float* u, const float* v, float* f, cudaStream_t st) {
  if (!s.box.force_ok) throw Error(FX_E_UNSUPPORTED, "box force form needs one beta, and lumped masses or no mass-proportional damping");
  force_t<float>(s, u, v, f, st);
}

// Meshes below this many elements take the launch shape that is fastest on large grids (16 x 8
// columns, 8 planes) without timing.
constexpr int32_t kTuneMinElements = 262144;

// Times every launch variant and plane count, as a grid and as a persistent launch, on the operator
// (unit stiffness) and, where the box force form applies, on the internal force, each in FP64 and
// in FP32, and keeps the fastest of each of the four: CUDA events on the stream, L2 flushed before
// each launch, median of 5 after 2 warm-ups.
void box_autotune(ForceState& s, cudaStream_t st) {
  if (!s.box.qualifies) return;
  if (s.count < kTuneMinElements) {  // launch-bound: timing costs more than it can save
    for (auto& per_mode : s.box.shape)
      for (auto& sh : per_mode) sh = BoxPlan::Shape{};
    s.box.tuned = true;
    return;
  }
  const size_t n = static_cast<size_t>(std::max(s.neq, 1));
  DeviceArray<double> x, y;
  DeviceArray<float> x32, y32;
  x.alloc(n);
  y.alloc(n);
  x32.alloc(n);
  y32.alloc(n);
  x.zero(st);
  FX_CUDA(cudaMemsetAsync(x32.ptr, 0, sizeof(float) * n, st));
  // an apply inside a solve finds little of its operand in L2 (the solver's vectors are larger):
  // a write larger than L2 between the timed applies keeps the timing in that regime
  DeviceArray<unsigned char> flush;
  flush.alloc(static_cast<size_t>(256) << 20);
  const double k[3] = {1.0, 0.0, 0.0};
  cudaEvent_t e0, e1;
  FX_CUDA(cudaEventCreate(&e0));
  FX_CUDA(cudaEventCreate(&e1));
  // plane counts: fewer planes add redundant bottom planes (1 in kz + 1), more planes leave fewer
  // tiles to balance over the SMs; the best depends on the grid. Besides a fixed ladder, the counts
  // that split the grid's nz + 1 node planes evenly into 2 to 12 tiles (no short last tile).
  std::vector<int> kzs = {5, 6, 7, 8, 10, 12, 16, 32, 64};
  for (int t = 2; t <= 12; ++t) {
    const int kz = (s.box.nz + 1 + t - 1) / t;
    if (kz >= 5 && std::find(kzs.begin(), kzs.end(), kz) == kzs.end()) kzs.push_back(kz);
  }
  std::sort(kzs.begin(), kzs.end());
  // the internal force (ExplicitDifference steps, Newton residuals) stages u and v: its own shape
  for (int job = 0; job < 4; ++job) {
    const int prec = job & 1, mode = job >> 1;
    if (mode == 1 && !s.box.force_ok) continue;
    BoxPlan::Shape& sh = s.box.shape[prec][mode];
    BoxPlan::Shape best_shape;
    float best = 1e30f;
    for (int v = 0; v < kNumVariants; ++v)
      for (int kz : kzs)
        for (int pers = 0; pers < 2; ++pers) {
          if (kz > 8 && kz >= 2 * (s.box.nz + 1)) continue;
          sh = BoxPlan::Shape{v, kz, pers != 0};
          std::vector<float> times;
          try {
            for (int r = 0; r < 7; ++r) {
              FX_CUDA(cudaMemsetAsync(flush.ptr, r, flush.n, st));
              FX_CUDA(cudaEventRecord(e0, st));
              if (mode == 0 && prec == 0) box_apply(s, k, x.ptr, y.ptr, st, nullptr);
              else if (mode == 0) box_apply_f32(s, k, x32.ptr, y32.ptr, st, nullptr);
              else if (prec == 0) box_force(s, x.ptr, x.ptr, y.ptr, st);
              else box_force_f32(s, x32.ptr, x32.ptr, y32.ptr, st);
              FX_CUDA(cudaEventRecord(e1, st));
              FX_CUDA(cudaEventSynchronize(e1));
              float ms = 0.f;
              FX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
              if (r >= 2) times.push_back(ms);
            }
          } catch (const Error& e) {
            if (e.code != FX_E_UNSUPPORTED) throw;
            continue;  // a shape this mode's staging does not fit (checked before any launch)
          }
          std::sort(times.begin(), times.end());
          const float med = times[times.size() / 2];
          if (med < best) {
            best = med;
            best_shape = sh;
          }
        }
    sh = best_shape;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s.box.tuned = true;
}

// ------------------------------------------------------------------ batches of grids
// One launch shape for batches: 16 x 8 element columns, 4 CTAs per SM (FP64) or 6 (FP32), kBatchKz
// node planes per tile.
namespace {
constexpr int kBatchBX = 16, kBatchBY = 8, kBatchKz = 8;
template <class T>
constexpr int kBatchMinB = sizeof(T) == 4 ? 6 : 4;  // FP32 fits 6 CTAs per SM without spills

template <class T>
void batch_launch(const void* inst, const int4* work, int nwork, int* queue, cudaStream_t st) {
  using S = Smem<kBatchBX, kBatchBY, T, 0, kPerSet>;
  auto kern = k_box_batch<kBatchBX, kBatchBY, T, 0, kBatchMinB<T>>;
  // CTAs per SM (set once, thread-safe: serving threads launch this concurrently)
  static const int resident = [&] {
    int r = 0;
    FX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::bytes)));
    FX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, kern, kBatchBX * kBatchBY, S::bytes));
    return std::max(r, 1);
  }();
  const int ctas = queue ? std::min(nwork, resident * num_sms()) : nwork;
  kern<<<ctas, kBatchBX * kBatchBY, S::bytes, st>>>(static_cast<const BoxArgs<T>*>(inst), work, nwork, queue);
  FX_LAUNCH_CHECK("box_batch");
}

template <class T>
void fill_args(ForceState& s, const double k[3], const void* x, void* y, const int* skip, void* dst) {
  ensure_coef(s, 0, k);
  BoxArgs<T> a = args<T>(s, 0, static_cast<const T*>(x), nullptr, static_cast<T*>(y));
  a.kz = kBatchKz;
  a.skip = skip;
  if (k[2] != 0.0 && s.has_nodal_mass) {
    a.nm1 = s.nodal_mass.ptr;
    a.c1 = k[2];
  }
  if (k[1] != 0.0 && s.has_nodal_alpha) {
    a.nm2 = s.nodal_alpha_mass.ptr;
    a.c2 = k[1];
  }
  std::memcpy(dst, &a, sizeof(a));
}
}  // namespace

// ------------------------------------------------------------------ host-buffer apply in pieces
BoxPlan::HostPipe::~HostPipe() {
  for (cudaEvent_t e : ev_in) cudaEventDestroy(e);
  for (cudaEvent_t e : ev_comp) cudaEventDestroy(e);
  if (ev_start) cudaEventDestroy(ev_start);
  if (ev_done) cudaEventDestroy(ev_done);
  if (in) cudaStreamDestroy(in);
  if (comp) cudaStreamDestroy(comp);
  if (out) cudaStreamDestroy(out);
}

namespace {

constexpr int kHostChunks = 8;              // equation ranges of the host apply
constexpr int64_t kHostPipeMinEq = 262144;  // smaller meshes: one copy each way

// The ranges, the tile order and the final prefixes of y for the FP64 operator's shape. Tile
// (bx, by, bz) reads the nodes i0 - 1 .. i0 + BX - 1, j0 - 1 .. j0 + BY - 1 of planes k0 - 1 .. k1
// (the staged slots of box_tile, clipped to the grid) and owns, writing their equations,
// i0 .. i0 + BX - 2, j0 .. j0 + BY - 2 of planes k0 .. k1 - 1.
void build_pipe(ForceState& s) {
  BoxPlan& p = s.box;
  BoxPlan::HostPipe& h = p.pipe;
  const BoxPlan::Shape& sh = p.shape[0][0];
  if (h.variant == sh.variant && h.kz == sh.kz) return;
  const int BX = kVariantBlock[sh.variant][0], BY = kVariantBlock[sh.variant][1], kz = sh.kz;
  const int NX = p.nx + 1, NY = p.ny + 1, NZ = p.nz + 1;
  const int gx = (NX + BX - 2) / (BX - 1), gy = (NY + BY - 2) / (BY - 1), gz = (NZ + kz - 1) / kz;
  const int ntiles = gx * gy * gz;
  // first and last equation of each grid node (-1: none free)
  auto lo_of = [&](int64_t g) -> int64_t {
    const uint32_t w = static_cast<uint32_t>(p.node_eq_h[g]);
    return (w >> 29) ? static_cast<int64_t>(w & 0x1FFFFFFFu) : -1;
  };
  auto hi_of = [&](int64_t g) -> int64_t {
    const uint32_t w = static_cast<uint32_t>(p.node_eq_h[g]);
    const int n = __builtin_popcount(w >> 29);
    return n ? static_cast<int64_t>(w & 0x1FFFFFFFu) + n - 1 : -1;
  };
  std::vector<int64_t> need(ntiles, -1);
  for (int bz = 0; bz < gz; ++bz)
    for (int by = 0; by < gy; ++by)
      for (int bx = 0; bx < gx; ++bx) {
        const int t = (bz * gy + by) * gx + bx;
        const int i0 = bx * (BX - 1), j0 = by * (BY - 1), k0 = bz * kz, k1 = std::min(k0 + kz, NZ);
        for (int k = std::max(k0 - 1, 0); k <= std::min(k1, NZ - 1); ++k)
          for (int j = std::max(j0 - 1, 0); j <= std::min(j0 + BY - 1, NY - 1); ++j)
            for (int i = std::max(i0 - 1, 0); i <= std::min(i0 + BX - 1, NX - 1); ++i)
              need[t] = std::max(need[t], hi_of(static_cast<int64_t>(k) * NY * NX + static_cast<int64_t>(j) * NX + i));
      }
  const int C = kHostChunks;
  h.chunks = C;
  h.edge.assign(C + 1, 0);
  for (int c = 0; c <= C; ++c) h.edge[c] = static_cast<int64_t>(s.neq) * c / C;
  auto range_of = [&](int64_t q) {  // the range holding equation q (q < 0: the first)
    if (q < 0) return 0;
    return static_cast<int>(std::upper_bound(h.edge.begin(), h.edge.end(), q) - h.edge.begin()) - 1;
  };
  std::vector<int> order(ntiles), rng(ntiles);
  for (int t = 0; t < ntiles; ++t) {
    order[t] = t;
    rng[t] = range_of(need[t]);
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return rng[a] < rng[b]; });
  h.seg.assign(C + 1, 0);
  for (int t = 0; t < ntiles; ++t) ++h.seg[rng[t] + 1];
  for (int c = 0; c < C; ++c) h.seg[c + 1] += h.seg[c];
  // the range of each equation's owner tile, then y's final prefix after each range
  std::vector<int8_t> eq_rng(static_cast<size_t>(s.neq), -1);
  for (int bz = 0; bz < gz; ++bz)
    for (int by = 0; by < gy; ++by)
      for (int bx = 0; bx < gx; ++bx) {
        const int t = (bz * gy + by) * gx + bx;
        const int i0 = bx * (BX - 1), j0 = by * (BY - 1), k0 = bz * kz, k1 = std::min(k0 + kz, NZ);
        for (int k = k0; k < k1; ++k)
          for (int j = j0; j <= std::min(j0 + BY - 2, NY - 1); ++j)
            for (int i = i0; i <= std::min(i0 + BX - 2, NX - 1); ++i) {
              const int64_t g = static_cast<int64_t>(k) * NY * NX + static_cast<int64_t>(j) * NX + i;
              for (int64_t q = lo_of(g); q >= 0 && q <= hi_of(g); ++q) eq_rng[q] = static_cast<int8_t>(rng[t]);
            }
      }
  h.ready.assign(C, s.neq);
  int pm = -1, c = 0;
  for (int64_t q = 0; q < s.neq; ++q) {
    pm = std::max(pm, static_cast<int>(eq_rng[q]));
    for (; c < pm; ++c) h.ready[c] = q;  // ranges before pm end their prefix at q
  }
  h.tiles.upload(order);
  if (!h.in) {
    FX_CUDA(cudaStreamCreateWithFlags(&h.in, cudaStreamNonBlocking));
    FX_CUDA(cudaStreamCreateWithFlags(&h.comp, cudaStreamNonBlocking));
    FX_CUDA(cudaStreamCreateWithFlags(&h.out, cudaStreamNonBlocking));
    FX_CUDA(cudaEventCreateWithFlags(&h.ev_start, cudaEventDisableTiming));
    FX_CUDA(cudaEventCreateWithFlags(&h.ev_done, cudaEventDisableTiming));
  }
  while (static_cast<int>(h.ev_in.size()) < C) {
    cudaEvent_t a, b;
    FX_CUDA(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    FX_CUDA(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
    h.ev_in.push_back(a);
    h.ev_comp.push_back(b);
  }
  h.variant = sh.variant;
  h.kz = sh.kz;
}

bool page_locked(const void* ptr) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

}  // namespace

bool box_apply_host(ForceState& s, const double k[3], const double* xh, double* yh, cudaStream_t st) {
  if (!s.use_box() || s.neq < kHostPipeMinEq || !page_locked(xh) || !page_locked(yh)) return false;
  ensure_coef(s, 0, k);
  build_pipe(s);
  BoxPlan::HostPipe& h = s.box.pipe;
  BoxArgs<double> a = args<double>(s, 0, s.wx.ptr, nullptr, s.wy.ptr);
  if (k[2] != 0.0 && s.has_nodal_mass) {
    a.nm1 = s.nodal_mass.ptr;
    a.c1 = k[2];
  }
  if (k[1] != 0.0 && s.has_nodal_alpha) {
    a.nm2 = s.nodal_alpha_mass.ptr;
    a.c2 = k[1];
  }
  a.kz = s.box.shape[0][0].kz;
  // the three streams start after the work already on st
  FX_CUDA(cudaEventRecord(h.ev_start, st));
  FX_CUDA(cudaStreamWaitEvent(h.in, h.ev_start, 0));
  FX_CUDA(cudaStreamWaitEvent(h.comp, h.ev_start, 0));
  FX_CUDA(cudaStreamWaitEvent(h.out, h.ev_start, 0));
  for (int c = 0; c < h.chunks; ++c) {
    const int64_t e0 = h.edge[c], n = h.edge[c + 1] - e0;
    if (n > 0) FX_CUDA(cudaMemcpyAsync(s.wx.ptr + e0, xh + e0, sizeof(double) * n, cudaMemcpyHostToDevice, h.in));
    FX_CUDA(cudaEventRecord(h.ev_in[c], h.in));
  }
  int64_t sent = 0;
  for (int c = 0; c < h.chunks; ++c) {
    FX_CUDA(cudaStreamWaitEvent(h.comp, h.ev_in[c], 0));
    a.tiles = h.tiles.ptr + h.seg[c];
    a.ntiles = h.seg[c + 1] - h.seg[c];
    launch<double, 0>(s.box, a, h.comp);
    FX_CUDA(cudaEventRecord(h.ev_comp[c], h.comp));
    // the last range's wait also keeps the call from returning before every tile has run
    if (h.ready[c] > sent || c == h.chunks - 1) FX_CUDA(cudaStreamWaitEvent(h.out, h.ev_comp[c], 0));
    if (h.ready[c] > sent) {
      FX_CUDA(cudaMemcpyAsync(yh + sent, s.wy.ptr + sent, sizeof(double) * (h.ready[c] - sent),
                              cudaMemcpyDeviceToHost, h.out));
      sent = h.ready[c];
    }
  }
  FX_CUDA(cudaEventRecord(h.ev_done, h.out));
  FX_CUDA(cudaStreamWaitEvent(st, h.ev_done, 0));
  return true;
}

size_t box_args_bytes(bool f32) { return f32 ? sizeof(BoxArgs<float>) : sizeof(BoxArgs<double>); }

void box_fill_args(ForceState& s, const double k[3], bool f32, const void* x, void* y, const int* skip, void* dst) {
  if (!s.box.qualifies) throw Error(FX_E_UNSUPPORTED, "batched operator: not a box grid: " + s.box.why_not);
  if (s.box.scaled) throw Error(FX_E_UNSUPPORTED, "batched operator: per-element moduli are not batched");
  if (f32) fill_args<float>(s, k, x, y, skip, dst);
  else fill_args<double>(s, k, x, y, skip, dst);
}

void box_batch_tiles(const ForceState& s, int& gx, int& gy, int& gz) {
  gx = (s.box.nx + 1 + kBatchBX - 2) / (kBatchBX - 1);
  gy = (s.box.ny + 1 + kBatchBY - 2) / (kBatchBY - 1);
  gz = (s.box.nz + 1 + kBatchKz - 1) / kBatchKz;
}

void box_batch_apply(bool f32, const void* inst, const int4* work, int nwork, int* queue, cudaStream_t st) {
  if (nwork <= 0) return;
  if (f32) batch_launch<float>(inst, work, nwork, queue, st);
  else batch_launch<double>(inst, work, nwork, queue, st);
}

}  // namespace fx
