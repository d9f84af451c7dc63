// Box execution path: stdBrick meshes that are structured grids of equal axis-aligned boxes
// (every configuration of the structured benchmarks).
//
// Element operator. On an axis-aligned box the Jacobian is constant and diagonal, and 2x2x2 Gauss
// integrates the trilinear element's stiffness and consistent mass exactly, so the element
// operator of the reference's Gauss-point form equals, up to rounding, the exact bilinear form
// written in the Walsh-Hadamard (modal) basis of the 8 corner values: 1, xi, eta, zeta, xi eta,
// ... In that basis the mass is diagonal and the stiffness is diagonal plus 24 couplings, so one
// element costs 3 x 24 butterflies forward, 24 products, 24 fused couplings and 3 x 24
// butterflies back: about 190 FP64 operations instead of several thousand.
//
// Scatter. Each CTA owns a (BX-1) x (BY-1) column of grid nodes over kz node planes and sweeps up
// the planes: it stages a plane of x (with a one-node halo) in shared memory, evaluates the
// BX x BY element columns around its nodes (the halo elements are evaluated by both neighbours:
// no atomics, no cross-CTA exchange), keeps the element values in shared memory and gives each
// owned node the sum of its eight element values in a fixed order. Every equation is written
// once, by its owner, in a fixed order: deterministic, and y needs no zeroing.
#include <algorithm>
#include <cmath>
#include <map>

#include "force.hpp"

namespace fx {

namespace {

// corner c = i + 2j + 4k (lexicographic) -> stdBrick local node
__host__ __device__ constexpr int lex_to_local(int c) {
  return c == 0 ? 0 : c == 1 ? 1 : c == 2 ? 3 : c == 3 ? 2 : c == 4 ? 4 : c == 5 ? 5 : c == 6 ? 7 : 6;
}

template <class T>
struct BoxArgs {
  int nx, ny, nz, kz;
  const int32_t* __restrict__ node_eq;
  const int32_t* __restrict__ elem_param;
  const void* __restrict__ coef;  // BoxCoef or BoxCoef32
  const T* __restrict__ x;        // apply: x; force: u
  const T* __restrict__ v;        // force: v
  T* __restrict__ y;
  const double* __restrict__ nm1;  // nodal mass (apply: k.mass) or NULL
  const double* __restrict__ nm2;  // nodal alpha mass (apply: k.damping; force: 1) or NULL
  double c1, c2;
  const int* skip;  // when set and nonzero on the device, the launch does nothing (a finished solve)
};

template <class T>
struct Coef;
template <>
struct Coef<double> {
  using type = BoxCoef;
};
template <>
struct Coef<float> {
  using type = BoxCoef32;
};

// Unnormalised Walsh-Hadamard transform of 8 corner values (lexicographic), in place:
// for each axis bit b: (v_i, v_{i+b}) -> (v_i + v_{i+b}, v_{i+b} - v_i).
template <class T>
__device__ __forceinline__ void wht_fwd(T v[8]) {
#pragma unroll
  for (int b = 1; b < 8; b <<= 1)
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (!(i & b)) {
        const T a = v[i], c = v[i + b];
        v[i] = a + c;
        v[i + b] = c - a;
      }
}
// Its transpose: (g_i, g_{i+b}) -> (g_i - g_{i+b}, g_i + g_{i+b}).
template <class T>
__device__ __forceinline__ void wht_bwd(T v[8]) {
#pragma unroll
  for (int b = 4; b >= 1; b >>= 1)
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (!(i & b)) {
        const T a = v[i], c = v[i + b];
        v[i] = a - c;
        v[i + b] = a + c;
      }
}

// The modal element operator: t[c][m] (transformed corner values of component c) -> g[c][m].
// Axis pairs (c, d, e): (0,1,2), (1,2,0), (2,0,1); for r in {0,1}: modes a = bit c + r bit e,
// b = bit d + r bit e; lambda couples (c,a)<->(d,b), mu couples (c,b)<->(d,a).
template <class T, class C>
__device__ __forceinline__ void modal_apply(const C& k, const T t[3][8], T g[3][8]) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int m = 0; m < 8; ++m) g[c][m] = T(k.dkm[c][m]) * t[c][m];
#pragma unroll
  for (int pr = 0; pr < 3; ++pr) {
    const int c = pr, d = (pr + 1) % 3, e = (pr + 2) % 3;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int ma = (1 << c) | (r << e), mb = (1 << d) | (r << e);
      const T kl = T(k.kap[pr * 4 + r * 2 + 0]), km = T(k.kap[pr * 4 + r * 2 + 1]);
      g[d][mb] = fma(kl, t[c][ma], g[d][mb]);
      g[c][ma] = fma(kl, t[d][mb], g[c][ma]);
      g[d][ma] = fma(km, t[c][mb], g[d][ma]);
      g[c][mb] = fma(km, t[d][ma], g[c][mb]);
    }
  }
}

template <class T>
__device__ __forceinline__ T load_dof(const T* __restrict__ x, int32_t packed, int d) {
  const uint32_t mask = static_cast<uint32_t>(packed) >> 29;
  if (!((mask >> d) & 1u)) return T(0);
  const int32_t base = packed & 0x1FFFFFFF;
  return x[base + __popc(mask & ((1u << d) - 1u))];
}

template <int BX, int BY, class T, int MODE>
struct Smem {
  static constexpr int NT = BX * BY, SX = BX + 1, SY = BY + 1, NS = SX * SY;
  static constexpr int NV = MODE == 1 ? 2 : 1;  // staged vectors: x (apply) or u, v (force)
  static constexpr size_t bytes = sizeof(T) * (24 * NT + 2 * 3 * NS * NV) + sizeof(int32_t) * 2 * NS;
};

// MODE 0: y = K_eff x (+ nodal masses). MODE 1: f = K (u + beta v) + alphaM M v - body
// (+ nodal alphaM masses times v). CONSISTENT: the modal mass term (else lumped, nodal space).
template <int BX, int BY, class T, int MODE, bool CONSISTENT>
__global__ void __launch_bounds__(BX* BY) k_box(BoxArgs<T> a) {
  using S = Smem<BX, BY, T, MODE>;
  using CT = typename Coef<T>::type;
  constexpr int NT = S::NT, SX = S::SX, NS = S::NS, NV = S::NV;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ys = reinterpret_cast<T*>(smem_raw);  // [24][NT]: element values, (corner, component) major
  T* xs = ys + 24 * NT;                    // [2 planes][NV][3][NS]
  int32_t* es = reinterpret_cast<int32_t*>(xs + 2 * 3 * NS * NV);  // [2][NS]
  const CT* __restrict__ coef = reinterpret_cast<const CT*>(a.coef);
  if (a.skip && *a.skip) return;

  const int t = threadIdx.x;
  const int ci = t % BX, cj = t / BX;
  const int i0 = blockIdx.x * (BX - 1), j0 = blockIdx.y * (BY - 1);
  const int k0 = blockIdx.z * a.kz;
  const int k1 = min(k0 + a.kz, a.nz + 1);
  const int NXn = a.nx + 1, NYn = a.ny + 1;
  const int ei = i0 - 1 + ci, ej = j0 - 1 + cj;
  const bool col_ok = ei >= 0 && ei < a.nx && ej >= 0 && ej < a.ny;
  const int gi = i0 + ci, gj = j0 + cj;
  const bool own = ci < BX - 1 && cj < BY - 1 && gi < NXn && gj < NYn;

  auto stage = [&](int k, int b) {
    for (int s = t; s < NS; s += NT) {
      const int si = s % SX, sj = s / SX;
      const int ni = i0 - 1 + si, nj = j0 - 1 + sj;
      int32_t packed = 0;
      if (k >= 0 && k <= a.nz && ni >= 0 && ni < NXn && nj >= 0 && nj < NYn)
        packed = a.node_eq[(static_cast<int64_t>(k) * NYn + nj) * NXn + ni];
      es[b * NS + s] = packed;
#pragma unroll
      for (int d = 0; d < 3; ++d) xs[((b * NV + 0) * 3 + d) * NS + s] = load_dof(a.x, packed, d);
      if (MODE == 1) {
#pragma unroll
        for (int d = 0; d < 3; ++d) xs[((b * NV + 1) * 3 + d) * NS + s] = load_dof(a.v, packed, d);
      }
    }
  };

  T acc[3] = {T(0), T(0), T(0)};
  int buf = 0;
  stage(k0 - 1, 0);
  for (int ek = k0 - 1; ek < k1; ++ek) {
    stage(ek + 1, buf ^ 1);
    __syncthreads();
    // ---- element (ei, ej, ek)
    T out[8][3];
    if (col_ok && ek >= 0 && ek < a.nz) {
      const CT& k = coef[a.elem_param[(static_cast<int64_t>(ek) * a.ny + ej) * a.nx + ei]];
      T tv[3][8];
      T vv[3][8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int pb = (c & 4) ? (buf ^ 1) : buf;
        const int s = (ci + (c & 1)) + (cj + ((c >> 1) & 1)) * SX;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const T xv = xs[((pb * NV + 0) * 3 + d) * NS + s];
          if (MODE == 1) {
            const T vd = xs[((pb * NV + 1) * 3 + d) * NS + s];
            vv[d][c] = vd;
            tv[d][c] = fma(T(k.beta), vd, xv);
          } else {
            tv[d][c] = xv;
            vv[d][c] = xv;
          }
        }
      }
      T g[3][8];
#pragma unroll
      for (int d = 0; d < 3; ++d) wht_fwd(tv[d]);
      modal_apply(k, tv, g);
      if (MODE == 1 && CONSISTENT) {  // alphaM times the consistent mass, on v
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          T mv[8];
#pragma unroll
          for (int c = 0; c < 8; ++c) mv[c] = vv[d][c];
          wht_fwd(mv);
#pragma unroll
          for (int m = 0; m < 8; ++m) g[d][m] = fma(T(k.dm[m]), mv[m], g[d][m]);
        }
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) wht_bwd(g[d]);
#pragma unroll
      for (int c = 0; c < 8; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          T val = g[d][c];
          if (!CONSISTENT) val = fma(T(k.mL), vv[d][c], val);  // lumped mass (apply: x; force: v)
          if (MODE == 1) val -= T(k.body[d]);
          out[c][d] = val;
        }
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) out[c][d] = T(0);
    }
#pragma unroll
    for (int c = 0; c < 8; ++c)
#pragma unroll
      for (int d = 0; d < 3; ++d) ys[(c * 3 + d) * NT + t] = out[c][d];
    __syncthreads();
    // ---- owned node (gi, gj): element columns (ci,cj) (node is its corner i=1,j=1),
    // (ci+1,cj) (i=0,j=1), (ci,cj+1) (i=1,j=0), (ci+1,cj+1) (i=0,j=0)
    if (own) {
      const int tA = ci + cj * BX, tB = tA + 1, tC = tA + BX, tD = tA + BX + 1;
      if (ek >= k0) {
        const int s = (ci + 1) + (cj + 1) * SX;
        const int32_t packed = es[buf * NS + s];
        const uint32_t mask = static_cast<uint32_t>(packed) >> 29;
        const int32_t base = packed & 0x1FFFFFFF;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          T val = acc[d];
          val += ys[(3 * 3 + d) * NT + tA];
          val += ys[(2 * 3 + d) * NT + tB];
          val += ys[(1 * 3 + d) * NT + tC];
          val += ys[(0 * 3 + d) * NT + tD];
          if ((mask >> d) & 1u) {
            const int32_t q = base + __popc(mask & ((1u << d) - 1u));
            if (a.nm1) val += T(a.c1 * a.nm1[q]) * xs[((buf * NV + 0) * 3 + d) * NS + s];
            if (a.nm2) val += T(a.c2 * a.nm2[q]) * xs[((buf * NV + (MODE == 1 ? 1 : 0)) * 3 + d) * NS + s];
            a.y[q] = val;
          }
        }
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        T val = ys[(7 * 3 + d) * NT + tA];
        val += ys[(6 * 3 + d) * NT + tB];
        val += ys[(5 * 3 + d) * NT + tC];
        val += ys[(4 * 3 + d) * NT + tD];
        acc[d] = val;
      }
    }
    __syncthreads();
    buf ^= 1;
  }
}

// ------------------------------------------------------------------ launch variants
struct Variant {
  int bx, by;
};
constexpr Variant kVariants[] = {{32, 8}, {16, 16}, {32, 4}, {64, 4}, {16, 8}, {32, 16}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

template <int BX, int BY, class T, int MODE, bool CONS>
void launch_one(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  using S = Smem<BX, BY, T, MODE>;
  static bool configured = false;
  if (!configured) {
    FX_CUDA(cudaFuncSetAttribute(k_box<BX, BY, T, MODE, CONS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(S::bytes)));
    configured = true;
  }
  dim3 grid((p.nx + 1 + BX - 2) / (BX - 1), (p.ny + 1 + BY - 2) / (BY - 1), (p.nz + 1 + a.kz - 1) / a.kz);
  k_box<BX, BY, T, MODE, CONS><<<grid, BX * BY, S::bytes, st>>>(a);
  FX_LAUNCH_CHECK("box_operator");
}

template <class T, int MODE, bool CONS>
void launch_variant(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  switch (p.variant) {
    case 0: return launch_one<32, 8, T, MODE, CONS>(p, a, st);
    case 1: return launch_one<16, 16, T, MODE, CONS>(p, a, st);
    case 2: return launch_one<32, 4, T, MODE, CONS>(p, a, st);
    case 3: return launch_one<64, 4, T, MODE, CONS>(p, a, st);
    case 4: return launch_one<16, 8, T, MODE, CONS>(p, a, st);
    default: return launch_one<32, 16, T, MODE, CONS>(p, a, st);
  }
}

template <class T, int MODE>
void launch(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  if (p.consistent) launch_variant<T, MODE, true>(p, a, st);
  else launch_variant<T, MODE, false>(p, a, st);
}

// ------------------------------------------------------------------ coefficients
// Exact element operator on a box with sides h (see the file comment). J = hx hy hz / 8,
// rho_d = 2 / h_d, w(0) = 2, w(1) = 2/3 (integrals of 1 and xi^2 over [-1, 1]).
// mode 0 (apply): stiffness factor sk = cK + c0 + cc, mass factor sm = cM'.
// mode 1 (force): stiffness factor 1 on u + beta v, mass factor alphaM on v, body force.
void build_coef(ForceState& s, int mode, const double k[3]) {
  BoxPlan& p = s.box;
  const double J = p.h[0] * p.h[1] * p.h[2] / 8.0;
  const double rd[3] = {2.0 / p.h[0], 2.0 / p.h[1], 2.0 / p.h[2]};
  auto w = [](int bit) { return bit ? 2.0 / 3.0 : 2.0; };
  std::vector<BoxCoef> h(static_cast<size_t>(s.nparams));
  std::vector<BoxCoef32> h32(static_cast<size_t>(s.nparams));
  for (int32_t i = 0; i < s.nparams; ++i) {
    const ParamGP& q = s.params_h[i];
    double l2m, lam, mu;
    lame(q, l2m, lam, mu);
    double sk, sm;
    if (mode == 0) {
      const OpFactors f = op_factors(q, k[0], k[1], k[2]);
      sk = f.cK + f.c0 + f.cc;
      sm = f.cM;
    } else {
      sk = 1.0;
      sm = q.alphaM;
    }
    const bool cons = q.mass_type == 0;
    BoxCoef c{};
    for (int comp = 0; comp < 3; ++comp)
      for (int m = 0; m < 8; ++m) {
        double dk = 0.0;
        auto bit = [&](int d) { return (m >> d) & 1; };
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
        double dm = 0.0;
        if (cons) dm = sm * q.rho * J * w(bit(0)) * w(bit(1)) * w(bit(2));
        if (mode == 0) {
          c.dkm[comp][m] = (dk + dm) / 64.0;
        } else {
          c.dkm[comp][m] = dk / 64.0;
          if (comp == 0) c.dm[m] = dm / 64.0;
        }
      }
    for (int pr = 0; pr < 3; ++pr) {
      const int cc = pr, d = (pr + 1) % 3;
      for (int r = 0; r < 2; ++r) {
        const double base = 4.0 * J * rd[cc] * rd[d] * w(r) * sk / 64.0;
        c.kap[pr * 4 + r * 2 + 0] = base * lam;
        c.kap[pr * 4 + r * 2 + 1] = base * mu;
      }
    }
    c.mL = cons ? 0.0 : sm * q.rho * J;
    c.beta = mode == 1 ? q.betaK + q.betaKinit + q.betaKcomm : 0.0;
    for (int d = 0; d < 3; ++d) c.body[d] = mode == 1 ? q.b[d] * J : 0.0;
    h[i] = c;
    BoxCoef32& f = h32[i];
    for (int comp = 0; comp < 3; ++comp)
      for (int m = 0; m < 8; ++m) f.dkm[comp][m] = static_cast<float>(c.dkm[comp][m]);
    for (int j = 0; j < 12; ++j) f.kap[j] = static_cast<float>(c.kap[j]);
    for (int j = 0; j < 8; ++j) f.dm[j] = static_cast<float>(c.dm[j]);
    f.mL = static_cast<float>(c.mL);
    f.beta = static_cast<float>(c.beta);
    for (int d = 0; d < 3; ++d) f.body[d] = static_cast<float>(c.body[d]);
    f.pad_ = 0.f;
  }
  if (p.coef.n != h.size()) p.coef.alloc(h.size());
  if (p.coef32.n != h32.size()) p.coef32.alloc(h32.size());
  FX_CUDA(cudaMemcpy(p.coef.ptr, h.data(), h.size() * sizeof(BoxCoef), cudaMemcpyHostToDevice));
  FX_CUDA(cudaMemcpy(p.coef32.ptr, h32.data(), h32.size() * sizeof(BoxCoef32), cudaMemcpyHostToDevice));
  p.last_mode = mode;
  for (int j = 0; j < 3; ++j) p.last_k[j] = k[j];
}

void ensure_coef(ForceState& s, int mode, const double k[3]) {
  const BoxPlan& p = s.box;
  if (p.last_mode == mode && p.last_k[0] == k[0] && p.last_k[1] == k[1] && p.last_k[2] == k[2]) return;
  build_coef(s, mode, k);
}

}  // namespace

int box_num_variants() { return kNumVariants; }

void box_prepare(ForceState& s, const double k[3]) { ensure_coef(s, 0, k); }

void box_set_launch(ForceState& s, int variant, int kz) {
  if (variant < 0 || variant >= kNumVariants) throw Error(FX_E_INVALID, "box launch variant out of range");
  if (kz < 1) throw Error(FX_E_INVALID, "kz must be positive");
  s.box.variant = variant;
  s.box.kz = kz;
  s.box.tuned = true;
}

// ------------------------------------------------------------------ plan
void box_build_plan(ForceState& s) {
  BoxPlan& p = s.box;
  p.qualifies = false;
  auto no = [&](const std::string& why) { p.why_not = why; };
  if (s.count == 0) return no("no elements");
  bool all_cons = true, all_lumped = true;
  for (const auto& q : s.params_h) {
    if (q.kind != 0) return no("a parameter set is not elastic");
    if (q.mass_type == 0) all_lumped = false;
    else all_cons = false;
  }
  if (!all_cons && !all_lumped) return no("mixed consistent and lumped masses");
  p.consistent = all_cons;
  const int32_t N = s.N, P = s.P;
  auto X = [&](int32_t n, int d) { return s.coords_h[static_cast<size_t>(d) * N + n]; };
  // spacing from element 0
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
    packed[g] = static_cast<int32_t>((mask << 29) | static_cast<uint32_t>(base < 0 ? 0 : base));
  }
  std::vector<int32_t> eparam(static_cast<size_t>(s.count));
  for (size_t c = 0; c < cell.size(); ++c) eparam[c] = s.param_h[cell[c]];
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  for (int d = 0; d < 3; ++d) p.h[d] = h[d];
  p.node_eq.upload(packed);
  p.elem_param.upload(eparam);
  p.grid_node_h = std::move(gnode);
  p.qualifies = true;
  p.why_not.clear();
  p.last_mode = -1;
}

// ------------------------------------------------------------------ operator entry points
template <class T>
static BoxArgs<T> args(const ForceState& s, const void* coef, const T* x, const T* v, T* y) {
  BoxArgs<T> a{};
  a.nx = s.box.nx;
  a.ny = s.box.ny;
  a.nz = s.box.nz;
  a.kz = s.box.kz;
  a.node_eq = s.box.node_eq.ptr;
  a.elem_param = s.box.elem_param.ptr;
  a.coef = coef;
  a.x = x;
  a.v = v;
  a.y = y;
  return a;
}

void box_apply(ForceState& s, const double k[3], const double* x, double* y, cudaStream_t st, const int* skip) {
  ensure_coef(s, 0, k);
  BoxArgs<double> a = args<double>(s, s.box.coef.ptr, x, nullptr, y);
  a.skip = skip;
  if (k[2] != 0.0 && s.has_nodal_mass) {
    a.nm1 = s.nodal_mass.ptr;
    a.c1 = k[2];
  }
  if (k[1] != 0.0 && s.has_nodal_alpha) {
    a.nm2 = s.nodal_alpha_mass.ptr;
    a.c2 = k[1];
  }
  launch<double, 0>(s.box, a, st);
}

void box_apply_f32(ForceState& s, const double k[3], const float* x, float* y, cudaStream_t st, const int* skip) {
  ensure_coef(s, 0, k);
  BoxArgs<float> a = args<float>(s, s.box.coef32.ptr, x, nullptr, y);
  a.skip = skip;
  if (k[2] != 0.0 && s.has_nodal_mass) {
    a.nm1 = s.nodal_mass.ptr;
    a.c1 = k[2];
  }
  if (k[1] != 0.0 && s.has_nodal_alpha) {
    a.nm2 = s.nodal_alpha_mass.ptr;
    a.c2 = k[1];
  }
  launch<float, 0>(s.box, a, st);
}

void box_force(ForceState& s, const double* u, const double* v, double* f, cudaStream_t st) {
  const double k1[3] = {1.0, 0.0, 0.0};
  ensure_coef(s, 1, k1);
  BoxArgs<double> a = args<double>(s, s.box.coef.ptr, u, v, f);
  if (s.has_nodal_alpha) {
    a.nm2 = s.nodal_alpha_mass.ptr;
    a.c2 = 1.0;
  }
  launch<double, 1>(s.box, a, st);
}

void box_force_f32(ForceState& s, const float* u, const float* v, float* f, cudaStream_t st) {
  const double k1[3] = {1.0, 0.0, 0.0};
  ensure_coef(s, 1, k1);
  BoxArgs<float> a = args<float>(s, s.box.coef32.ptr, u, v, f);
  if (s.has_nodal_alpha) {
    a.nm2 = s.nodal_alpha_mass.ptr;
    a.c2 = 1.0;
  }
  launch<float, 1>(s.box, a, st);
}

// Times every launch variant and a few plane counts on the operator (FP64, coefficients of a
// unit stiffness) and keeps the fastest: CUDA events on the stream, median of 5 after 2 warm-ups.
void box_autotune(ForceState& s, cudaStream_t st) {
  if (!s.box.qualifies) return;
  DeviceArray<double> x, y;
  x.alloc(static_cast<size_t>(std::max(s.neq, 1)));
  y.alloc(static_cast<size_t>(std::max(s.neq, 1)));
  x.zero(st);
  const double k[3] = {1.0, 0.0, 0.0};
  cudaEvent_t e0, e1;
  FX_CUDA(cudaEventCreate(&e0));
  FX_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int bv = 0, bk = 16;
  const int kzs[] = {4, 8, 16, 32, 64};
  for (int v = 0; v < kNumVariants; ++v)
    for (int kz : kzs) {
      if (kz > s.box.nz + 1 && kz != 4) continue;
      s.box.variant = v;
      s.box.kz = kz;
      std::vector<float> times;
      for (int r = 0; r < 7; ++r) {
        FX_CUDA(cudaEventRecord(e0, st));
        box_apply(s, k, x.ptr, y.ptr, st);
        FX_CUDA(cudaEventRecord(e1, st));
        FX_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        FX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (r >= 2) times.push_back(ms);
      }
      std::sort(times.begin(), times.end());
      const float med = times[times.size() / 2];
      if (med < best) {
        best = med;
        bv = v;
        bk = kz;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s.box.variant = bv;
  s.box.kz = bk;
  s.box.tuned = true;
}

}  // namespace fx
