// Box execution path: stdBrick meshes that are structured grids of equal axis-aligned boxes
// (every configuration of the structured benchmarks).
//
// Element operator. On an axis-aligned box the Jacobian is constant and diagonal, and 2x2x2 Gauss
// integrates the trilinear element's stiffness and consistent mass exactly, so the element
// operator of the reference's Gauss-point form equals, up to rounding, the exact bilinear form
// written in the Walsh-Hadamard (modal) basis of the 8 corner values (1, xi, eta, zeta, xi eta,
// ...). In that basis the mass (consistent, or lumped since H^T H = 8 I) is diagonal and the
// stiffness is diagonal plus 24 couplings.
//
// The transform is split by axis. An element column sweeps up the grid, so the 2D transform of
// the face it shares with the element above is computed once and kept in registers; the two faces'
// transforms give the element's modes with 24 butterflies; the modal operator is 24 products and
// 24 fused couplings; the result is split back into a bottom and a top face; the bottom face is
// added (in modal form) to the top face left by the element below, and one 2D inverse transform
// gives the four corner values of the face. About 165 FP64 operations per element.
//
// Scatter. Each CTA owns a (BX-1) x (BY-1) column of grid nodes over kz node planes. Per plane it
// stages the node values of the plane above (one-node halo) in shared memory, evaluates the BX x BY
// element columns around its nodes (halo columns are evaluated by both neighbouring CTAs: no
// atomics, no cross-CTA exchange), and gives each owned node the sum of the face corner values of
// its four columns in a fixed order. Every equation is written once, by its owner, in a fixed
// order: deterministic for any launch shape, and y needs no zeroing. Equations and values are
// copied into a shared-memory ring several planes ahead (cp.async), so global latency overlaps the
// element work; one barrier per plane.
#include <algorithm>
#include <cstring>
#include <cmath>

#include "force.hpp"

namespace fx {

namespace {

constexpr int kParamsInShared = 16;  // coefficient tables of up to this many parameter sets in shared memory

template <class T>
struct BoxArgs {
  int nx, ny, nz, kz;
  int nparams;
  const int32_t* __restrict__ node_eq;
  const int32_t* __restrict__ elem_param;
  const void* __restrict__ coef;  // BoxCoef or BoxCoef32
  const T* __restrict__ x;        // apply: x; force: u
  const T* __restrict__ v;        // force: v
  T* __restrict__ y;
  const double* __restrict__ nm1;  // apply: nodal mass (with c1 = k.mass) or NULL
  const double* __restrict__ nm2;  // apply: nodal alpha mass (c2 = k.damping); force: lumped alphaM masses
  double c1, c2;
  T beta;           // force: u + beta v
  const int* skip;  // when set and nonzero on the device, the launch does nothing (a finished solve)
  const T* __restrict__ escale;  // per-element E scale (sets that differ only in E), or NULL
  int* queue;       // persistent launch: [next tile, CTAs done]; NULL: one CTA per tile (the grid)
  int gx, gy, gz;   // tiles per axis (persistent launch)
};

template <class T>
struct Coef;
template <>
struct Coef<double> {
  using type = BoxCoef;
  using scaled = BoxScaled;
};
template <>
struct Coef<float> {
  using type = BoxCoef32;
  using scaled = BoxScaled32;
};

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
  static constexpr int NO = (BX - 1) * (BY - 1);  // owned nodes per plane
  // Planes are gathered D planes ahead; their equations D + 2 planes ahead; the ring holds D + 3.
  static constexpr int D = 4, NB = D + 3;
  static constexpr int NV = MODE == 1 ? 2 : 1;  // staged vectors: x, or u and v
  static constexpr size_t coef_bytes = sizeof(typename Coef<T>::type) * kParamsInShared;
  static constexpr size_t bytes =
      coef_bytes + sizeof(T) * (6 * NT + NB * NV * 3 * NS + 6 * NO) + sizeof(int32_t) * (NB * NS + 2 * NO);
};

__device__ __forceinline__ void cp_async_zfill(void* smem, const void* gmem, int bytes, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int src = valid ? bytes : 0;  // 0: the destination is filled with zeros, nothing is read
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// n values from 16-byte aligned coefficient storage, two (double) or four (float) per load
template <int N>
__device__ __forceinline__ void load_coef(const double* __restrict__ src, double* dst) {
#pragma unroll
  for (int i = 0; i < N / 2; ++i) {
    const double2 v = reinterpret_cast<const double2*>(src)[i];
    dst[2 * i] = v.x;
    dst[2 * i + 1] = v.y;
  }
}
template <int N>
__device__ __forceinline__ void load_coef(const float* __restrict__ src, float* dst) {
#pragma unroll
  for (int i = 0; i < N / 4; ++i) {
    const float4 v = reinterpret_cast<const float4*>(src)[i];
    dst[4 * i] = v.x;
    dst[4 * i + 1] = v.y;
    dst[4 * i + 2] = v.z;
    dst[4 * i + 3] = v.w;
  }
}
__device__ __forceinline__ void load_pair(const double* __restrict__ src, double& a, double& b) {
  const double2 v = *reinterpret_cast<const double2*>(src);
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void load_pair(const float* __restrict__ src, float& a, float& b) {
  const float2 v = *reinterpret_cast<const float2*>(src);
  a = v.x;
  b = v.y;
}

// The modal operator, in place on the modes t[c][m] of the three components. Unknown (c, m)
// belongs to group s = m ^ 2^c and only unknowns of one group are coupled, so each group is a
// 3 x 3 block: its diagonal, then its couplings in the order of their axis pairs (pair 0 couples
// components 0 and 1, pair 1 components 1 and 2, pair 2 components 2 and 0). Groups 1..6 hold one
// coupling: lambda between the pair's components for s = 2^e (e the pair's third axis: 4, 1, 2),
// mu for s = 2^c0 + 2^c1 (3, 6, 5); group 0 holds the three lambda couplings of r = 0, group 7
// the three mu couplings of r = 1.
// VEC: the table is in shared or global memory (16-byte loads); otherwise it is a kernel
// parameter, read value by value.
// SCALED: k is a BoxScaled table; each group's result is sc times its stiffness part plus the
// mass diagonal dmm of its modes.
template <bool VEC, bool SCALED = false, class T, class CT>
__device__ __forceinline__ void modal_apply(const CT& k, T t[3][8], T sc = T(1)) {
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    T c[4];
    if constexpr (VEC) {
      load_coef<4>(k.grp[s], c);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) c[j] = k.grp[s][j];
    }
    const T u0 = t[0][s ^ 1], u1 = t[1][s ^ 2], u2 = t[2][s ^ 4];
    T o0 = c[0] * u0, o1 = c[1] * u1, o2 = c[2] * u2;
    if (s == 0 || s == 7) {
      T k1, k2;
      if constexpr (VEC) {
        load_pair(k.more + (s == 7 ? 2 : 0), k1, k2);
      } else {
        k1 = k.more[s == 7 ? 2 : 0];
        k2 = k.more[s == 7 ? 3 : 1];
      }
      o1 = fma(c[3], u0, o1);  // pair 0
      o0 = fma(c[3], u1, o0);
      o2 = fma(k1, u1, o2);  // pair 1
      o1 = fma(k1, u2, o1);
      o0 = fma(k2, u2, o0);  // pair 2
      o2 = fma(k2, u0, o2);
    } else if (s == 4 || s == 3) {
      o1 = fma(c[3], u0, o1);
      o0 = fma(c[3], u1, o0);
    } else if (s == 1 || s == 6) {
      o2 = fma(c[3], u1, o2);
      o1 = fma(c[3], u2, o1);
    } else {
      o0 = fma(c[3], u2, o0);
      o2 = fma(c[3], u0, o2);
    }
    if constexpr (SCALED) {
      o0 = fma(sc, o0, T(k.dmm[s ^ 1]) * u0);
      o1 = fma(sc, o1, T(k.dmm[s ^ 2]) * u1);
      o2 = fma(sc, o2, T(k.dmm[s ^ 4]) * u2);
    }
    t[0][s ^ 1] = o0;
    t[1][s ^ 2] = o1;
    t[2][s ^ 4] = o2;
  }
}

// MODE 0: y = K_eff x (+ k.mass nodal masses x + k.damping nodal alphaM masses x).
// MODE 1: f = K (u + beta v) - body + la v (la: lumped alphaM masses, element and nodal).
// MINB: CTAs per SM the register budget is sized for. CACHE: keep the bottom face's transform
// in registers from the plane below (fewer operations, more registers) or transform it again
// from the staged plane (fewer registers, more resident warps).
//
// Staging ring (all copies asynchronous): in the iteration of element plane ek the CTA copies
// the equations of plane ek + D + 2 (one node per thread slot) and, from the equations it copied
// two iterations before, the node values of plane ek + D; one commit group per iteration; waiting
// for all but the newest group at the end of the iteration leaves planes up to ek + D + 1
// (equations) and ek + D - 1 (values) landed.
//
// Node values are gathered, and results stored, by (node, component) items: consecutive lanes
// take the three components of one node, so one warp instruction touches about one cache line
// per node whatever the equation numbering (the reference's RCM numbering puts neighbouring
// grid nodes hundreds of equations apart). The owners of a plane's nodes leave their sums and
// equations in shared memory; the stores run in the next iteration, after the barrier.
// Where the element coefficients come from: a table per parameter set in a.coef (shared memory
// for few sets), the layered tables *tab (a kernel parameter), or one table in a.coef scaled per
// element by a.escale (sets that differ only in E).
enum CoefMode : int { kPerSet = 0, kLayered = 1, kScaled = 2 };

// One CTA's tile (bx, by, bz) of grid a, the coefficients by CM.
template <int BX, int BY, class T, int MODE, bool CACHE, int CM>
__device__ __forceinline__ void box_tile(const BoxArgs<T>& a, const BoxTable<typename Coef<T>::type>* tab, int bx,
                                         int by, int bz) {
  using S = Smem<BX, BY, T, MODE>;
  using CT = typename Coef<T>::type;
  constexpr int NT = S::NT, SX = S::SX, NS = S::NS, NB = S::NB, NV = S::NV, D = S::D, NO = S::NO;
  static_assert(BX == 16 || BX == 32, "a row of element columns must lie within one warp");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CT* cs = reinterpret_cast<CT*>(smem_raw);
  // ys, yo and yq have two buffers, by the parity of the plane: one barrier per plane suffices
  T* ys = reinterpret_cast<T*>(smem_raw + S::coef_bytes);  // [2][3][NT]: row sums for the row below
  T* xs = ys + 6 * NT;                                      // [NB planes][NV][3][NS]: node values
  T* yo = xs + NB * NV * 3 * NS;                            // [2][3][NO]: owned nodes' sums
  int32_t* es = reinterpret_cast<int32_t*>(yo + 6 * NO);   // [NB][NS]: equations
  int32_t* yq = es + NB * NS;                               // [2][NO]: owned nodes' equations (0: none)
  if (a.skip && *a.skip) return;

  const int t = threadIdx.x;
  const int ci = t % BX, cj = t / BX;
  const int i0 = bx * (BX - 1), j0 = by * (BY - 1);
  const int k0 = bz * a.kz;
  const int k1 = min(k0 + a.kz, a.nz + 1);
  const int NXn = a.nx + 1, NYn = a.ny + 1;
  const int64_t plane_stride = static_cast<int64_t>(NXn) * NYn;
  const int ei = i0 - 1 + ci, ej = j0 - 1 + cj;
  const bool col_ok = ei >= 0 && ei < a.nx && ej >= 0 && ej < a.ny;
  const bool owner_slot = ci < BX - 1 && cj < BY - 1;
  const bool own = owner_slot && i0 + ci < NXn && j0 + cj < NYn;
  const int o_idx = ci + cj * (BX - 1);  // owned node index (owner_slot)
  const int s00 = ci + cj * SX;          // staging slot of the column's corner (0, 0)

  // coefficient tables in shared memory (few parameter sets) or read through L1
  using ST = typename Coef<T>::scaled;
  constexpr bool LAYERED = CM == kLayered;
  constexpr bool scaled = CM == kScaled;
  const bool shared_coef = !LAYERED && (scaled || a.nparams <= kParamsInShared);
  if (shared_coef) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(a.coef);
    uint32_t* dst = reinterpret_cast<uint32_t*>(cs);
    const int words = scaled ? static_cast<int>(sizeof(ST) / 4) : a.nparams * static_cast<int>(sizeof(CT) / 4);
    for (int w = t; w < words; w += NT) dst[w] = __ldg(&src[w]);
  }
  const CT* coef = shared_coef ? cs : reinterpret_cast<const CT*>(a.coef);
  const ST& stab = *reinterpret_cast<const ST*>(cs);

  // ---- this thread's fixed work items
  constexpr int SPT = (NS + NT - 1) / NT;             // node slots (equation copies)
  constexpr int IPT = (3 * NS + NT - 1) / NT;         // (slot, component) gathers
  constexpr int OPT = (3 * NO + NT - 1) / NT;         // (owned node, component) stores
  int slot_off[SPT];  // node offset within a plane; -1: outside the grid; -2: past the slots
#pragma unroll
  for (int j = 0; j < SPT; ++j) {
    const int s = t + j * NT;
    const int ni = i0 - 1 + s % SX, nj = j0 - 1 + s / SX;
    slot_off[j] = s >= NS ? -2 : (ni >= 0 && ni < NXn && nj >= 0 && nj < NYn) ? nj * NXn + ni : -1;
  }
  int gitem[IPT], oitem[OPT];  // item i = t + j NT: (i / 3) << 2 | i % 3, or -1 past the items
#pragma unroll
  for (int j = 0; j < IPT; ++j) {
    const int i = t + j * NT;
    gitem[j] = i < 3 * NS ? ((i / 3) << 2) | (i % 3) : -1;
  }
#pragma unroll
  for (int j = 0; j < OPT; ++j) {
    const int i = t + j * NT;
    oitem[j] = i < 3 * NO ? ((i / 3) << 2) | (i % 3) : -1;
  }
  // (planes above k1 are never read: nothing is copied for them)
  auto copy_equations = [&](int k) {  // plane k's equations into its ring buffer
    if (k > k1) return;
    const int b = (k - k0 + 1) % NB;
#pragma unroll
    for (int j = 0; j < SPT; ++j) {
      if (slot_off[j] == -2) continue;
      const bool valid = slot_off[j] >= 0 && k >= 0 && k <= a.nz;
      cp_async_zfill(&es[b * NS + t + j * NT], valid ? a.node_eq + k * plane_stride + slot_off[j] : a.node_eq, 4, valid);
    }
  };
  auto copy_values = [&](int k) {  // plane k's node values, from its landed equations
    if (k > k1) return;
    const int b = (k - k0 + 1) % NB;
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      if (gitem[j] < 0) continue;
      const int s = gitem[j] >> 2, d = gitem[j] & 3;
      const int32_t packed = es[b * NS + s];
      const uint32_t mask = static_cast<uint32_t>(packed) >> 29;
      const int32_t q = (packed & 0x1FFFFFFF) + __popc(mask & ((1u << d) - 1u));
      const bool free_dof = (mask >> d) & 1u;
      cp_async_zfill(&xs[((b * NV + 0) * 3 + d) * NS + s], free_dof ? a.x + q : a.x, sizeof(T), free_dof);
      if (MODE == 1)
        cp_async_zfill(&xs[((b * NV + 1) * 3 + d) * NS + s], free_dof ? a.v + q : a.v, sizeof(T), free_dof);
    }
  };
  auto store_plane = [&](int par) {  // the owned nodes' sums of a plane, with the nodal terms
    const T* yop = yo + par * 3 * NO;
    const int32_t* yqp = yq + par * NO;
#pragma unroll
    for (int j = 0; j < OPT; ++j) {
      if (oitem[j] < 0) continue;
      const int o = oitem[j] >> 2, d = oitem[j] & 3;
      const int32_t packed = yqp[o];
      const uint32_t mask = static_cast<uint32_t>(packed) >> 29;
      if (!((mask >> d) & 1u)) continue;
      const int32_t q = (packed & 0x1FFFFFFF) + __popc(mask & ((1u << d) - 1u));
      T val = yop[d * NO + o];
      if (MODE == 0) {
        if (a.nm1) val += T(a.c1 * a.nm1[q]) * a.x[q];
        if (a.nm2) val += T(a.c2 * a.nm2[q]) * a.x[q];
      } else if (a.nm2) {
        val += T(a.nm2[q]) * a.v[q];
      }
      a.y[q] = val;
    }
  };
  const int64_t col_off = static_cast<int64_t>(ej) * a.nx + ei;
  const int64_t layer = static_cast<int64_t>(a.nx) * a.ny;
  auto param_of = [&](int ek) {
    if constexpr (LAYERED) return (ek >= 0 && ek < a.nz) ? static_cast<int>(tab->layer[ek]) : -1;  // same for all threads
    return (col_ok && ek >= 0 && ek < a.nz) ? __ldg(&a.elem_param[ek * layer + col_off]) : -1;
  };
  // 2D transform of the column's face of plane buffer b (MODE 1: of u + beta v): f = p + 2q
  // (p: x mode, q: y mode), written to f[d * stride + 0..3]
  auto face = [&](int b, T* f, const int stride) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T* p = xs + ((b * NV + 0) * 3 + d) * NS + s00;
      T a00 = p[0], a10 = p[1], a01 = p[SX], a11 = p[SX + 1];
      if (MODE == 1) {
        const T* q = xs + ((b * NV + 1) * 3 + d) * NS + s00;
        a00 = fma(a.beta, q[0], a00);
        a10 = fma(a.beta, q[1], a10);
        a01 = fma(a.beta, q[SX], a01);
        a11 = fma(a.beta, q[SX + 1], a11);
      }
      const T s0 = a00 + a10, d0 = a10 - a00, s1 = a01 + a11, d1 = a11 - a01;
      f[d * stride + 0] = s0 + s1;
      f[d * stride + 1] = d0 + d1;
      f[d * stride + 2] = s1 - s0;
      f[d * stride + 3] = d1 - d0;
    }
  };

  // prologue: equations of planes k0 - 1 .. k0 + D, then values of k0 - 1 .. k0 + D - 2 (the loop's
  // first iteration continues with k0 + D + 1 and k0 + D - 1)
  for (int k = k0 - 1; k <= k0 + D; ++k) copy_equations(k);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();  // the values' copies read other threads' equations
  for (int k = k0 - 1; k <= k0 + D - 2; ++k) copy_values(k);
  cp_async_commit();
  cp_async_wait<0>();
  auto scale_of = [&](int ek) {
    if constexpr (scaled) return (col_ok && ek >= 0 && ek < a.nz) ? __ldg(&a.escale[ek * layer + col_off]) : T(0);
    return T(0);
  };
  int p_cur = param_of(k0 - 1), p_nxt = param_of(k0);
  T s_cur = scale_of(k0 - 1), s_nxt = scale_of(k0);
  __syncthreads();
  T fb[3][4], facc[3][4];
  if constexpr (CACHE) face(0, &fb[0][0], 4);
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int f = 0; f < 4; ++f) facc[d][f] = T(0);
  int bb = 0;  // buffer of plane ek; plane ek + i is in (bb + i) % NB

  int par = 0;  // buffer of ys, yo, yq for plane ek
  for (int ek = k0 - 1; ek < k1; ++ek, par ^= 1) {
    const int tb = bb + 1 == NB ? 0 : bb + 1;
    copy_equations(ek + D + 2);
    copy_values(ek + D);
    cp_async_commit();
    const int p_here = p_cur;
    p_cur = p_nxt;
    p_nxt = param_of(ek + 2);
    const T s_here = s_cur;
    s_cur = s_nxt;
    s_nxt = scale_of(ek + 2);
    const bool out_plane = own && ek >= k0;
    const int32_t own_packed = out_plane ? es[bb * NS + s00 + SX + 1] : 0;
    // ---- element (ei, ej, ek): modes from the top face (transformed here) and the bottom face
    T tv[3][8];
    face(tb, &tv[0][0], 8);  // top face into tv[.][0..3]
    if constexpr (!CACHE) face(bb, &fb[0][0], 4);
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const T top = tv[d][f], bot = fb[d][f];
        tv[d][f] = top + bot;
        tv[d][f + 4] = top - bot;
        if constexpr (CACHE) fb[d][f] = top;
      }
    T cor[3][4];  // face corner values c = i + 2j of the three components
    if (p_here >= 0 && (!LAYERED || col_ok)) {
      T body[3] = {T(0), T(0), T(0)};
      if constexpr (LAYERED) {
        modal_apply<false>(tab->c[p_here], tv);
        if (MODE == 1)
          for (int d = 0; d < 3; ++d) body[d] = T(tab->c[p_here].body[d]);
      } else if constexpr (scaled) {
        modal_apply<true, true>(stab, tv, s_here);
        if (MODE == 1)
          for (int d = 0; d < 3; ++d) body[d] = T(stab.body[d]);
      } else {
        const CT& k = coef[p_here];
        modal_apply<true>(k, tv);
        if (MODE == 1)
          for (int d = 0; d < 3; ++d) body[d] = T(k.body[d]);
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        T* g = tv[d];
        if (MODE == 1) g[0] -= body[d];
        T h[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          h[f] = facc[d][f] + (g[f] - g[f + 4]);  // bottom face, plus the element below's top face
          facc[d][f] = g[f] + g[f + 4];            // top face, for the plane above
        }
        // inverse 2D transform of the face
        const T u0 = h[0] - h[2], u2 = h[0] + h[2], u1 = h[1] - h[3], u3 = h[1] + h[3];
        cor[d][0] = u0 - u1;
        cor[d][1] = u0 + u1;
        cor[d][2] = u2 - u3;
        cor[d][3] = u2 + u3;
      }
    } else {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const T u0 = facc[d][0] - facc[d][2], u2 = facc[d][0] + facc[d][2];
        const T u1 = facc[d][1] - facc[d][3], u3 = facc[d][1] + facc[d][3];
        cor[d][0] = u0 - u1;
        cor[d][1] = u0 + u1;
        cor[d][2] = u2 - u3;
        cor[d][3] = u2 + u3;
#pragma unroll
        for (int f = 0; f < 4; ++f) facc[d][f] = T(0);
      }
    }
    // The owned node (ci, cj) of plane ek is corner (1,1) of column (ci, cj), corner (0,1) of
    // (ci+1, cj), corner (1,0) of (ci, cj+1) and corner (0,0) of (ci+1, cj+1); its value is the
    // sum of its row's pair plus the pair of the row above, in that order. Column ci+1 of the same
    // row is the next lane (a row of columns lies within one warp), so its corners come by
    // shuffle; the pair sums for the row below go through shared memory.
    T phi[3];
    T* ysp = ys + par * 3 * NT;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T c01n = __shfl_down_sync(0xffffffffu, cor[d][2], 1);
      const T c00n = __shfl_down_sync(0xffffffffu, cor[d][0], 1);
      phi[d] = cor[d][3] + c01n;
      ysp[d * NT + t] = cor[d][1] + c00n;
    }
    // The one barrier of the plane: this plane's pair sums, the last plane's owned sums and the
    // staging ring's copies up to the planes the next iteration reads are all in place after it.
    cp_async_wait<1>();
    __syncthreads();
    if (ek - 1 >= k0) store_plane(par ^ 1);  // plane ek - 1
    if (owner_slot) {
      if (out_plane) {
#pragma unroll
        for (int d = 0; d < 3; ++d) yo[(par * 3 + d) * NO + o_idx] = phi[d] + ysp[d * NT + t + BX];
      }
      yq[par * NO + o_idx] = own_packed;
    }
    bb = tb;
  }
  cp_async_wait<0>();
  __syncthreads();
  if (k1 - 1 >= k0) store_plane(par ^ 1);  // the last plane (par has advanced past it)
}

template <int BX, int BY, class T, int MODE, int MINB, bool CACHE, int CM>
__global__ void __launch_bounds__(BX* BY, MINB)
    k_box(BoxArgs<T> a, const __grid_constant__ BoxTable<typename Coef<T>::type> tab) {
  if (!a.queue) {
    box_tile<BX, BY, T, MODE, CACHE, CM>(a, &tab, blockIdx.x, blockIdx.y, blockIdx.z);
    return;
  }
  // Persistent launch (one wave of CTAs): each CTA takes the next tile (x fastest) from the queue
  // until none is left, so the last wave of a one-CTA-per-tile grid leaves no SM idle. The last
  // CTA to finish resets the queue for the next launch (every CTA has stopped taking tiles then).
  __shared__ int s_tile;
  const int ntiles = a.gx * a.gy * a.gz;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&a.queue[0], 1);
    __syncthreads();
    const int tile = s_tile;
    __syncthreads();
    if (tile >= ntiles) break;
    box_tile<BX, BY, T, MODE, CACHE, CM>(a, &tab, tile % a.gx, (tile / a.gx) % a.gy, tile / (a.gx * a.gy));
    __syncthreads();
  }
  if (threadIdx.x == 0 && atomicAdd(&a.queue[1], 1) == static_cast<int>(gridDim.x) - 1) {
    a.queue[0] = 0;
    a.queue[1] = 0;
  }
}

// Many grids in one launch: CTA b takes work item work[b] = (grid, tile x, tile y, tile z) of the
// grids inst[] describes (each with its own maps, tables, vectors and skip flag).
template <int BX, int BY, class T, int MODE, int MINB>
__global__ void __launch_bounds__(BX* BY, MINB)
    k_box_batch(const BoxArgs<T>* __restrict__ inst, const int4* __restrict__ work) {
  const int4 w = work[blockIdx.x];
  const BoxArgs<T> a = inst[w.x];
  box_tile<BX, BY, T, MODE, false, kPerSet>(a, nullptr, w.y, w.z, w.w);
}

// ------------------------------------------------------------------ launch variants
// (BX, BY, CTAs per SM for the register budget, face caching)
constexpr int kNumVariants = 9;  // see launch()

template <class T>
const BoxTable<typename Coef<T>::type>& table_of(const BoxPlan& p, int mode);
template <>
const BoxTable<BoxCoef>& table_of<double>(const BoxPlan& p, int mode) {
  return p.cset[mode].tab;
}
template <>
const BoxTable<BoxCoef32>& table_of<float>(const BoxPlan& p, int mode) {
  return p.cset[mode].tab32;
}

template <int BX, int BY, int MINB, bool CACHE, int CM, class T, int MODE>
void launch_shape(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  using S = Smem<BX, BY, T, MODE>;
  auto kern = k_box<BX, BY, T, MODE, MINB, CACHE, CM>;
  static int resident = 0;  // CTAs per SM at this shape's registers and shared memory
  if (!resident) {
    FX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::bytes)));
    FX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, BX * BY, S::bytes));
    resident = std::max(resident, 1);
  }
  dim3 grid((p.nx + 1 + BX - 2) / (BX - 1), (p.ny + 1 + BY - 2) / (BY - 1), (p.nz + 1 + a.kz - 1) / a.kz);
  if (p.shape[sizeof(T) == 4 ? 1 : 0].persistent) {
    BoxArgs<T> b = a;
    b.queue = p.queue.ptr;
    b.gx = static_cast<int>(grid.x);
    b.gy = static_cast<int>(grid.y);
    b.gz = static_cast<int>(grid.z);
    const int ntiles = b.gx * b.gy * b.gz;
    const int ctas = std::min(ntiles, resident * num_sms());
    kern<<<ctas, BX * BY, S::bytes, st>>>(b, table_of<T>(p, MODE));
  } else {
    kern<<<grid, BX * BY, S::bytes, st>>>(a, table_of<T>(p, MODE));
  }
  FX_LAUNCH_CHECK("box_operator");
}

template <int BX, int BY, int MINB, bool CACHE, class T, int MODE>
void launch_one(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  if (p.layered) return launch_shape<BX, BY, MINB, CACHE, kLayered, T, MODE>(p, a, st);
  if (p.scaled) return launch_shape<BX, BY, MINB, CACHE, kScaled, T, MODE>(p, a, st);
  return launch_shape<BX, BY, MINB, CACHE, kPerSet, T, MODE>(p, a, st);
}

template <class T, int MODE>
void launch(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  switch (p.shape[sizeof(T) == 4 ? 1 : 0].variant) {
    case 0: return launch_one<32, 8, 2, false, T, MODE>(p, a, st);
    case 1: return launch_one<16, 16, 2, false, T, MODE>(p, a, st);
    case 2: return launch_one<16, 8, 4, false, T, MODE>(p, a, st);
    case 3: return launch_one<32, 16, 1, false, T, MODE>(p, a, st);
    case 4: return launch_one<16, 8, 2, true, T, MODE>(p, a, st);
    case 5: return launch_one<16, 8, 5, false, T, MODE>(p, a, st);
    case 6: return launch_one<16, 8, 6, false, T, MODE>(p, a, st);
    case 7: return launch_one<32, 4, 4, false, T, MODE>(p, a, st);
    default: return launch_one<16, 32, 1, false, T, MODE>(p, a, st);
  }
}

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
    if (mode == 0) {
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
  for (auto& sh : s.box.shape) {
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
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  for (int d = 0; d < 3; ++d) p.h[d] = h[d];
  p.node_eq.upload(packed);
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
  a.nx = s.box.nx;
  a.ny = s.box.ny;
  a.nz = s.box.nz;
  a.kz = s.box.shape[sizeof(T) == 4 ? 1 : 0].kz;
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
// (unit stiffness) in FP64 and in FP32 and keeps the fastest of each: CUDA events on the stream,
// L2 flushed before each apply, median of 5 after 2 warm-ups.
void box_autotune(ForceState& s, cudaStream_t st) {
  if (!s.box.qualifies) return;
  if (s.count < kTuneMinElements) {  // launch-bound: timing costs more than it can save
    for (auto& sh : s.box.shape) sh = BoxPlan::Shape{};
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
  const int kzs[] = {8, 16, 32, 64};  // (kz = 4 adds a quarter of redundant planes)
  for (int prec = 0; prec < 2; ++prec) {
    BoxPlan::Shape& sh = s.box.shape[prec];
    BoxPlan::Shape best_shape;
    float best = 1e30f;
    for (int v = 0; v < kNumVariants; ++v)
      for (int kz : kzs)
        for (int pers = 0; pers < 2; ++pers) {
          if (kz > 8 && kz >= 2 * (s.box.nz + 1)) continue;
          sh = BoxPlan::Shape{v, kz, pers != 0};
          std::vector<float> times;
          for (int r = 0; r < 7; ++r) {
            FX_CUDA(cudaMemsetAsync(flush.ptr, r, flush.n, st));
            FX_CUDA(cudaEventRecord(e0, st));
            if (prec == 0) box_apply(s, k, x.ptr, y.ptr, st, nullptr);
            else box_apply_f32(s, k, x32.ptr, y32.ptr, st, nullptr);
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
void batch_launch(const void* inst, const int4* work, int nwork, cudaStream_t st) {
  using S = Smem<kBatchBX, kBatchBY, T, 0>;
  static bool configured = false;
  if (!configured) {
    FX_CUDA(cudaFuncSetAttribute(k_box_batch<kBatchBX, kBatchBY, T, 0, kBatchMinB<T>>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::bytes)));
    configured = true;
  }
  k_box_batch<kBatchBX, kBatchBY, T, 0, kBatchMinB<T>>
      <<<nwork, kBatchBX * kBatchBY, S::bytes, st>>>(static_cast<const BoxArgs<T>*>(inst), work);
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

void box_batch_apply(bool f32, const void* inst, const int4* work, int nwork, cudaStream_t st) {
  if (nwork <= 0) return;
  if (f32) batch_launch<float>(inst, work, nwork, st);
  else batch_launch<double>(inst, work, nwork, st);
}

}  // namespace fx
