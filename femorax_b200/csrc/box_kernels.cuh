// Box execution path, device side: the kernels for stdBrick meshes that are structured grids of
// equal axis-aligned boxes, their launch shapes, and launch<T, MODE>, which box_f64_apply.cu,
// box_f64_force.cu, box_f32_apply.cu and box_f32_force.cu instantiate (one translation unit each,
// compiled in parallel).
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
#pragma once

#include <algorithm>

#include "force.hpp"

namespace fx {
namespace boxk {

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
  const int* tiles;  // tile-list launch: CTA b takes tile tiles[b] (x fastest); NULL: the grid
  int ntiles;        // (host side) the list's length
  int gx, gy, gz;   // tiles per axis (persistent and tile-list launches)
  int cset;         // (host side) the coefficient set whose tables the launch passes
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

// Where the element coefficients come from: a table per parameter set in a.coef (shared memory
// for few sets), the layered tables *tab (a kernel parameter), or one table in a.coef scaled per
// element by a.escale (sets that differ only in E).
enum CoefMode : int { kPerSet = 0, kLayered = 1, kScaled = 2 };

template <int BX, int BY, class T, int MODE, int CM>
struct Smem {
  static constexpr int NT = BX * BY, SX = BX + 1, SY = BY + 1, NS = SX * SY;
  static constexpr int NO = (BX - 1) * (BY - 1);  // owned nodes per plane
  // Planes are gathered D planes ahead; their equations D + 2 planes ahead; the ring holds D + 3.
  static constexpr int D = 4, NB = D + 3;
  static constexpr int NV = MODE == 1 ? 2 : 1;  // staged vectors: x, or u and v
  // coefficient tables in shared memory: none for layered grids (kernel parameter), one scaled
  // table, or up to kParamsInShared per-set tables
  static constexpr size_t coef_bytes =
      CM == kLayered ? 0
      : CM == kScaled ? (sizeof(typename Coef<T>::scaled) + 15) / 16 * 16
                      : sizeof(typename Coef<T>::type) * kParamsInShared;
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
// MODE 2: MODE 1's force from w = u + beta v formed beforehand (x = w, v read by the owners for
// la v only): one staged vector, as the apply.
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
// FULL: every grid node has all three DOFs free or none (mask 7 or 0; the plan checks it): the
// packed word of a free node is negative and its equations are base + d, so a (node, component)
// item needs no mask arithmetic.
// One CTA's tile (bx, by, bz) of grid a, the coefficients by CM.
template <int BX, int BY, class T, int MODE, bool CACHE, int CM, bool FULL>
__device__ __forceinline__ void box_tile(const BoxArgs<T>& a, const BoxTable<typename Coef<T>::type>* tab, int bx,
                                         int by, int bz) {
  using S = Smem<BX, BY, T, MODE, CM>;
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
  // plane k of buffer b = (k - k0 + 1) mod NB: the loop steps the buffers with the planes
  auto copy_equations = [&](int k, int b) {  // plane k's equations into its ring buffer
    if (k > k1) return;
#pragma unroll
    for (int j = 0; j < SPT; ++j) {
      if (slot_off[j] == -2) continue;
      const bool valid = slot_off[j] >= 0 && k >= 0 && k <= a.nz;
      cp_async_zfill(&es[b * NS + t + j * NT], valid ? a.node_eq + k * plane_stride + slot_off[j] : a.node_eq, 4, valid);
    }
  };
  auto copy_values = [&](int k, int b) {  // plane k's node values, from its landed equations
    if (k > k1) return;
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
      if (gitem[j] < 0) continue;
      const int s = gitem[j] >> 2, d = gitem[j] & 3;
      const int32_t packed = es[b * NS + s];
      int32_t q;
      bool free_dof;
      if constexpr (FULL) {
        free_dof = packed < 0;
        q = (packed & 0x1FFFFFFF) + d;
      } else {
        const uint32_t mask = static_cast<uint32_t>(packed) >> 29;
        q = (packed & 0x1FFFFFFF) + __popc(mask & ((1u << d) - 1u));
        free_dof = (mask >> d) & 1u;
      }
      // FULL: a fixed or outside node's word is 0, so q = d < 3 <= neq is in bounds (and nothing
      // is read: the copy size is 0); otherwise the address of a fixed DOF is replaced by x
      const int32_t qa = FULL || free_dof ? q : 0;
      cp_async_zfill(&xs[((b * NV + 0) * 3 + d) * NS + s], a.x + qa, sizeof(T), free_dof);
      if (MODE == 1) cp_async_zfill(&xs[((b * NV + 1) * 3 + d) * NS + s], a.v + qa, sizeof(T), free_dof);
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
      int32_t q;
      if constexpr (FULL) {
        if (packed >= 0) continue;
        q = (packed & 0x1FFFFFFF) + d;
      } else {
        const uint32_t mask = static_cast<uint32_t>(packed) >> 29;
        if (!((mask >> d) & 1u)) continue;
        q = (packed & 0x1FFFFFFF) + __popc(mask & ((1u << d) - 1u));
      }
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
  for (int k = k0 - 1; k <= k0 + D; ++k) copy_equations(k, k - k0 + 1);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();  // the values' copies read other threads' equations
  for (int k = k0 - 1; k <= k0 + D - 2; ++k) copy_values(k, k - k0 + 1);
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
  int bb = 0;           // buffer of plane ek; plane ek + i is in (bb + i) mod NB
  int be = D + 2, bv = D;  // buffers of planes ek + D + 2 (equations) and ek + D (values)

  int par = 0;  // buffer of ys, yo, yq for plane ek
  for (int ek = k0 - 1; ek < k1; ++ek, par ^= 1) {
    const int tb = bb + 1 == NB ? 0 : bb + 1;
    copy_equations(ek + D + 2, be);
    copy_values(ek + D, bv);
    be = be + 1 == NB ? 0 : be + 1;
    bv = bv + 1 == NB ? 0 : bv + 1;
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
        if (MODE >= 1)
          for (int d = 0; d < 3; ++d) body[d] = T(tab->c[p_here].body[d]);
      } else if constexpr (scaled) {
        modal_apply<true, true>(stab, tv, s_here);
        if (MODE >= 1)
          for (int d = 0; d < 3; ++d) body[d] = T(stab.body[d]);
      } else {
        const CT& k = coef[p_here];
        modal_apply<true>(k, tv);
        if (MODE >= 1)
          for (int d = 0; d < 3; ++d) body[d] = T(k.body[d]);
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        T* g = tv[d];
        if (MODE >= 1) g[0] -= body[d];
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

template <int BX, int BY, class T, int MODE, int MINB, bool CACHE, int CM, bool FULL>
__global__ void __launch_bounds__(BX* BY, MINB)
    k_box(BoxArgs<T> a, const __grid_constant__ BoxTable<typename Coef<T>::type> tab) {
  if (a.tiles) {  // a part of the grid's tiles, in the list's order
    const int tile = a.tiles[blockIdx.x];
    box_tile<BX, BY, T, MODE, CACHE, CM, FULL>(a, &tab, tile % a.gx, (tile / a.gx) % a.gy, tile / (a.gx * a.gy));
    return;
  }
  if (!a.queue) {
    box_tile<BX, BY, T, MODE, CACHE, CM, FULL>(a, &tab, blockIdx.x, blockIdx.y, blockIdx.z);
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
    box_tile<BX, BY, T, MODE, CACHE, CM, FULL>(a, &tab, tile % a.gx, (tile / a.gx) % a.gy, tile / (a.gx * a.gy));
    __syncthreads();
  }
  if (threadIdx.x == 0 && atomicAdd(&a.queue[1], 1) == static_cast<int>(gridDim.x) - 1) {
    a.queue[0] = 0;
    a.queue[1] = 0;
  }
}

// Many grids in one launch: work items work[i] = (grid, tile x, tile y, tile z) of the grids inst[]
// describes (each with its own maps, tables, vectors and skip flag). With queue == NULL, CTA b takes
// item b (one CTA per item); otherwise a persistent wave of CTAs takes the items in list order from
// the counter queue[0] until none is left, and the last CTA to finish resets queue[0..1] for the
// next launch (every CTA has stopped taking items then), as k_box's persistent form.
template <int BX, int BY, class T, int MODE, int MINB>
__global__ void __launch_bounds__(BX* BY, MINB)
    k_box_batch(const BoxArgs<T>* __restrict__ inst, const int4* __restrict__ work, int nwork, int* queue) {
  if (!queue) {
    const int4 w = work[blockIdx.x];
    const BoxArgs<T> a = inst[w.x];
    box_tile<BX, BY, T, MODE, false, kPerSet, false>(a, nullptr, w.y, w.z, w.w);
    return;
  }
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&queue[0], 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= nwork) break;
    const int4 w = work[item];
    const BoxArgs<T> a = inst[w.x];
    box_tile<BX, BY, T, MODE, false, kPerSet, false>(a, nullptr, w.y, w.z, w.w);
    __syncthreads();
  }
  if (threadIdx.x == 0 && atomicAdd(&queue[1], 1) == static_cast<int>(gridDim.x) - 1) {
    queue[0] = 0;
    queue[1] = 0;
  }
}

// ------------------------------------------------------------------ launch variants
// (BX, BY, CTAs per SM for the register budget, face caching)
constexpr int kNumVariants = 11;  // see launch()
// the block of element columns (BX, BY) of each variant, for the host's tile geometry
constexpr int kVariantBlock[kNumVariants][2] = {{32, 8}, {16, 16}, {16, 8}, {32, 16}, {16, 8}, {16, 8},
                                                {16, 8}, {32, 4},  {16, 32}, {16, 8}, {16, 8}};

template <class T>
const BoxTable<typename Coef<T>::type>& table_of(const BoxPlan& p, int mode);
template <>
inline const BoxTable<BoxCoef>& table_of<double>(const BoxPlan& p, int mode) {
  return p.cset[mode].tab;
}
template <>
inline const BoxTable<BoxCoef32>& table_of<float>(const BoxPlan& p, int mode) {
  return p.cset[mode].tab32;
}

template <int BX, int BY, int MINB, bool CACHE, int CM, bool FULL, class T, int MODE>
void launch_kernel(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  using S = Smem<BX, BY, T, MODE, CM>;
  auto kern = k_box<BX, BY, T, MODE, MINB, CACHE, CM, FULL>;
  // CTAs per SM at this shape's registers and shared memory (set once, thread-safe)
  static const int resident = [&] {
    int dev = 0, max_smem = 0, r = 0;
    FX_CUDA(cudaGetDevice(&dev));
    FX_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (S::bytes > static_cast<size_t>(max_smem))
      throw Error(FX_E_UNSUPPORTED, "box launch shape: its staging needs more shared memory than a CTA can have");
    FX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::bytes)));
    FX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, kern, BX * BY, S::bytes));
    return std::max(r, 1);
  }();
  dim3 grid((p.nx + 1 + BX - 2) / (BX - 1), (p.ny + 1 + BY - 2) / (BY - 1), (p.nz + 1 + a.kz - 1) / a.kz);
  if (a.tiles) {
    BoxArgs<T> b = a;
    b.queue = nullptr;
    b.gx = static_cast<int>(grid.x);
    b.gy = static_cast<int>(grid.y);
    b.gz = static_cast<int>(grid.z);
    if (a.ntiles > 0) kern<<<a.ntiles, BX * BY, S::bytes, st>>>(b, table_of<T>(p, a.cset));
  } else if (p.shape[sizeof(T) == 4 ? 1 : 0][MODE == 1 ? 1 : 0].persistent) {
    BoxArgs<T> b = a;
    b.queue = p.queue.ptr;
    b.gx = static_cast<int>(grid.x);
    b.gy = static_cast<int>(grid.y);
    b.gz = static_cast<int>(grid.z);
    const int ntiles = b.gx * b.gy * b.gz;
    const int ctas = std::min(ntiles, resident * num_sms());
    kern<<<ctas, BX * BY, S::bytes, st>>>(b, table_of<T>(p, a.cset));
  } else {
    kern<<<grid, BX * BY, S::bytes, st>>>(a, table_of<T>(p, a.cset));
  }
  FX_LAUNCH_CHECK("box_operator");
}

template <int BX, int BY, int MINB, bool CACHE, int CM, class T, int MODE>
void launch_shape(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  if (p.full) launch_kernel<BX, BY, MINB, CACHE, CM, true, T, MODE>(p, a, st);
  else launch_kernel<BX, BY, MINB, CACHE, CM, false, T, MODE>(p, a, st);
}

template <int BX, int BY, int MINB, bool CACHE, class T, int MODE>
void launch_one(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  if (p.layered) return launch_shape<BX, BY, MINB, CACHE, kLayered, T, MODE>(p, a, st);
  if (p.scaled) return launch_shape<BX, BY, MINB, CACHE, kScaled, T, MODE>(p, a, st);
  return launch_shape<BX, BY, MINB, CACHE, kPerSet, T, MODE>(p, a, st);
}

template <class T, int MODE>
void launch(const BoxPlan& p, const BoxArgs<T>& a, cudaStream_t st) {
  // (MODE 2 stages one vector, as the apply: the apply's shape)
  switch (p.shape[sizeof(T) == 4 ? 1 : 0][MODE == 1 ? 1 : 0].variant) {
    case 0: return launch_one<32, 8, 2, false, T, MODE>(p, a, st);
    case 1: return launch_one<16, 16, 2, false, T, MODE>(p, a, st);
    case 2: return launch_one<16, 8, 4, false, T, MODE>(p, a, st);
    case 3: return launch_one<32, 16, 1, false, T, MODE>(p, a, st);
    case 4: return launch_one<16, 8, 2, true, T, MODE>(p, a, st);
    case 5: return launch_one<16, 8, 5, false, T, MODE>(p, a, st);
    case 6: return launch_one<16, 8, 6, false, T, MODE>(p, a, st);
    case 7: return launch_one<32, 4, 4, false, T, MODE>(p, a, st);
    case 8: return launch_one<16, 32, 1, false, T, MODE>(p, a, st);
    case 9: return launch_one<16, 8, 3, true, T, MODE>(p, a, st);
    default: return launch_one<16, 8, 4, true, T, MODE>(p, a, st);
  }
}

}  // namespace boxk
}  // namespace fx
