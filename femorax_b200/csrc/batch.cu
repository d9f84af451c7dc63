// Batched and served solves: many independent box-grid meshes resident on one GPU ("slots"),
// solved together. Each slot is one fx_force with its own right-hand side and solution; the
// engine solves K_eff x = b for every running slot by FP32 Jacobi-PCG inside FP64 iterative
// refinement (the FX_SOLVER_IR method of solve.cu, step for step), with
//   - one launch per operator apply for all slots: the box kernel over a work list of every
//     running slot's element tiles (k_box_batch), each slot with its own maps, coefficient
//     tables, vectors and skip flag;
//   - per-slot CG scalars and stopping flags on the device (a slot that has converged is
//     skipped by every kernel while the others continue);
//   - the inner iterations as CUDA graphs of 8 iterations over the whole batch.
//
// The vectors of all slots live in one set of engine vectors; slot s owns the entries
// [off_s, off_s + n_s), off_s a multiple of the 2048-entry reduction chunk, so a slot's chunks
// hold its own entries only. Its reductions are the documented chunk/lane order over its own
// range (the second level a warp per slot over its chunk sums), exactly as a single solve of
// the same mesh: a slot's result is bit for bit the same alone and in any mix.
//
// The engine advances in ticks (fx_engine_round): a tick corrects the slots whose inner solve has
// ended (x += d, the round's counters), gives them and newly admitted slots their outer step (FP64
// residual and test, then the inner solve's start), and runs 8 inner iterations of every slot whose
// inner solve is running; each slot's phase is held in device flags, so no slot waits for another's
// inner solve to end. Every slot performs the same operations in the same order as FX_SOLVER_IR
// on its mesh alone. Between ticks the host admits new requests into free slots and chunk ranges
// (they join at the next tick) and retires finished ones.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "force.hpp"
#include "vector.hpp"

namespace fx {
namespace {

constexpr int kWarps = 8;
static_assert(32 * kWarps == 256 && kChunkBlock == 256, "both forms of the CG kernels launch 256 threads");
constexpr int64_t kMaxSlotChunks = 2048;  // one level of chunk sums: n <= 2048 * 2048 per slot

// per-slot scalars
enum : int {
  S_RZ = 0, S_PAP, S_ALPHA, S_BETA, S_RNORM, S_TOL, S_RHS, S_RR, S_RZNEW, S_INIT,  // inner CG
  O_RR, O_BB, O_BNORM, O_RNORM, O_INIT, O_PREV,                                     // outer
  NSC = 16
};
// per-slot flags
enum : int {
  F_DONE = 0,  // inner solve finished (the FP32 apply's skip flag)
  F_CONV, F_INDEF, F_ITERS, F_MAXIT,
  G_SKIP,      // not in this round's outer step (the FP64 apply's skip flag)
  G_FIN,       // finished (converged or given up)
  G_CONV,      // converged to the FP64 tolerance
  G_OUTER, G_INNER, G_INNER_RAN,
  G_NEED_OUTER,  // due for an outer step (admitted, or corrected and not finished)
  F_BEGIN,       // its inner solve starts in this tick (set by the outer step)
  NFL = 13
};

struct SlotDev {
  int64_t off, n;  // entries
  int64_t c0, nc;  // chunks
};

__device__ __forceinline__ int slot_of_chunk(const int* chunk_slot, int64_t c) { return chunk_slot[c]; }

// a fused multiply-add in the inner solve's precision
__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }

// Called by every lane of the warp whose lane 0 has just written chunk sums of a slot: true (in
// all lanes) in the warp that counted the slot's last chunk, which then sees every chunk sum of the
// slot and resets the slot's counter for the next launch.
__device__ __forceinline__ bool slot_last(unsigned* cnt, int64_t nc, int lane) {
  unsigned t = 0;
  if (lane == 0) {
    __threadfence();
    t = atomicAdd(cnt, 1u);
  }
  t = __shfl_sync(0xffffffffu, t, 0);
  const bool last = t == static_cast<unsigned>(nc - 1);
  if (last) {
    if (lane == 0) *cnt = 0u;
    __threadfence();
  }
  return last;
}

// The second level of one slot's column j of chunk sums (k_b_level's order), by one warp, the
// chunk sums read through L2 (other warps of the launch wrote them); the sum in every lane.
__device__ __forceinline__ double slot_level(const double* part, int64_t ld, int j, const SlotDev& sd, int lanes,
                                             int lane) {
  const double* p = part + static_cast<int64_t>(j) * ld + sd.c0;
  double acc = 0.0;
  if (lane < lanes)
    for (int64_t k = lane; k < sd.nc; k += lanes) acc += __ldcg(p + k);
  double total = 0.0;
  for (int l = 0; l < lanes; ++l) total += __shfl_sync(0xffffffffu, acc, l);
  return total;
}

// second level: slot s's `ncol` columns of chunk sums (column j at part + j * nchunks) into
// sc[s * NSC + dst + j], one warp per (slot, column), for slots whose flag `gate` is 0 (inv = 0) or
// nonzero (inv = 1)
__global__ void k_b_level(const double* __restrict__ part, int64_t nchunks, int ncol, const SlotDev* __restrict__ sd,
                          const int* __restrict__ fl, int gate, int inv, int nslots, int lanes,
                          const int* __restrict__ used, double* __restrict__ sc, int dst) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= nslots * ncol) return;
  const int s = w / ncol, j = w % ncol;
  if (!used[s] || ((fl[s * NFL + gate] != 0) != (inv != 0))) return;
  const double* p = part + static_cast<int64_t>(j) * nchunks + sd[s].c0;
  const int64_t nc = sd[s].nc;
  double acc = 0.0;
  if (lane < lanes)
    for (int64_t k = lane; k < nc; k += lanes) acc += p[k];
  double total = 0.0;
  for (int l = 0; l < lanes; ++l) total += __shfl_sync(0xffffffffu, acc, l);
  if (lane == 0) sc[s * NSC + dst + j] = total;
}

// outer step: r = b - ap (FP64); chunk sums of r.r (column 0) and b.b (column 1, at part + ld)
__global__ void __launch_bounds__(32 * kWarps)
    k_b_residual(const double* __restrict__ b, const double* __restrict__ ap, double* __restrict__ r, int64_t nchunks,
                 const int* __restrict__ chunk_slot, const SlotDev* __restrict__ sd, const int* __restrict__ fl,
                 int lanes, double* __restrict__ part, int64_t ld) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = slot_of_chunk(chunk_slot, c);
  if (s < 0 || fl[s * NFL + G_SKIP]) return;
  const int64_t begin = c * kChunk;
  const int64_t end = sd[s].off + sd[s].n;
  const int64_t len = (end - begin < kChunk) ? end - begin : kChunk;
  lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<double, 2>{{b[i], ap[i]}}; },
               [&](int64_t i, const Ops<double, 2>& o) { r[i] = o.v[0] - o.v[1]; });
  __syncwarp();
  double srr = 0.0, sbb = 0.0;
  if (lane < lanes)
    lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<double, 2>{{r[i], b[i]}}; },
                 [&](int64_t, const Ops<double, 2>& o) {
                   srr = fma(o.v[0], o.v[0], srr);
                   sbb = fma(o.v[1], o.v[1], sbb);
                 });
  double trr = 0.0, tbb = 0.0;
  for (int j = 0; j < lanes; ++j) {
    trr += __shfl_sync(0xffffffffu, srr, j);
    tbb += __shfl_sync(0xffffffffu, sbb, j);
  }
  if (lane == 0) {
    part[c] = trr;
    part[ld + c] = tbb;
  }
}

// per slot: the outer test (ir: ||b - K x|| <= max(rtol ||b||, atol); given up at the limits or
// when a round did not halve ||b - K x||), then the inner solve's limits, or the end of the
// slot's solve
__global__ void k_b_outer(double* sc, int* fl, const int* used, int nslots, double rtol, double atol, int max_outer,
                          int max_it) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots || !used[s]) return;
  int* f = fl + s * NFL;
  double* c = sc + s * NSC;
  if (f[G_SKIP]) return;
  f[G_NEED_OUTER] = 0;
  if (f[G_OUTER] == 0) {
    c[O_BNORM] = sqrt(c[O_BB]);
    c[O_INIT] = sqrt(c[O_RR]);
  }
  const double rn = sqrt(c[O_RR]);
  c[O_RNORM] = rn;
  const double tol = rtol * c[O_BNORM];
  if (rn <= (tol > atol ? tol : atol)) {
    f[G_CONV] = 1;
    f[G_FIN] = 1;
  } else if (f[G_OUTER] >= max_outer || f[G_INNER] >= max_it || (f[G_OUTER] > 0 && rn > kIrStall * c[O_PREV])) {
    f[G_FIN] = 1;  // the limits, or a round that did not halve the FP64 residual
  }
  c[O_PREV] = rn;
  if (f[G_FIN]) {
    f[F_DONE] = 1;
    f[G_INNER_RAN] = 0;
    return;
  }
  f[F_DONE] = 0;
  f[F_MAXIT] = max_it - f[G_INNER];
  f[G_INNER_RAN] = 1;
  f[F_BEGIN] = 1;
}

// inner setup (TI: the inner solve's type): ri = (TI) r, d = 0; CG begin from d = 0 (K d = 0):
// rr = ri, z = inv ri, p = z; chunk sums of rr.rr (column 0) and rr.z (column 1, at part + ld)
template <class TI>
__global__ void __launch_bounds__(32 * kWarps)
    k_b_inner_begin(const double* __restrict__ r, TI* __restrict__ r32, TI* __restrict__ d,
                    TI* __restrict__ rr, TI* __restrict__ p, const TI* __restrict__ inv, int64_t nchunks,
                    const int* __restrict__ chunk_slot, const SlotDev* __restrict__ sd, const int* __restrict__ fl,
                    int lanes, double* __restrict__ part, int64_t ld) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = slot_of_chunk(chunk_slot, c);
  if (s < 0 || !fl[s * NFL + F_BEGIN]) return;
  const int64_t begin = c * kChunk;
  const int64_t end = sd[s].off + sd[s].n;
  const int64_t len = (end - begin < kChunk) ? end - begin : kChunk;
  lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<double, 1>{{r[i]}}; },
               [&](int64_t i, const Ops<double, 1>& o) {
                 r32[i] = static_cast<TI>(o.v[0]);
                 d[i] = TI(0);
               });
  __syncwarp();
  double srr = 0.0, srz = 0.0;
  if (lane < lanes)
    lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<TI, 2>{{r32[i], inv[i]}}; },
                 [&](int64_t i, const Ops<TI, 2>& o) {
                   const TI ri = fma_t(TI(-1), TI(0), o.v[0]);
                   const TI zi = o.v[1] * ri;
                   rr[i] = ri;
                   p[i] = zi;
                   srr = fma(static_cast<double>(ri), static_cast<double>(ri), srr);
                   srz = fma(static_cast<double>(ri), static_cast<double>(zi), srz);
                 });
  double trr = 0.0, trz = 0.0;
  for (int j = 0; j < lanes; ++j) {
    trr += __shfl_sync(0xffffffffu, srr, j);
    trz += __shfl_sync(0xffffffffu, srz, j);
  }
  if (lane == 0) {
    part[c] = trr;
    part[ld + c] = trz;
  }
}

__global__ void k_b_inner_start(double* sc, int* fl, const int* used, int nslots, double rtol) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots || !used[s]) return;
  int* f = fl + s * NFL;
  double* c = sc + s * NSC;
  if (!f[F_BEGIN]) return;
  f[F_BEGIN] = 0;
  c[S_RHS] = sqrt(c[S_RR]);  // b.b of the inner system: the same sum as r.r at d = 0
  const double rn = sqrt(c[S_RR]);
  c[S_RNORM] = rn;
  c[S_INIT] = rn;
  c[S_RZ] = c[S_RZNEW];
  const double tol = rtol * c[S_RHS];
  c[S_TOL] = tol > 0.0 ? tol : 0.0;
  f[F_ITERS] = 0;
  f[F_INDEF] = 0;
  f[F_CONV] = rn <= c[S_TOL];
  f[F_DONE] = f[F_CONV] || f[F_MAXIT] <= 0;
}

// The inner CG's vector kernels in two forms with the same arithmetic and sums: BLOCK, a block of
// kChunkBlock threads per chunk (every entry's loads in flight at once, the chunk's sums by one warp
// from shared memory), for batches of at most kBlockChunks chunks; otherwise a warp per chunk (8 per
// block, lane_loop). Both launch 256 threads per block.

// An inner iteration's p.ap: chunk sums of the running slots (T accumulated in double, fused
// multiply-adds, lane order), then in the warp that counts a slot's last chunk its second level
// and ConjugateGradient's alpha step (p.ap <= 0: indefinite, the inner solve ends).
template <class TI, bool BLOCK>
__global__ void __launch_bounds__(256)
    k_b_pap(const TI* __restrict__ p, const TI* __restrict__ ap, int64_t nchunks, int64_t ld,
            const int* __restrict__ chunk_slot, const SlotDev* __restrict__ sd, int* __restrict__ fl, int lanes,
            double* __restrict__ part, double* __restrict__ sc, unsigned* __restrict__ cnt) {
  int lane;
  int64_t c;
  int s;
  double total;
  if constexpr (BLOCK) {
    __shared__ TI sa[kChunk], sb[kChunk];
    c = blockIdx.x;
    s = slot_of_chunk(chunk_slot, c);
    if (s < 0 || fl[s * NFL + F_DONE]) return;
    const int64_t begin = c * kChunk;
    const int64_t end = sd[s].off + sd[s].n;
    const int len = static_cast<int>((end - begin < kChunk) ? end - begin : kChunk);
    TI va[kChunkPer], vb[kChunkPer];
#pragma unroll
    for (int k = 0; k < kChunkPer; ++k) {
      const int j = threadIdx.x + k * kChunkBlock;
      if (j < len) {
        va[k] = p[begin + j];
        vb[k] = ap[begin + j];
      }
    }
#pragma unroll
    for (int k = 0; k < kChunkPer; ++k) {
      const int j = threadIdx.x + k * kChunkBlock;
      if (j < len) {
        sa[j] = va[k];
        sb[j] = vb[k];
      }
    }
    __syncthreads();
    if (threadIdx.x >= 32) return;
    lane = threadIdx.x;
    total = chunk_fma_sum(sa, sb, len, lanes, lane);
  } else {
    lane = threadIdx.x & 31;
    c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
    if (c >= nchunks) return;
    s = slot_of_chunk(chunk_slot, c);
    if (s < 0 || fl[s * NFL + F_DONE]) return;
    const int64_t begin = c * kChunk;
    const int64_t end = sd[s].off + sd[s].n;
    const int64_t len = (end - begin < kChunk) ? end - begin : kChunk;
    double acc = 0.0;
    if (lane < lanes)
      lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<TI, 2>{{p[i], ap[i]}}; },
                   [&](int64_t, const Ops<TI, 2>& o) {
                     acc = fma(static_cast<double>(o.v[0]), static_cast<double>(o.v[1]), acc);
                   });
    total = 0.0;
    for (int j = 0; j < lanes; ++j) total += __shfl_sync(0xffffffffu, acc, j);
  }
  if (lane == 0) part[c] = total;
  if (!slot_last(cnt + s, sd[s].nc, lane)) return;
  const double pap = slot_level(part, ld, 0, sd[s], lanes, lane);
  if (lane == 0) {
    int* f = fl + s * NFL;
    double* cs = sc + s * NSC;
    cs[S_PAP] = pap;
    if (!(pap > 0.0)) {
      f[F_INDEF] = 1;
      f[F_DONE] = 1;
    } else {
      cs[S_ALPHA] = cs[S_RZ] / pap;
    }
  }
}

// d += alpha p; rr -= alpha ap; chunk sums of rr.rr and rr.z (column 1 at part + ld); then in the
// warp that counts a slot's last chunk the two second levels and the iteration's end
// (ConjugateGradient's test on ||rr||, the iteration limit, beta)
template <class TI, bool BLOCK>
__global__ void __launch_bounds__(256)
    k_b_update(double* __restrict__ sc, int* __restrict__ fl, const TI* __restrict__ p,
               const TI* __restrict__ ap, const TI* __restrict__ inv, TI* __restrict__ d,
               TI* __restrict__ rr, int64_t nchunks, const int* __restrict__ chunk_slot,
               const SlotDev* __restrict__ sd, int lanes, double* __restrict__ part, int64_t ld,
               unsigned* __restrict__ cnt) {
  int lane;
  int64_t c;
  int s;
  double trr, trz;
  if constexpr (BLOCK) {
    __shared__ TI sr[kChunk], sz[kChunk];
    c = blockIdx.x;
    s = slot_of_chunk(chunk_slot, c);
    if (s < 0 || fl[s * NFL + F_DONE]) return;
    const TI alpha = static_cast<TI>(sc[s * NSC + S_ALPHA]);
    const int64_t begin = c * kChunk;
    const int64_t end = sd[s].off + sd[s].n;
    const int len = static_cast<int>((end - begin < kChunk) ? end - begin : kChunk);
    TI vp[kChunkPer], vap[kChunkPer], vinv[kChunkPer], vd[kChunkPer], vrr[kChunkPer];
#pragma unroll
    for (int k = 0; k < kChunkPer; ++k) {
      const int j = threadIdx.x + k * kChunkBlock;
      if (j < len) {
        const int64_t i = begin + j;
        vp[k] = p[i];
        vap[k] = ap[i];
        vinv[k] = inv[i];
        vd[k] = d[i];
        vrr[k] = rr[i];
      }
    }
#pragma unroll
    for (int k = 0; k < kChunkPer; ++k) {
      const int j = threadIdx.x + k * kChunkBlock;
      if (j < len) {
        const int64_t i = begin + j;
        d[i] = fma_t(alpha, vp[k], vd[k]);
        const TI ri = fma_t(-alpha, vap[k], vrr[k]);
        rr[i] = ri;
        sr[j] = ri;
        sz[j] = vinv[k] * ri;
      }
    }
    __syncthreads();
    if (threadIdx.x >= 32) return;
    lane = threadIdx.x;
    trr = chunk_fma_sum(sr, sr, len, lanes, lane);
    trz = chunk_fma_sum(sr, sz, len, lanes, lane);
  } else {
    lane = threadIdx.x & 31;
    c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
    if (c >= nchunks) return;
    s = slot_of_chunk(chunk_slot, c);
    if (s < 0 || fl[s * NFL + F_DONE]) return;
    const TI alpha = static_cast<TI>(sc[s * NSC + S_ALPHA]);
    const int64_t begin = c * kChunk;
    const int64_t end = sd[s].off + sd[s].n;
    const int64_t len = (end - begin < kChunk) ? end - begin : kChunk;
    double srr = 0.0, srz = 0.0;
    if (lane < lanes)
      lane_loop<4>(begin, len, lane, lanes,
                   [&](int64_t i) { return Ops<TI, 5>{{p[i], ap[i], inv[i], d[i], rr[i]}}; },
                   [&](int64_t i, const Ops<TI, 5>& o) {
                     d[i] = fma_t(alpha, o.v[0], o.v[3]);
                     const TI ri = fma_t(-alpha, o.v[1], o.v[4]);
                     rr[i] = ri;
                     const TI zi = o.v[2] * ri;
                     srr = fma(static_cast<double>(ri), static_cast<double>(ri), srr);
                     srz = fma(static_cast<double>(ri), static_cast<double>(zi), srz);
                   });
    trr = 0.0;
    trz = 0.0;
    for (int j = 0; j < lanes; ++j) {
      trr += __shfl_sync(0xffffffffu, srr, j);
      trz += __shfl_sync(0xffffffffu, srz, j);
    }
  }
  if (lane == 0) {
    part[c] = trr;
    part[ld + c] = trz;
  }
  if (!slot_last(cnt + s, sd[s].nc, lane)) return;
  const double srr_all = slot_level(part, ld, 0, sd[s], lanes, lane);
  const double srz_all = slot_level(part, ld, 1, sd[s], lanes, lane);
  if (lane != 0) return;
  int* f = fl + s * NFL;
  double* cs = sc + s * NSC;
  cs[S_RR] = srr_all;
  cs[S_RZNEW] = srz_all;
  const double rn = sqrt(cs[S_RR]);
  cs[S_RNORM] = rn;
  const int it = ++f[F_ITERS];
  if (rn <= cs[S_TOL]) {
    f[F_CONV] = 1;
    f[F_DONE] = 1;
    return;
  }
  if (it >= f[F_MAXIT]) {
    f[F_DONE] = 1;
    return;
  }
  cs[S_BETA] = cs[S_RZNEW] / cs[S_RZ];
  cs[S_RZ] = cs[S_RZNEW];
}

// p = inv rr + beta p (the beta of a slot that finished this iteration is stale: its p is
// never read again)
template <class TI, bool BLOCK>
__global__ void __launch_bounds__(256)
    k_b_p(const double* __restrict__ sc, const int* __restrict__ fl, const TI* __restrict__ inv,
          const TI* __restrict__ rr, TI* __restrict__ p, int64_t nchunks, const int* __restrict__ chunk_slot,
          const SlotDev* __restrict__ sd) {
  if constexpr (BLOCK) {
    const int64_t c = blockIdx.x;
    const int s = slot_of_chunk(chunk_slot, c);
    if (s < 0 || fl[s * NFL + F_DONE]) return;
    const TI beta = static_cast<TI>(sc[s * NSC + S_BETA]);
    const int64_t begin = c * kChunk;
    const int64_t end = sd[s].off + sd[s].n;
    const int len = static_cast<int>((end - begin < kChunk) ? end - begin : kChunk);
    TI vp[kChunkPer], vinv[kChunkPer], vrr[kChunkPer];
#pragma unroll
    for (int k = 0; k < kChunkPer; ++k) {
      const int j = threadIdx.x + k * kChunkBlock;
      if (j < len) {
        vp[k] = p[begin + j];
        vinv[k] = inv[begin + j];
        vrr[k] = rr[begin + j];
      }
    }
#pragma unroll
    for (int k = 0; k < kChunkPer; ++k) {
      const int j = threadIdx.x + k * kChunkBlock;
      if (j < len) p[begin + j] = fma_t(beta, vp[k], vinv[k] * vrr[k]);
    }
  } else {
    const int lane = threadIdx.x & 31;
    const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
    if (c >= nchunks) return;
    const int s = slot_of_chunk(chunk_slot, c);
    if (s < 0 || fl[s * NFL + F_DONE]) return;
    const TI beta = static_cast<TI>(sc[s * NSC + S_BETA]);
    const int64_t begin = c * kChunk;
    const int64_t end = sd[s].off + sd[s].n;
    const int64_t len = (end - begin < kChunk) ? end - begin : kChunk;
    lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<TI, 3>{{p[i], inv[i], rr[i]}}; },
                 [&](int64_t i, const Ops<TI, 3>& o) { p[i] = fma_t(beta, o.v[0], o.v[1] * o.v[2]); });
  }
}

// x += (double) d for slots that ran an inner solve this round; the round's counters
template <class TI>
__global__ void __launch_bounds__(32 * kWarps)
    k_b_correct(const TI* __restrict__ d, double* __restrict__ x, int64_t nchunks,
                const int* __restrict__ chunk_slot, const SlotDev* __restrict__ sd, const int* __restrict__ fl) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = slot_of_chunk(chunk_slot, c);
  if (s < 0 || !fl[s * NFL + F_DONE] || !fl[s * NFL + G_INNER_RAN]) return;  // its inner solve has ended
  const int64_t begin = c * kChunk;
  const int64_t end = sd[s].off + sd[s].n;
  const int64_t len = (end - begin < kChunk) ? end - begin : kChunk;
  lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<double, 2>{{static_cast<double>(d[i]), x[i]}}; },
               [&](int64_t i, const Ops<double, 2>& o) { x[i] = o.v[1] + o.v[0]; });
}

__global__ void k_b_round_end(int* fl, const int* used, int nslots) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots || !used[s]) return;
  int* f = fl + s * NFL;
  if (!f[F_DONE] || !f[G_INNER_RAN]) return;
  f[G_INNER] += f[F_ITERS];
  f[G_OUTER] += 1;
  if (f[F_ITERS] == 0 && !f[F_CONV]) f[G_FIN] = 1;  // the inner solve made no progress
  f[G_INNER_RAN] = 0;
  if (!f[G_FIN]) f[G_NEED_OUTER] = 1;
}

// the tick's outer step: the slots due for one (the FP64 apply's skip flag is G_SKIP)
__global__ void k_b_phase(int* fl, const int* used, int nslots) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots || !used[s]) return;
  int* f = fl + s * NFL;
  f[G_SKIP] = f[G_FIN] || !f[G_NEED_OUTER];
}

// slot set-up: inverse diagonal (FP64 and FP32), zero x
__global__ void k_b_setup(const double* __restrict__ diag, double* __restrict__ inv, float* __restrict__ inv32,
                          double* __restrict__ x, int64_t n, int* zeros) {
  int local = 0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    local += diag[i] == 0.0;
    inv[i] = 1.0 / diag[i];
    inv32[i] = static_cast<float>(1.0 / diag[i]);
    x[i] = 0.0;
  }
  if (local) atomicAdd(zeros, local);
}

unsigned chunk_grid(int64_t nchunks) { return static_cast<unsigned>(std::max<int64_t>(1, (nchunks + kWarps - 1) / kWarps)); }

}  // namespace

struct Engine {
  int device = 0;
  cudaStream_t cs = nullptr;
  int max_slots = 0;
  int64_t nchunks = 0;  // capacity in chunks
  double k[3] = {1, 0, 0};
  fx_solve_opts o{};
  double inner_rtol = 1e-4;
  int max_outer = 50;
  // vectors over the capacity
  DeviceArray<double> b, x, r, ap, inv;
  DeviceArray<float> r32, d32, rr32, p32, ap32, inv32;
  // FP64 inner solves (fx_engine_set_precision): the inner vectors in double, the preconditioner
  // inv, the operator's FP64 form on p64 -> ap64
  bool inner64 = false;
  DeviceArray<double> r64, d64, rr64, p64, ap64;
  DeviceArray<int> chunk_slot;
  DeviceArray<double> part;  // [2][nchunks]
  DeviceArray<double> sc;
  DeviceArray<int> fl, used_dev, zeros;
  DeviceArray<unsigned> cnt;  // per slot: chunks counted by the fused reductions (0 between launches)
  DeviceArray<SlotDev> sd_dev;
  DeviceArray<unsigned char> inst64, inst32;  // descriptors per slot
  DeviceArray<unsigned char> inst64i;         // FP64 inner solves: the inner apply's descriptors
  DeviceArray<int4> work;
  int nwork = 0;
  DeviceArray<int> queue;  // [next item, CTAs done] of the persistent batched apply, zero between launches
  // The batched apply as one CTA per work item (the default: 0.480-0.485 s against 0.501 s for the
  // persistent wave on 120 static solves with FP32 inner solves, equal with FP64 ones, B200) or as a
  // persistent wave of CTAs taking the items from `queue`.
  bool persistent = false;
  // host state
  struct Slot {
    bool used = false;
    fx_force* f = nullptr;
    int64_t c0 = 0, nc = 0, n = 0;
  };
  std::vector<Slot> slots;
  std::vector<int> chunk_slot_h;
  std::vector<int> used_h;
  int* fl_h = nullptr;      // pinned [max_slots * NFL]
  double* sc_h = nullptr;   // pinned [max_slots * NSC]
  size_t a64 = 0, a32 = 0;  // descriptor sizes
  int64_t high = 0;         // chunks in use up to here
  bool dirty = true;        // the work list / slot tables changed
  cudaGraphExec_t graph = nullptr;
  int64_t rounds = 0;

  ~Engine() {
    if (graph) cudaGraphExecDestroy(graph);
    if (fl_h) cudaFreeHost(fl_h);
    if (sc_h) cudaFreeHost(sc_h);
    if (cs) cudaStreamDestroy(cs);
  }

  int64_t find_range(int64_t need) const {
    int64_t run = 0;
    for (int64_t c = 0; c < nchunks; ++c) {
      run = chunk_slot_h[c] < 0 ? run + 1 : 0;
      if (run == need) return c - need + 1;
    }
    return -1;
  }

  void read_flags() {
    FX_CUDA(cudaMemcpyAsync(fl_h, fl.ptr, sizeof(int) * NFL * max_slots, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaMemcpyAsync(sc_h, sc.ptr, sizeof(double) * NSC * max_slots, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
  }

  void upload_tables() {
    if (!dirty) return;
    // chunk owners, slot table, used flags, work list of every slot that is not finished
    std::vector<SlotDev> sdh(static_cast<size_t>(max_slots), SlotDev{0, 0, 0, 0});
    high = 0;
    for (int s = 0; s < max_slots; ++s)
      if (slots[s].used) {
        sdh[s] = SlotDev{slots[s].c0 * kChunk, slots[s].n, slots[s].c0, slots[s].nc};
        high = std::max(high, slots[s].c0 + slots[s].nc);
      }
    std::vector<int4> wl;
    for (int s = 0; s < max_slots; ++s) {
      if (!slots[s].used || fl_h[s * NFL + G_FIN]) continue;
      int gx, gy, gz;
      box_batch_tiles(slots[s].f->s, gx, gy, gz);
      for (int z = 0; z < gz; ++z)
        for (int y = 0; y < gy; ++y)
          for (int xx = 0; xx < gx; ++xx) wl.push_back(make_int4(s, xx, y, z));
    }
    nwork = static_cast<int>(wl.size());
    if (work.n < wl.size()) work.alloc(std::max<size_t>(wl.size(), 1024));
    FX_CUDA(cudaMemcpyAsync(sd_dev.ptr, sdh.data(), sizeof(SlotDev) * max_slots, cudaMemcpyHostToDevice, cs));
    FX_CUDA(cudaMemcpyAsync(chunk_slot.ptr, chunk_slot_h.data(), sizeof(int) * nchunks, cudaMemcpyHostToDevice, cs));
    FX_CUDA(cudaMemcpyAsync(used_dev.ptr, used_h.data(), sizeof(int) * max_slots, cudaMemcpyHostToDevice, cs));
    if (nwork)
      FX_CUDA(cudaMemcpyAsync(work.ptr, wl.data(), sizeof(int4) * wl.size(), cudaMemcpyHostToDevice, cs));
    FX_CUDA(cudaStreamSynchronize(cs));  // the host vectors above go out of scope
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    dirty = false;
  }

  void level(int ncol, int gate, int dst, int inv = 0) {
    const int warps = max_slots * ncol;
    k_b_level<<<(warps + 7) / 8, 256, 0, cs>>>(part.ptr, nchunks, ncol, sd_dev.ptr, fl.ptr, gate, inv, max_slots, o.lanes,
                                               used_dev.ptr, sc.ptr, dst);
    FX_LAUNCH_CHECK("batch_level");
  }
  unsigned slot_grid() const { return static_cast<unsigned>((max_slots + 127) / 128); }

  template <class TI>
  void inner_iteration_t(const unsigned char* inst, TI* p, TI* ap, const TI* iv, TI* d, TI* rr) {
    box_batch_apply(sizeof(TI) == 4, inst, work.ptr, nwork, persistent ? queue.ptr : nullptr, cs);
    if (high <= kBlockChunks) {  // a block per chunk
      const unsigned gb = static_cast<unsigned>(high);
      k_b_pap<TI, true><<<gb, kChunkBlock, 0, cs>>>(p, ap, high, nchunks, chunk_slot.ptr, sd_dev.ptr, fl.ptr, o.lanes,
                                                    part.ptr, sc.ptr, cnt.ptr);
      k_b_update<TI, true><<<gb, kChunkBlock, 0, cs>>>(sc.ptr, fl.ptr, p, ap, iv, d, rr, high, chunk_slot.ptr,
                                                       sd_dev.ptr, o.lanes, part.ptr, nchunks, cnt.ptr);
      k_b_p<TI, true><<<gb, kChunkBlock, 0, cs>>>(sc.ptr, fl.ptr, iv, rr, p, high, chunk_slot.ptr, sd_dev.ptr);
    } else {  // a warp per chunk
      const unsigned g = chunk_grid(high);
      k_b_pap<TI, false><<<g, 32 * kWarps, 0, cs>>>(p, ap, high, nchunks, chunk_slot.ptr, sd_dev.ptr, fl.ptr, o.lanes,
                                                    part.ptr, sc.ptr, cnt.ptr);
      k_b_update<TI, false><<<g, 32 * kWarps, 0, cs>>>(sc.ptr, fl.ptr, p, ap, iv, d, rr, high, chunk_slot.ptr,
                                                       sd_dev.ptr, o.lanes, part.ptr, nchunks, cnt.ptr);
      k_b_p<TI, false><<<g, 32 * kWarps, 0, cs>>>(sc.ptr, fl.ptr, iv, rr, p, high, chunk_slot.ptr, sd_dev.ptr);
    }
    FX_LAUNCH_CHECK("batch_inner");
  }
  void inner_iteration() {
    if (inner64) inner_iteration_t<double>(inst64i.ptr, p64.ptr, ap64.ptr, inv.ptr, d64.ptr, rr64.ptr);
    else inner_iteration_t<float>(inst32.ptr, p32.ptr, ap32.ptr, inv32.ptr, d32.ptr, rr32.ptr);
  }

  // the inner solves in FP64 (on) or FP32 (off); only while no slot is in use
  void set_inner64(bool on) {
    for (const auto& sl : slots)
      if (sl.used) throw Error(FX_E_INVALID, "fx_engine_set_precision: slots are in use");
    if (on && !r64.ptr) {
      const size_t n = static_cast<size_t>(nchunks * kChunk);
      for (auto* v : {&r64, &d64, &rr64, &p64, &ap64}) v->alloc(n);
      inst64i.alloc(a64 * max_slots);
    }
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    inner64 = on;
    dirty = true;
  }



  // One tick (see the top of the file); returns the number of unfinished slots it saw. The host's
  // copy of the flags is read at the end of every tick, so finished() sees the tick's outcome.
  int round() {
    int running = 0;
    bool any_corr = false, any_outer = false;
    for (int s = 0; s < max_slots; ++s) {
      if (!slots[s].used || fl_h[s * NFL + G_FIN]) continue;
      ++running;
      any_corr |= fl_h[s * NFL + F_DONE] && fl_h[s * NFL + G_INNER_RAN];
      any_outer |= fl_h[s * NFL + G_NEED_OUTER] != 0;
    }
    if (!running) return 0;
    upload_tables();
    const unsigned g = chunk_grid(high);
    if (any_corr) {  // the slots whose inner solve has ended: x += d, the round's counters
      if (inner64)
        k_b_correct<double><<<g, 32 * kWarps, 0, cs>>>(d64.ptr, x.ptr, high, chunk_slot.ptr, sd_dev.ptr, fl.ptr);
      else
        k_b_correct<float><<<g, 32 * kWarps, 0, cs>>>(d32.ptr, x.ptr, high, chunk_slot.ptr, sd_dev.ptr, fl.ptr);
      k_b_round_end<<<slot_grid(), 128, 0, cs>>>(fl.ptr, used_dev.ptr, max_slots);
      FX_LAUNCH_CHECK("batch_correct");
      any_outer = true;
    }
    if (any_outer) {  // the slots due for it: r = b - K x (FP64), norms, test, the inner solve's start
      k_b_phase<<<slot_grid(), 128, 0, cs>>>(fl.ptr, used_dev.ptr, max_slots);
      box_batch_apply(false, inst64.ptr, work.ptr, nwork, persistent ? queue.ptr : nullptr, cs);
      k_b_residual<<<g, 32 * kWarps, 0, cs>>>(b.ptr, ap.ptr, r.ptr, high, chunk_slot.ptr, sd_dev.ptr, fl.ptr, o.lanes,
                                              part.ptr, nchunks);
      level(2, G_SKIP, O_RR);
      k_b_outer<<<slot_grid(), 128, 0, cs>>>(sc.ptr, fl.ptr, used_dev.ptr, max_slots, o.rtol, o.atol, max_outer,
                                             o.max_iterations);
      if (inner64)
        k_b_inner_begin<double><<<g, 32 * kWarps, 0, cs>>>(r.ptr, r64.ptr, d64.ptr, rr64.ptr, p64.ptr, inv.ptr, high,
                                                           chunk_slot.ptr, sd_dev.ptr, fl.ptr, o.lanes, part.ptr,
                                                           nchunks);
      else
        k_b_inner_begin<float><<<g, 32 * kWarps, 0, cs>>>(r.ptr, r32.ptr, d32.ptr, rr32.ptr, p32.ptr, inv32.ptr, high,
                                                          chunk_slot.ptr, sd_dev.ptr, fl.ptr, o.lanes, part.ptr,
                                                          nchunks);
      level(2, F_BEGIN, S_RR, 1);
      k_b_inner_start<<<slot_grid(), 128, 0, cs>>>(sc.ptr, fl.ptr, used_dev.ptr, max_slots, inner_rtol);
      FX_LAUNCH_CHECK("batch_outer");
    }
    // 8 inner iterations of every slot whose inner solve runs (a CUDA graph, kept until the work list changes)
    const int block = 8;
    if (!graph) {
      cudaGraph_t gr = nullptr;
      FX_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      try {
        for (int i = 0; i < block; ++i) inner_iteration();
      } catch (...) {
        cudaStreamEndCapture(cs, &gr);
        if (gr) cudaGraphDestroy(gr);
        throw;
      }
      FX_CUDA(cudaStreamEndCapture(cs, &gr));
      const cudaError_t e = cudaGraphInstantiate(&graph, gr, 0);
      cudaGraphDestroy(gr);
      FX_CUDA(e);
    }
    FX_CUDA(cudaGraphLaunch(graph, cs));
    read_flags();
    // slots that finished leave the work list
    for (int s = 0; s < max_slots; ++s)
      if (slots[s].used && fl_h[s * NFL + G_FIN]) dirty = true;
    ++rounds;
    return running;
  }

  void admit(fx_force* f, const double* b_host, int* slot_out) {
    ForceState& s = f->s;
    if (s.device != device) throw Error(FX_E_INVALID, "fx_engine_admit: the mesh lives on another device");
    if (!s.use_box()) throw Error(FX_E_UNSUPPORTED, "fx_engine_admit: the batched operator needs a box grid: " + s.box.why_not);
    const int64_t n = s.neq;
    if (n <= 0) throw Error(FX_E_INVALID, "fx_engine_admit: no equations");
    const int64_t nc = chunks_of(n);
    if (nc > kMaxSlotChunks) throw Error(FX_E_UNSUPPORTED, "fx_engine_admit: more than 2048 * 2048 equations");
    int slot = -1;
    for (int i = 0; i < max_slots; ++i)
      if (!slots[i].used) {
        slot = i;
        break;
      }
    if (slot < 0) throw Error(FX_E_NOMEM, "fx_engine_admit: no free slot");
    const int64_t c0 = find_range(nc);
    if (c0 < 0) throw Error(FX_E_NOMEM, "fx_engine_admit: no free range of " + std::to_string(nc) + " chunks");
    const int64_t off = c0 * kChunk, span = nc * kChunk;
    // zero the slot's range of every vector, then b, the inverse diagonals and x
    FX_CUDA(cudaMemsetAsync(b.ptr + off, 0, sizeof(double) * span, cs));
    FX_CUDA(cudaMemsetAsync(x.ptr + off, 0, sizeof(double) * span, cs));
    FX_CUDA(cudaMemsetAsync(r.ptr + off, 0, sizeof(double) * span, cs));
    FX_CUDA(cudaMemsetAsync(ap.ptr + off, 0, sizeof(double) * span, cs));
    FX_CUDA(cudaMemsetAsync(inv.ptr + off, 0, sizeof(double) * span, cs));
    for (float* v : {r32.ptr, d32.ptr, rr32.ptr, p32.ptr, ap32.ptr, inv32.ptr})
      FX_CUDA(cudaMemsetAsync(v + off, 0, sizeof(float) * span, cs));
    if (inner64)
      for (double* v : {r64.ptr, d64.ptr, rr64.ptr, p64.ptr, ap64.ptr})
        FX_CUDA(cudaMemsetAsync(v + off, 0, sizeof(double) * span, cs));
    FX_CUDA(cudaMemcpyAsync(b.ptr + off, b_host, sizeof(double) * n, cudaMemcpyHostToDevice, cs));
    general_diagonal(s, k, r.ptr + off, cs);  // the diagonal, in r for now
    FX_CUDA(cudaMemsetAsync(zeros.ptr, 0, sizeof(int), cs));
    k_b_setup<<<static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 4096)), 256, 0, cs>>>(
        r.ptr + off, inv.ptr + off, inv32.ptr + off, x.ptr + off, n, zeros.ptr);
    FX_LAUNCH_CHECK("batch_setup");
    int nz = 0;
    FX_CUDA(cudaMemcpyAsync(&nz, zeros.ptr, sizeof(int), cudaMemcpyDeviceToHost, cs));
    // descriptors: FP64 operator x -> ap (skipped while the slot is not in the outer step),
    // FP32 operator p32 -> ap32 (skipped once its inner solve is done)
    std::vector<unsigned char> d64(a64), d32h(a32);
    box_fill_args(s, k, false, x.ptr + off, ap.ptr + off, fl.ptr + slot * NFL + G_SKIP, d64.data());
    box_fill_args(s, k, true, p32.ptr + off, ap32.ptr + off, fl.ptr + slot * NFL + F_DONE, d32h.data());
    FX_CUDA(cudaMemcpyAsync(inst64.ptr + static_cast<size_t>(slot) * a64, d64.data(), a64, cudaMemcpyHostToDevice, cs));
    FX_CUDA(cudaMemcpyAsync(inst32.ptr + static_cast<size_t>(slot) * a32, d32h.data(), a32, cudaMemcpyHostToDevice, cs));
    std::vector<unsigned char> d64i;
    if (inner64) {  // FP64 operator p64 -> ap64 (skipped once the inner solve is done)
      d64i.resize(a64);
      box_fill_args(s, k, false, p64.ptr + off, ap64.ptr + off, fl.ptr + slot * NFL + F_DONE, d64i.data());
      FX_CUDA(cudaMemcpyAsync(inst64i.ptr + static_cast<size_t>(slot) * a64, d64i.data(), a64, cudaMemcpyHostToDevice,
                              cs));
    }
    std::vector<int> f0(NFL, 0);
    f0[F_DONE] = 1;
    f0[G_NEED_OUTER] = 1;
    std::vector<double> s0(NSC, 0.0);
    FX_CUDA(cudaMemcpyAsync(fl.ptr + slot * NFL, f0.data(), sizeof(int) * NFL, cudaMemcpyHostToDevice, cs));
    FX_CUDA(cudaMemcpyAsync(sc.ptr + slot * NSC, s0.data(), sizeof(double) * NSC, cudaMemcpyHostToDevice, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
    if (nz > 0) {
      // leave the range free again: nothing points at it
      throw Error(FX_E_INVALID, "Jacobi: " + std::to_string(nz) + " zero diagonal entries");
    }
    std::memcpy(fl_h + slot * NFL, f0.data(), sizeof(int) * NFL);
    slots[slot] = Slot{true, f, c0, nc, n};
    for (int64_t c = c0; c < c0 + nc; ++c) chunk_slot_h[c] = slot;
    used_h[slot] = 1;
    dirty = true;
    *slot_out = slot;
  }

  void retire(int slot, double* x_host, fx_solve_result* res) {
    if (slot < 0 || slot >= max_slots || !slots[slot].used) throw Error(FX_E_INVALID, "fx_engine_retire: no such slot");
    read_flags();
    const int* f = fl_h + slot * NFL;
    const double* c = sc_h + slot * NSC;
    const Slot& sl = slots[slot];
    if (x_host)
      FX_CUDA(cudaMemcpyAsync(x_host, x.ptr + sl.c0 * kChunk, sizeof(double) * sl.n, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
    if (res) {
      *res = fx_solve_result{};
      res->converged = f[G_CONV];
      res->iterations = f[G_INNER];
      res->refinements = f[G_OUTER];
      res->rhs_norm = c[O_BNORM];
      res->initial_residual = c[O_INIT];
      res->final_residual = c[O_RNORM];
      res->status = f[G_CONV] ? FX_OK : FX_E_DIVERGED;
    }
    for (int64_t cc = sl.c0; cc < sl.c0 + sl.nc; ++cc) chunk_slot_h[cc] = -1;
    slots[slot] = Slot{};
    used_h[slot] = 0;
    dirty = true;
  }
};

}  // namespace fx

struct fx_engine {
  fx::Engine e;
};

namespace {
template <class F>
int guard(F&& f) {
  try {
    f();
    return FX_OK;
  } catch (const fx::Error& e) {
    fx::set_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    fx::set_error(e.what());
    return FX_E_INVALID;
  }
}
}  // namespace

extern "C" {

int fx_engine_create(int32_t device, int64_t capacity, int32_t max_slots, fx_coeffs k, fx_solve_opts o,
                     double inner_rtol, fx_engine** out) {
  return guard([&] {
    if (!out || capacity <= 0 || max_slots <= 0) throw fx::Error(FX_E_INVALID, "fx_engine_create: bad arguments");
    if (!(inner_rtol > 0.0 && inner_rtol < 1.0)) throw fx::Error(FX_E_INVALID, "inner tolerance must be in (0, 1)");
    if (o.lanes <= 0) o.lanes = 32;
    if (o.lanes > 32) throw fx::Error(FX_E_INVALID, "lanes must be in 1..32");
    if (o.max_iterations < 0) throw fx::Error(FX_E_INVALID, "max_iterations must be >= 0");
    FX_CUDA(cudaSetDevice(device));
    auto* h = new fx_engine;
    fx::Engine& e = h->e;
    try {
      e.device = device;
      e.max_slots = max_slots;
      e.k[0] = k.stiffness;
      e.k[1] = k.damping;
      e.k[2] = k.mass;
      e.o = o;
      e.inner_rtol = inner_rtol;
      e.nchunks = fx::chunks_of(capacity);
      const size_t n = static_cast<size_t>(e.nchunks * fx::kChunk);
      FX_CUDA(cudaStreamCreateWithFlags(&e.cs, cudaStreamNonBlocking));
      for (auto* v : {&e.b, &e.x, &e.r, &e.ap, &e.inv}) v->alloc(n);
      for (auto* v : {&e.r32, &e.d32, &e.rr32, &e.p32, &e.ap32, &e.inv32}) v->alloc(n);
      e.chunk_slot.alloc(static_cast<size_t>(e.nchunks));
      e.part.alloc(static_cast<size_t>(e.nchunks) * 2);
      e.sc.alloc(static_cast<size_t>(max_slots) * fx::NSC);
      e.fl.alloc(static_cast<size_t>(max_slots) * fx::NFL);
      e.used_dev.alloc(static_cast<size_t>(max_slots));
      e.cnt.alloc(static_cast<size_t>(max_slots));
      FX_CUDA(cudaMemset(e.cnt.ptr, 0, sizeof(unsigned) * max_slots));
      e.zeros.alloc(1);
      e.sd_dev.alloc(static_cast<size_t>(max_slots));
      e.a64 = fx::box_args_bytes(false);
      e.a32 = fx::box_args_bytes(true);
      e.inst64.alloc(e.a64 * max_slots);
      e.inst32.alloc(e.a32 * max_slots);
      e.work.alloc(1024);
      e.queue.upload(std::vector<int>(2, 0));
      e.slots.assign(static_cast<size_t>(max_slots), fx::Engine::Slot{});
      e.chunk_slot_h.assign(static_cast<size_t>(e.nchunks), -1);
      e.used_h.assign(static_cast<size_t>(max_slots), 0);
      FX_CUDA(cudaMallocHost(&e.fl_h, sizeof(int) * fx::NFL * max_slots));
      FX_CUDA(cudaMallocHost(&e.sc_h, sizeof(double) * fx::NSC * max_slots));
      std::vector<int> f0(static_cast<size_t>(max_slots) * fx::NFL, 0);
      for (int s = 0; s < max_slots; ++s) f0[s * fx::NFL + fx::F_DONE] = 1;
      std::memcpy(e.fl_h, f0.data(), sizeof(int) * f0.size());
      FX_CUDA(cudaMemcpy(e.fl.ptr, f0.data(), sizeof(int) * f0.size(), cudaMemcpyHostToDevice));
      FX_CUDA(cudaMemset(e.sc.ptr, 0, sizeof(double) * fx::NSC * max_slots));
      FX_CUDA(cudaMemset(e.used_dev.ptr, 0, sizeof(int) * max_slots));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

void fx_engine_destroy(fx_engine* e) { delete e; }

int fx_engine_set_persistent(fx_engine* e, int32_t on) {
  return guard([&] {
    if (!e) throw fx::Error(FX_E_INVALID, "fx_engine_set_persistent: null handle");
    FX_CUDA(cudaSetDevice(e->e.device));
    if (e->e.graph) {  // the inner iterations' graph holds the other launch form
      cudaGraphExecDestroy(e->e.graph);
      e->e.graph = nullptr;
    }
    e->e.persistent = on != 0;
  });
}

int fx_engine_set_precision(fx_engine* e, int32_t inner) {
  return guard([&] {
    if (!e || (inner != FX_ENGINE_INNER_FP32 && inner != FX_ENGINE_INNER_FP64))
      throw fx::Error(FX_E_INVALID, "fx_engine_set_precision: bad arguments");
    FX_CUDA(cudaSetDevice(e->e.device));
    e->e.set_inner64(inner == FX_ENGINE_INNER_FP64);
  });
}

int fx_engine_admit(fx_engine* e, fx_force* f, const double* b_host, int32_t* slot) {
  return guard([&] {
    if (!e || !f || !b_host || !slot) throw fx::Error(FX_E_INVALID, "fx_engine_admit: bad arguments");
    FX_CUDA(cudaSetDevice(e->e.device));
    int s = -1;
    e->e.admit(f, b_host, &s);
    *slot = s;
  });
}

int fx_engine_round(fx_engine* e, int32_t* running) {
  return guard([&] {
    if (!e) throw fx::Error(FX_E_INVALID, "fx_engine_round: null engine");
    FX_CUDA(cudaSetDevice(e->e.device));
    const int r = e->e.round();
    if (running) *running = r;
  });
}

int fx_engine_finished(fx_engine* e, int32_t slot, int32_t* finished) {
  return guard([&] {
    if (!e || !finished || slot < 0 || slot >= e->e.max_slots) throw fx::Error(FX_E_INVALID, "fx_engine_finished: bad arguments");
    *finished = e->e.slots[slot].used && e->e.fl_h[slot * fx::NFL + fx::G_FIN];
  });
}

int fx_engine_retire(fx_engine* e, int32_t slot, double* x_host, fx_solve_result* r) {
  return guard([&] {
    if (!e) throw fx::Error(FX_E_INVALID, "fx_engine_retire: null engine");
    FX_CUDA(cudaSetDevice(e->e.device));
    e->e.retire(slot, x_host, r);
  });
}

int fx_engine_info(const fx_engine* e, int64_t* info) {
  return guard([&] {
    if (!e || !info) throw fx::Error(FX_E_INVALID, "fx_engine_info: bad arguments");
    const fx::Engine& g = e->e;
    int64_t used_chunks = 0, used_slots = 0;
    for (const auto& s : g.slots)
      if (s.used) {
        used_chunks += s.nc;
        ++used_slots;
      }
    info[0] = g.nchunks * fx::kChunk;
    info[1] = used_chunks * fx::kChunk;
    info[2] = g.max_slots;
    info[3] = used_slots;
    info[4] = g.rounds;
    info[5] = static_cast<int64_t>(g.nchunks * fx::kChunk) * (5 * 8 + 6 * 4);  // vector bytes
  });
}

}  // extern "C"
