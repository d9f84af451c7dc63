// Batched quasi-static Newton on many independent meshes (the batched J2 configuration): the
// meshes are concatenated into one mesh whose element kernels and gather run every instance in
// one launch each, and each instance keeps its own Newton test and its own Jacobi-PCG recurrence
// on the device (scalars and stopping flags per instance; each CG loop one CUDA graph with a
// device-side while node).
//
// Instance s owns the equations [off_s, off_s + n_s) of the combined numbering, off_s a multiple
// of the 2048-entry reduction chunk; its elements keep their order, so every equation's gather
// sums the same (element, DOF) values in the same order as the instance alone, and the chunk
// reductions over its range are the documented order of a vector of n_s entries. An instance's
// Newton iterates, CG iterates and material states are therefore bit for bit those of
// fx_solver_newton (NormUnbalance) on the instance alone.
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
constexpr int64_t kMaxInstanceChunks = 2048;  // one level of chunk sums per instance

// per-instance scalars and flags
enum : int {
  N_RN = 0, N_BB, N_RZ, N_PAP, N_ALPHA, N_BETA, N_RR, N_RZNEW, N_TOL, N_RNORM,
  N_QBB, N_QRR, N_QBNORM,  // refinement: b.b, q.q (q = b - K du), ||b||
  N_QPREV,                 // refinement: ||q|| of the previous round
  NNS = 16
};
enum : int {
  G_NEWTON_DONE = 0,  // the Newton test has passed or the iteration limit is reached
  G_CONV,             // the Newton test passed
  G_ITERS,            // Newton solves
  G_CG_DONE,          // this CG solve is finished (the apply's and the vector kernels' gate)
  G_CG_ITERS, G_CG_TOTAL, G_CG_CONV, G_INDEF,
  G_CG_MAXIT,         // this CG solve's iteration limit
  G_IR_DONE,          // refinement: this linear solve is finished
  G_IR_OUTER,         // refinement rounds of this linear solve
  G_IR_INNER,         // inner iterations of this linear solve
  G_IR_REFS,          // refinement rounds in all
  NNF = 16
};

struct Range {
  int64_t off, n, c0, nc;
};

__device__ __forceinline__ int64_t chunk_len(const Range& r, int64_t begin) {
  const int64_t end = r.off + r.n;
  return (end - begin < kChunk) ? end - begin : kChunk;
}

// Called by every lane of the warp whose lane 0 has just written chunk sums of an instance: true
// (in all lanes) in the warp that counted the instance's last chunk, which then sees every chunk
// sum of the instance and resets its counter for the next launch.
__device__ __forceinline__ bool instance_last(unsigned* cnt, int64_t nc, int lane) {
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

// The second level of one instance's column j of chunk sums (k_nb_level's order), by one warp, the
// chunk sums read through L2 (other warps of the launch wrote them); the sum in every lane.
__device__ __forceinline__ double instance_level(const double* part, int64_t ld, int j, const Range& r, int lanes,
                                                 int lane) {
  const double* p = part + static_cast<int64_t>(j) * ld + r.c0;
  double acc = 0.0;
  if (lane < lanes)
    for (int64_t k = lane; k < r.nc; k += lanes) acc += __ldcg(p + k);
  double total = 0.0;
  for (int l = 0; l < lanes; ++l) total += __shfl_sync(0xffffffffu, acc, l);
  return total;
}

// chunk sums of x.y over the chunks of instances whose flag `gate` is 0 (column 0 of part)
template <class T>
__global__ void __launch_bounds__(32 * kWarps)
    k_nb_dot(const T* __restrict__ x, const T* __restrict__ y, int64_t nchunks,
             const int* __restrict__ owner, const Range* __restrict__ rg, const int* __restrict__ fl, int gate,
             int lanes, double* __restrict__ part) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = owner[c];
  if (s < 0 || fl[s * NNF + gate]) return;
  const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
  double acc = 0.0;
  if (lane < lanes)
    lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<T, 2>{{x[i], y[i]}}; },
                 [&](int64_t, const Ops<T, 2>& o) {
                   acc = fma(static_cast<double>(o.v[0]), static_cast<double>(o.v[1]), acc);
                 });
  double total = 0.0;
  for (int j = 0; j < lanes; ++j) total += __shfl_sync(0xffffffffu, acc, j);
  if (lane == 0) part[c] = total;
}

// second level: instance s's `ncol` columns of chunk sums (column j at part + j * ld) into
// sc[s * NNS + dst + j], a warp per (instance, column), for instances whose flag `gate` is 0
__global__ void k_nb_level(const double* __restrict__ part, int64_t ld, int ncol, const Range* __restrict__ rg,
                           const int* __restrict__ fl, int gate, int count, int lanes, double* __restrict__ sc,
                           int dst) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= count * ncol) return;
  const int s = w / ncol, j = w % ncol;
  if (fl[s * NNF + gate]) return;
  const double* p = part + static_cast<int64_t>(j) * ld + rg[s].c0;
  double acc = 0.0;
  if (lane < lanes)
    for (int64_t k = lane; k < rg[s].nc; k += lanes) acc += p[k];
  double total = 0.0;
  for (int l = 0; l < lanes; ++l) total += __shfl_sync(0xffffffffu, acc, l);
  if (lane == 0) sc[s * NNS + dst + j] = total;
}

// r = f_ext - f_int for instances still iterating
__global__ void __launch_bounds__(32 * kWarps)
    k_nb_residual(const double* __restrict__ fext, double* __restrict__ r, int64_t nchunks,
                  const int* __restrict__ owner, const Range* __restrict__ rg, const int* __restrict__ fl) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = owner[c];
  if (s < 0 || fl[s * NNF + G_NEWTON_DONE]) return;
  const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
  lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<double, 2>{{fext[i], r[i]}}; },
               [&](int64_t i, const Ops<double, 2>& o) { r[i] = o.v[0] - o.v[1]; });
}

// the Newton test per instance (NormUnbalance, absolute); instances that continue start a CG
// solve: G_CG_DONE = 0
__global__ void k_nb_test(double* sc, int* fl, int count, double tol, int max_newton) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  int* f = fl + s * NNF;
  double* c = sc + s * NNS;
  if (f[G_NEWTON_DONE]) return;
  const double rn = sqrt(c[N_RN]);
  c[N_RNORM] = rn;
  if (rn <= tol) {
    f[G_CONV] = 1;
    f[G_NEWTON_DONE] = 1;
  } else if (f[G_ITERS] >= max_newton) {
    f[G_NEWTON_DONE] = 1;
  }
  f[G_CG_DONE] = f[G_NEWTON_DONE];
}

// inverse of the tangent's diagonal (0 at equations of no instance)
__global__ void k_nb_inverse(const double* __restrict__ d, double* __restrict__ inv, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    inv[i] = d[i] != 0.0 ? 1.0 / d[i] : 0.0;
}

// CG from du = 0 (K 0 = 0): du = 0, rr = r, z = inv rr, p = z; chunk sums of rr.rr and rr.z
__global__ void __launch_bounds__(32 * kWarps)
    k_nb_cg_begin(const double* __restrict__ r, double* __restrict__ du, double* __restrict__ rr,
                  double* __restrict__ p, const double* __restrict__ inv, int64_t nchunks,
                  const int* __restrict__ owner, const Range* __restrict__ rg, const int* __restrict__ fl, int lanes,
                  double* __restrict__ part, int64_t ld) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = owner[c];
  if (s < 0 || fl[s * NNF + G_CG_DONE]) return;
  const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
  for (int64_t k = lane; k < len; k += 32) du[begin + k] = 0.0;
  double srr = 0.0, srz = 0.0;
  if (lane < lanes)
    lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<double, 2>{{r[i], inv[i]}}; },
                 [&](int64_t i, const Ops<double, 2>& o) {
                   const double ri = fma(-1.0, 0.0, o.v[0]);
                   const double zi = o.v[1] * ri;
                   rr[i] = ri;
                   p[i] = zi;
                   srr = fma(ri, ri, srr);
                   srz = fma(ri, zi, srz);
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

// per instance: the CG start (ConjugateGradient's tolerance max(rtol ||b||, atol), b = r)
// (ir: the inner solve of a refinement round, whose limit is what the linear solve has left)
__global__ void k_nb_cg_start(double* sc, int* fl, int count, double rtol, double atol, int max_it, int ir) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  int* f = fl + s * NNF;
  double* c = sc + s * NNS;
  if (f[G_CG_DONE]) return;
  if (ir) max_it -= f[G_IR_INNER];
  f[G_CG_MAXIT] = max_it;
  const double rhs = sqrt(c[N_RR]);  // b.b: the same sum as rr.rr at du = 0
  const double rn = sqrt(c[N_RR]);
  c[N_RZ] = c[N_RZNEW];
  const double tol = rtol * rhs;
  c[N_TOL] = tol > atol ? tol : atol;
  f[G_CG_ITERS] = 0;
  f[G_CG_CONV] = rn <= c[N_TOL];
  f[G_CG_DONE] = f[G_CG_CONV] || max_it <= 0;
}

// The CG's vector kernels in two forms with the same arithmetic and sums: BLOCK, a block of
// kChunkBlock threads per chunk (every entry's loads in flight at once, the chunk's sums by one warp
// from shared memory), for combined meshes of at most kBlockChunks chunks; otherwise a warp per
// chunk (8 per block, lane_loop). Both launch 256 threads per block.

// A CG iteration's p.ap: chunk sums of the instances still solving (T accumulated in double, fused
// multiply-adds, lane order), then in the warp that counts an instance's last chunk its second
// level and ConjugateGradient's alpha step (p.ap <= 0: indefinite, the solve ends).
template <class T, bool BLOCK>
__global__ void __launch_bounds__(256)
    k_nb_pap(const T* __restrict__ p, const T* __restrict__ ap, int64_t nchunks, const int* __restrict__ owner,
             const Range* __restrict__ rg, int* __restrict__ fl, int lanes, double* __restrict__ part,
             double* __restrict__ sc, unsigned* __restrict__ cnt) {
  int lane;
  int64_t c;
  int s;
  double total;
  if constexpr (BLOCK) {
    __shared__ T sa[kChunk], sb[kChunk];
    c = blockIdx.x;
    s = owner[c];
    if (s < 0 || fl[s * NNF + G_CG_DONE]) return;
    const int64_t begin = c * kChunk;
    const int len = static_cast<int>(chunk_len(rg[s], begin));
    T va[kChunkPer], vb[kChunkPer];
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
    s = owner[c];
    if (s < 0 || fl[s * NNF + G_CG_DONE]) return;
    const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
    double acc = 0.0;
    if (lane < lanes)
      lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<T, 2>{{p[i], ap[i]}}; },
                   [&](int64_t, const Ops<T, 2>& o) {
                     acc = fma(static_cast<double>(o.v[0]), static_cast<double>(o.v[1]), acc);
                   });
    total = 0.0;
    for (int j = 0; j < lanes; ++j) total += __shfl_sync(0xffffffffu, acc, j);
  }
  if (lane == 0) part[c] = total;
  if (!instance_last(cnt + s, rg[s].nc, lane)) return;
  const double pap = instance_level(part, nchunks, 0, rg[s], lanes, lane);
  if (lane == 0) {
    int* f = fl + s * NNF;
    double* cs = sc + s * NNS;
    cs[N_PAP] = pap;
    if (!(pap > 0.0)) {
      f[G_INDEF] = 1;
      f[G_CG_DONE] = 1;
    } else {
      cs[N_ALPHA] = cs[N_RZ] / pap;
    }
  }
}

// du += alpha p; rr -= alpha ap; chunk sums of rr.rr and rr.z (vectors of type T, sums in double);
// then in the warp that counts an instance's last chunk the two second levels and the iteration's
// end (ConjugateGradient's test on ||rr||, the iteration limit, beta)
template <class T, bool BLOCK>
__global__ void __launch_bounds__(256)
    k_nb_update(double* __restrict__ sc, int* __restrict__ fl, const T* __restrict__ p,
                const T* __restrict__ ap, const T* __restrict__ inv, T* __restrict__ du, T* __restrict__ rr,
                int64_t nchunks, const int* __restrict__ owner, const Range* __restrict__ rg, int lanes,
                double* __restrict__ part, int64_t ld, unsigned* __restrict__ cnt) {
  int lane;
  int64_t c;
  int s;
  double trr, trz;
  if constexpr (BLOCK) {
    __shared__ T sr[kChunk], sz[kChunk];
    c = blockIdx.x;
    s = owner[c];
    if (s < 0 || fl[s * NNF + G_CG_DONE]) return;
    const T alpha = static_cast<T>(sc[s * NNS + N_ALPHA]);
    const int64_t begin = c * kChunk;
    const int len = static_cast<int>(chunk_len(rg[s], begin));
    T vp[kChunkPer], vap[kChunkPer], vinv[kChunkPer], vdu[kChunkPer], vrr[kChunkPer];
#pragma unroll
    for (int k = 0; k < kChunkPer; ++k) {
      const int j = threadIdx.x + k * kChunkBlock;
      if (j < len) {
        const int64_t i = begin + j;
        vp[k] = p[i];
        vap[k] = ap[i];
        vinv[k] = inv[i];
        vdu[k] = du[i];
        vrr[k] = rr[i];
      }
    }
#pragma unroll
    for (int k = 0; k < kChunkPer; ++k) {
      const int j = threadIdx.x + k * kChunkBlock;
      if (j < len) {
        const int64_t i = begin + j;
        du[i] = fma(alpha, vp[k], vdu[k]);
        const T ri = fma(-alpha, vap[k], vrr[k]);
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
    s = owner[c];
    if (s < 0 || fl[s * NNF + G_CG_DONE]) return;
    const T alpha = static_cast<T>(sc[s * NNS + N_ALPHA]);
    const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
    double srr = 0.0, srz = 0.0;
    if (lane < lanes)
      lane_loop<4>(begin, len, lane, lanes,
                   [&](int64_t i) { return Ops<T, 5>{{p[i], ap[i], inv[i], du[i], rr[i]}}; },
                   [&](int64_t i, const Ops<T, 5>& o) {
                     du[i] = fma(alpha, o.v[0], o.v[3]);
                     const T ri = fma(-alpha, o.v[1], o.v[4]);
                     rr[i] = ri;
                     const T zi = o.v[2] * ri;
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
  if (!instance_last(cnt + s, rg[s].nc, lane)) return;
  const double srr_all = instance_level(part, ld, 0, rg[s], lanes, lane);
  const double srz_all = instance_level(part, ld, 1, rg[s], lanes, lane);
  if (lane != 0) return;
  int* f = fl + s * NNF;
  double* cs = sc + s * NNS;
  cs[N_RR] = srr_all;
  cs[N_RZNEW] = srz_all;
  const int max_it = f[G_CG_MAXIT];
  const double rn = sqrt(cs[N_RR]);
  const int it = ++f[G_CG_ITERS];
  if (rn <= cs[N_TOL]) {
    f[G_CG_CONV] = 1;
    f[G_CG_DONE] = 1;
    return;
  }
  if (it >= max_it) {
    f[G_CG_DONE] = 1;
    return;
  }
  cs[N_BETA] = cs[N_RZNEW] / cs[N_RZ];
  cs[N_RZ] = cs[N_RZNEW];
}

// p = inv rr + beta p
template <class T, bool BLOCK>
__global__ void __launch_bounds__(256)
    k_nb_p(const double* __restrict__ sc, const int* __restrict__ fl, const T* __restrict__ inv,
           const T* __restrict__ rr, T* __restrict__ p, int64_t nchunks, const int* __restrict__ owner,
           const Range* __restrict__ rg) {
  if constexpr (BLOCK) {
    const int64_t c = blockIdx.x;
    const int s = owner[c];
    if (s < 0 || fl[s * NNF + G_CG_DONE]) return;
    const T beta = static_cast<T>(sc[s * NNS + N_BETA]);
    const int64_t begin = c * kChunk;
    const int len = static_cast<int>(chunk_len(rg[s], begin));
    T vp[kChunkPer], vinv[kChunkPer], vrr[kChunkPer];
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
      if (j < len) p[begin + j] = fma(beta, vp[k], vinv[k] * vrr[k]);
    }
  } else {
    const int lane = threadIdx.x & 31;
    const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
    if (c >= nchunks) return;
    const int s = owner[c];
    if (s < 0 || fl[s * NNF + G_CG_DONE]) return;
    const T beta = static_cast<T>(sc[s * NNS + N_BETA]);
    const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
    lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<T, 3>{{p[i], inv[i], rr[i]}}; },
                 [&](int64_t i, const Ops<T, 3>& o) { p[i] = fma(beta, o.v[0], o.v[1] * o.v[2]); });
  }
}

// u += du for instances that solved this iteration; their counters
__global__ void __launch_bounds__(32 * kWarps)
    k_nb_correct(const double* __restrict__ du, double* __restrict__ u, int64_t nchunks,
                 const int* __restrict__ owner, const Range* __restrict__ rg, const int* __restrict__ fl) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = owner[c];
  if (s < 0 || fl[s * NNF + G_NEWTON_DONE]) return;
  const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
  lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<double, 2>{{u[i], du[i]}}; },
               [&](int64_t i, const Ops<double, 2>& o) { u[i] = o.v[0] + o.v[1]; });
}

// ---- FP32 CG inside FP64 refinement per instance: Solver::ir on each instance's equations
// the start of a linear solve: the instances still in Newton refine from du = 0
__global__ void k_nb_ir_start(int* fl, int count) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  int* f = fl + s * NNF;
  f[G_IR_DONE] = f[G_NEWTON_DONE];
  f[G_IR_OUTER] = 0;
  f[G_IR_INNER] = 0;
  f[G_CG_DONE] = 1;
}

// q = b - K du (b: the Newton residual r; K du in ap) for instances still refining
__global__ void __launch_bounds__(32 * kWarps)
    k_nb_ir_residual(const double* __restrict__ r, const double* __restrict__ ap, double* __restrict__ q,
                     int64_t nchunks, const int* __restrict__ owner, const Range* __restrict__ rg,
                     const int* __restrict__ fl) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = owner[c];
  if (s < 0 || fl[s * NNF + G_IR_DONE]) return;
  const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
  lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<double, 2>{{r[i], ap[i]}}; },
               [&](int64_t i, const Ops<double, 2>& o) { q[i] = o.v[0] - o.v[1]; });
}

// the refinement test: finished at ||q|| <= max(rtol ||b||, atol), at the round or inner
// iteration limit, or when the last round did not halve ||q|| (the FP64 residual has reached
// what FP64 can resolve: Solver::ir's stagnation test); otherwise an inner solve follows
// (G_CG_DONE = 0)
__global__ void k_nb_ir_test(double* sc, int* fl, int count, double rtol, double atol, int max_outer, int max_it) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  int* f = fl + s * NNF;
  double* c = sc + s * NNS;
  if (f[G_IR_DONE]) return;
  if (f[G_IR_OUTER] == 0) c[N_QBNORM] = sqrt(c[N_QBB]);
  const double rn = sqrt(c[N_QRR]);
  const double tol = rtol * c[N_QBNORM];
  const bool stalled = f[G_IR_OUTER] > 0 && rn > kIrStall * c[N_QPREV];
  if (rn <= (tol > atol ? tol : atol) || stalled || f[G_IR_OUTER] >= max_outer || f[G_IR_INNER] >= max_it) {
    f[G_IR_DONE] = 1;
    return;
  }
  c[N_QPREV] = rn;
  f[G_CG_DONE] = 0;
}

// the inner solve's start, FP32 CG from d = 0 (K 0 = 0): r32 = (float) q, d = 0, rr = r32,
// z = inv32 rr, p = z; chunk sums of rr.rr and rr.z (columns 0 and 1 of part)
__global__ void __launch_bounds__(32 * kWarps)
    k_nb_ir_begin(const double* __restrict__ q, float* __restrict__ r32, float* __restrict__ d32,
                  float* __restrict__ rr, float* __restrict__ p, const float* __restrict__ inv, int64_t nchunks,
                  const int* __restrict__ owner, const Range* __restrict__ rg, const int* __restrict__ fl, int lanes,
                  double* __restrict__ part, int64_t ld) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = owner[c];
  if (s < 0 || fl[s * NNF + G_CG_DONE]) return;
  const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
  lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<double, 1>{{q[i]}}; },
               [&](int64_t i, const Ops<double, 1>& o) {
                 r32[i] = static_cast<float>(o.v[0]);
                 d32[i] = 0.f;
               });
  __syncwarp();
  double srr = 0.0, srz = 0.0;
  if (lane < lanes)
    lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<float, 2>{{r32[i], inv[i]}}; },
                 [&](int64_t i, const Ops<float, 2>& o) {
                   const float ri = fmaf(-1.f, 0.f, o.v[0]);
                   const float zi = o.v[1] * ri;
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

// the CG loop's condition: another pass while an instance's solve is running, at most `cap` passes
__global__ void k_nb_cond(cudaGraphConditionalHandle h, const int* __restrict__ fl, int count, int* __restrict__ passes,
                          int cap) {
  int mine = 0;
  for (int s = threadIdx.x; s < count; s += blockDim.x) mine |= !fl[s * NNF + G_CG_DONE];
  const int running = __syncthreads_or(mine);
  if (threadIdx.x == 0) {
    const int c = ++*passes;
    cudaGraphSetConditional(h, (running && c < cap) ? 1u : 0u);
  }
}

// du += (double) d32 for instances that ran this round's inner solve
__global__ void __launch_bounds__(32 * kWarps)
    k_nb_ir_correct(const float* __restrict__ d32, double* __restrict__ du, int64_t nchunks,
                    const int* __restrict__ owner, const Range* __restrict__ rg, const int* __restrict__ fl) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int s = owner[c];
  if (s < 0 || fl[s * NNF + G_IR_DONE]) return;
  const int64_t begin = c * kChunk, len = chunk_len(rg[s], begin);
  lane_loop<8>(begin, len, lane, 32, [&](int64_t i) { return Ops<double, 2>{{du[i], static_cast<double>(d32[i])}}; },
               [&](int64_t i, const Ops<double, 2>& o) { du[i] = o.v[0] + o.v[1]; });
}

// the end of a round: the counters, and the end of the solve when its inner solve made no
// progress; the inner iterations are added to the Newton iteration's total here
__global__ void k_nb_ir_round_end(int* fl, int count) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  int* f = fl + s * NNF;
  if (f[G_IR_DONE]) return;
  f[G_IR_INNER] += f[G_CG_ITERS];
  f[G_CG_TOTAL] += f[G_CG_ITERS];
  f[G_IR_OUTER] += 1;
  f[G_IR_REFS] += 1;
  if (f[G_CG_ITERS] == 0 && !f[G_CG_CONV]) f[G_IR_DONE] = 1;
  f[G_CG_ITERS] = 0;
}

// the inverse of the tangent's diagonal in FP32 (0 at equations of no instance)
__global__ void k_nb_inverse32(const double* __restrict__ d, float* __restrict__ inv, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    inv[i] = d[i] != 0.0 ? static_cast<float>(1.0 / d[i]) : 0.f;
}

__global__ void k_nb_iteration_end(int* fl, int count) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  int* f = fl + s * NNF;
  if (f[G_NEWTON_DONE]) return;
  f[G_CG_TOTAL] += f[G_CG_ITERS];
  f[G_ITERS] += 1;
}

unsigned chunk_grid(int64_t nchunks) { return static_cast<unsigned>(std::max<int64_t>(1, (nchunks + kWarps - 1) / kWarps)); }
unsigned ew(int64_t n) {
  const int64_t blocks = (n + 255) / 256;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(blocks, static_cast<int64_t>(num_sms()) * 8)));
}

}  // namespace

struct NBatch {
  int device = 0;
  int count = 0;
  int64_t total = 0, nchunks = 0;
  fx_force* force = nullptr;
  fx_solve_opts o{};
  cudaStream_t cs = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::vector<Range> rg_h;
  DeviceArray<Range> rg;
  DeviceArray<int> owner;
  DeviceArray<double> r, du, rr, p, ap, d, inv, zero, part, sc;
  DeviceArray<int> fl;
  DeviceArray<unsigned> cnt;  // per instance: chunks counted by the fused reductions (0 between launches)
  DeviceArray<int> passes;    // the CG loop graph's pass count
  int* fl_h = nullptr;
  double* sc_h = nullptr;
  cudaGraphExec_t graph = nullptr;
  // FP32 CG inside FP64 refinement (FX_SOLVER_IR): q = b - K du, the FP32 inner vectors
  int method = FX_SOLVER_CG;
  double inner_rtol = 1e-4;
  DeviceArray<double> q;
  DeviceArray<float> r32, d32, rr32, p32, ap32, inv32;
  cudaGraphExec_t graph32 = nullptr;

  ~NBatch() {
    if (graph) cudaGraphExecDestroy(graph);
    if (graph32) cudaGraphExecDestroy(graph32);
    if (fl_h) cudaFreeHost(fl_h);
    if (sc_h) cudaFreeHost(sc_h);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (cs) cudaStreamDestroy(cs);
    if (force) fx_force_destroy(force);
  }

  void read_flags() {
    FX_CUDA(cudaMemcpyAsync(fl_h, fl.ptr, sizeof(int) * NNF * count, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaMemcpyAsync(sc_h, sc.ptr, sizeof(double) * NNS * count, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
  }
  unsigned inst_grid() const { return static_cast<unsigned>((count + 127) / 128); }
  void level(int ncol, int gate, int dst) {
    const int warps = count * ncol;
    k_nb_level<<<(warps + 7) / 8, 256, 0, cs>>>(part.ptr, nchunks, ncol, rg.ptr, fl.ptr, gate, count, o.lanes,
                                                sc.ptr, dst);
    FX_LAUNCH_CHECK("nbatch_level");
  }

  // the vector kernels of one CG iteration (in vectors of type T), in the form for this many chunks
  template <class T>
  void cg_vectors(T* pv, T* apv, const T* iv, T* dv, T* rv) {
    if (nchunks <= kBlockChunks) {  // a block per chunk
      const unsigned gb = static_cast<unsigned>(nchunks);
      k_nb_pap<T, true><<<gb, kChunkBlock, 0, cs>>>(pv, apv, nchunks, owner.ptr, rg.ptr, fl.ptr, o.lanes, part.ptr,
                                                    sc.ptr, cnt.ptr);
      k_nb_update<T, true><<<gb, kChunkBlock, 0, cs>>>(sc.ptr, fl.ptr, pv, apv, iv, dv, rv, nchunks, owner.ptr,
                                                       rg.ptr, o.lanes, part.ptr, nchunks, cnt.ptr);
      k_nb_p<T, true><<<gb, kChunkBlock, 0, cs>>>(sc.ptr, fl.ptr, iv, rv, pv, nchunks, owner.ptr, rg.ptr);
    } else {  // a warp per chunk
      const unsigned g = chunk_grid(nchunks);
      k_nb_pap<T, false><<<g, 32 * kWarps, 0, cs>>>(pv, apv, nchunks, owner.ptr, rg.ptr, fl.ptr, o.lanes, part.ptr,
                                                    sc.ptr, cnt.ptr);
      k_nb_update<T, false><<<g, 32 * kWarps, 0, cs>>>(sc.ptr, fl.ptr, pv, apv, iv, dv, rv, nchunks, owner.ptr,
                                                       rg.ptr, o.lanes, part.ptr, nchunks, cnt.ptr);
      k_nb_p<T, false><<<g, 32 * kWarps, 0, cs>>>(sc.ptr, fl.ptr, iv, rv, pv, nchunks, owner.ptr, rg.ptr);
    }
  }

  void cg_iteration() {
    const double k[3] = {1.0, 0.0, 0.0};
    general_apply(force->s, k, p.ptr, ap.ptr, cs);
    cg_vectors<double>(p.ptr, ap.ptr, inv.ptr, du.ptr, rr.ptr);
    FX_LAUNCH_CHECK("nbatch_cg");
  }

  // one iteration of the inner FP32 CG (the FP32 operator on the stored point tangents)
  void cg_iteration32() {
    const double k[3] = {1.0, 0.0, 0.0};
    general_apply_f32(force->s, k, p32.ptr, ap32.ptr, cs);
    cg_vectors<float>(p32.ptr, ap32.ptr, inv32.ptr, d32.ptr, rr32.ptr);
    FX_LAUNCH_CHECK("nbatch_cg32");
  }

  // CG iterations until every instance's solve is done: a first block of 8 eagerly (the first
  // applies build lazy state), then a kept graph (one per precision) whose while node runs blocks of
  // 8 iterations and a condition kernel until no instance is running, with one host read at the end
  void cg_loop(bool f32) {
    const int block = 8;
    for (int i = 0; i < block; ++i) {
      if (f32) cg_iteration32();
      else cg_iteration();
    }
    read_flags();
    cudaGraphExec_t& gx = f32 ? graph32 : graph;
    if (any(G_CG_DONE, 0)) {
      if (!gx) {
        cudaGraph_t g = nullptr;
        FX_CUDA(cudaGraphCreate(&g, 0));
        try {
          cudaGraphConditionalHandle h;
          FX_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
          cudaGraphNodeParams cp{};
          cp.type = cudaGraphNodeTypeConditional;
          cp.conditional.handle = h;
          cp.conditional.type = cudaGraphCondTypeWhile;
          cp.conditional.size = 1;
          cudaGraphNode_t node;
          FX_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
          cudaGraph_t body = cp.conditional.phGraph_out[0];
          FX_CUDA(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
          try {
            for (int i = 0; i < block; ++i) {
              if (f32) cg_iteration32();
              else cg_iteration();
            }
            // every solve ends within its iteration limit; the cap only bounds the loop
            const int cap = (std::max(o.max_iterations, 0) + block - 1) / block + 2;
            k_nb_cond<<<1, 128, 0, cs>>>(h, fl.ptr, count, passes.ptr, cap);
            FX_LAUNCH_CHECK("nbatch_cg_condition");
          } catch (...) {
            cudaStreamEndCapture(cs, &body);
            throw;
          }
          FX_CUDA(cudaStreamEndCapture(cs, &body));
          FX_CUDA(cudaGraphInstantiate(&gx, g, 0));
        } catch (...) {
          if (gx) cudaGraphExecDestroy(gx);
          gx = nullptr;
          cudaGraphDestroy(g);
          throw;
        }
        cudaGraphDestroy(g);
      }
      FX_CUDA(cudaMemsetAsync(passes.ptr, 0, sizeof(int), cs));
      FX_CUDA(cudaGraphLaunch(gx, cs));
      read_flags();
      // every solve ends within its iteration limit, well inside the loop's cap
      if (any(G_CG_DONE, 0)) throw Error(FX_E_INVALID, "batched CG: a solve did not end within its iteration limit");
    }
  }

  // K_t du = r per instance by FP32 CG inside FP64 refinement (Solver::ir's rounds)
  void linear_ir() {
    const double k[3] = {1.0, 0.0, 0.0};
    const unsigned g = chunk_grid(nchunks);
    FX_CUDA(cudaMemsetAsync(du.ptr, 0, sizeof(double) * static_cast<size_t>(total), cs));
    k_nb_ir_start<<<inst_grid(), 128, 0, cs>>>(fl.ptr, count);
    for (int round = 0;; ++round) {
      general_apply(force->s, k, du.ptr, ap.ptr, cs);
      k_nb_ir_residual<<<g, 32 * kWarps, 0, cs>>>(r.ptr, ap.ptr, q.ptr, nchunks, owner.ptr, rg.ptr, fl.ptr);
      if (round == 0) {
        k_nb_dot<double><<<g, 32 * kWarps, 0, cs>>>(r.ptr, r.ptr, nchunks, owner.ptr, rg.ptr, fl.ptr, G_IR_DONE,
                                                    o.lanes, part.ptr);
        level(1, G_IR_DONE, N_QBB);
      }
      k_nb_dot<double><<<g, 32 * kWarps, 0, cs>>>(q.ptr, q.ptr, nchunks, owner.ptr, rg.ptr, fl.ptr, G_IR_DONE, o.lanes,
                                                  part.ptr);
      level(1, G_IR_DONE, N_QRR);
      k_nb_ir_test<<<inst_grid(), 128, 0, cs>>>(sc.ptr, fl.ptr, count, o.rtol, o.atol, 50, o.max_iterations);
      FX_LAUNCH_CHECK("nbatch_ir_test");
      read_flags();
      if (!any(G_IR_DONE, 0)) break;
      k_nb_ir_begin<<<g, 32 * kWarps, 0, cs>>>(q.ptr, r32.ptr, d32.ptr, rr32.ptr, p32.ptr, inv32.ptr, nchunks,
                                               owner.ptr, rg.ptr, fl.ptr, o.lanes, part.ptr, nchunks);
      level(2, G_CG_DONE, N_RR);
      k_nb_cg_start<<<inst_grid(), 128, 0, cs>>>(sc.ptr, fl.ptr, count, inner_rtol, 0.0, o.max_iterations, 1);
      FX_LAUNCH_CHECK("nbatch_ir_inner_begin");
      cg_loop(true);
      k_nb_ir_correct<<<g, 32 * kWarps, 0, cs>>>(d32.ptr, du.ptr, nchunks, owner.ptr, rg.ptr, fl.ptr);
      k_nb_ir_round_end<<<inst_grid(), 128, 0, cs>>>(fl.ptr, count);
      FX_LAUNCH_CHECK("nbatch_ir_round");
    }
  }

  bool any(int flag, int value) const {
    for (int s = 0; s < count; ++s)
      if (fl_h[s * NNF + flag] == value) return true;
    return false;
  }

  // one load step of every instance (NormUnbalance, absolute tol)
  void step(const double* fext, double* u, double tol, int max_newton) {
    const double k[3] = {1.0, 0.0, 0.0};
    const unsigned g = chunk_grid(nchunks);
    FX_CUDA(cudaMemsetAsync(fl.ptr, 0, sizeof(int) * NNF * count, cs));
    for (;;) {
      general_force(force->s, u, zero.ptr, r.ptr, cs);
      k_nb_residual<<<g, 32 * kWarps, 0, cs>>>(fext, r.ptr, nchunks, owner.ptr, rg.ptr, fl.ptr);
      k_nb_dot<<<g, 32 * kWarps, 0, cs>>>(r.ptr, r.ptr, nchunks, owner.ptr, rg.ptr, fl.ptr, G_NEWTON_DONE, o.lanes,
                                          part.ptr);
      level(1, G_NEWTON_DONE, N_RN);
      k_nb_test<<<inst_grid(), 128, 0, cs>>>(sc.ptr, fl.ptr, count, tol, max_newton);
      FX_LAUNCH_CHECK("nbatch_test");
      read_flags();
      if (!any(G_NEWTON_DONE, 0)) break;
      general_diagonal(force->s, k, d.ptr, cs);
      k_nb_inverse<<<ew(total), 256, 0, cs>>>(d.ptr, inv.ptr, total);
      if (method == FX_SOLVER_IR) {
        k_nb_inverse32<<<ew(total), 256, 0, cs>>>(d.ptr, inv32.ptr, total);
        linear_ir();
      } else {
        k_nb_cg_begin<<<g, 32 * kWarps, 0, cs>>>(r.ptr, du.ptr, rr.ptr, p.ptr, inv.ptr, nchunks, owner.ptr, rg.ptr,
                                                 fl.ptr, o.lanes, part.ptr, nchunks);
        level(2, G_CG_DONE, N_RR);
        k_nb_cg_start<<<inst_grid(), 128, 0, cs>>>(sc.ptr, fl.ptr, count, o.rtol, o.atol, o.max_iterations, 0);
        FX_LAUNCH_CHECK("nbatch_cg_begin");
        cg_loop(false);
      }
      k_nb_correct<<<g, 32 * kWarps, 0, cs>>>(du.ptr, u, nchunks, owner.ptr, rg.ptr, fl.ptr);
      k_nb_iteration_end<<<inst_grid(), 128, 0, cs>>>(fl.ptr, count);
      FX_LAUNCH_CHECK("nbatch_correct");
    }
  }
};

}  // namespace fx

struct fx_nbatch {
  fx::NBatch b;
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

int fx_nbatch_create(const fx_mesh* meshes, int32_t count, int32_t device, fx_solve_opts o, fx_nbatch** out) {
  return guard([&] {
    if (!meshes || count <= 0 || !out) throw fx::Error(FX_E_INVALID, "fx_nbatch_create: bad arguments");
    if (o.lanes <= 0) o.lanes = 32;
    if (o.lanes > 32 || o.max_iterations < 0) throw fx::Error(FX_E_INVALID, "fx_nbatch_create: bad solver options");
    // offsets of every instance in the combined mesh
    int64_t N = 0, E = 0, Pn = 0, Q = 0;
    std::vector<int64_t> no(count), eo(count), po(count), qo(count);
    for (int i = 0; i < count; ++i) {
      const fx_mesh& m = meshes[i];
      if (m.num_equations <= 0) throw fx::Error(FX_E_INVALID, "fx_nbatch_create: an instance has no equations");
      if (fx::chunks_of(m.num_equations) > fx::kMaxInstanceChunks)
        throw fx::Error(FX_E_UNSUPPORTED, "fx_nbatch_create: an instance has more than 2048 * 2048 equations");
      no[i] = N, eo[i] = E, po[i] = Pn, qo[i] = Q;
      N += m.num_nodes;
      E += m.count;
      Pn += m.num_params;
      Q += fx::chunks_of(m.num_equations) * fx::kChunk;
    }
    if (N > INT32_MAX || E > INT32_MAX || Q > INT32_MAX) throw fx::Error(FX_E_UNSUPPORTED, "fx_nbatch_create: too large");
    const int64_t P = (E + 31) / 32 * 32;
    std::vector<double> coords(static_cast<size_t>(3 * N));
    std::vector<int32_t> node(static_cast<size_t>(8 * P), 0), eq(static_cast<size_t>(24 * P), -1),
        param(static_cast<size_t>(P), 0);
    std::vector<fx_param_set> params(static_cast<size_t>(Pn));
    std::vector<double> lumped(static_cast<size_t>(Q), 0.0), nmass(static_cast<size_t>(Q), 0.0),
        namass(static_cast<size_t>(Q), 0.0);
    std::vector<int8_t> eqdof(static_cast<size_t>(Q), 0);
    bool any_lumped = false, any_nmass = false, any_namass = false;
    for (int i = 0; i < count; ++i) {
      const fx_mesh& m = meshes[i];
      for (int d = 0; d < 3; ++d)
        std::copy(m.coords + static_cast<int64_t>(d) * m.num_nodes, m.coords + static_cast<int64_t>(d + 1) * m.num_nodes,
                  coords.begin() + d * N + no[i]);
      for (int32_t e = 0; e < m.count; ++e) {
        const int64_t ce = eo[i] + e;
        for (int a = 0; a < 8; ++a)
          node[a * P + ce] = static_cast<int32_t>(m.node[static_cast<int64_t>(a) * m.padded + e] + no[i]);
        for (int k = 0; k < 24; ++k) {
          const int32_t q = m.eq[static_cast<int64_t>(k) * m.padded + e];
          eq[k * P + ce] = q >= 0 ? static_cast<int32_t>(q + qo[i]) : -1;
        }
        param[ce] = static_cast<int32_t>(m.param[e] + po[i]);
      }
      std::copy(m.params, m.params + m.num_params, params.begin() + po[i]);
      auto put = [&](const double* src, std::vector<double>& dst, bool& any) {
        if (!src) return;
        any = true;
        std::copy(src, src + m.num_equations, dst.begin() + qo[i]);
      };
      put(m.lumped_mass, lumped, any_lumped);
      put(m.nodal_mass, nmass, any_nmass);
      put(m.nodal_alpha_mass, namass, any_namass);
      if (m.eq_dof) std::copy(m.eq_dof, m.eq_dof + m.num_equations, eqdof.begin() + qo[i]);
    }
    fx_mesh cm{};
    cm.num_nodes = static_cast<int32_t>(N);
    cm.num_equations = static_cast<int32_t>(Q);
    cm.coords = coords.data();
    cm.count = static_cast<int32_t>(E);
    cm.padded = static_cast<int32_t>(P);
    cm.node = node.data();
    cm.eq = eq.data();
    cm.param = param.data();
    cm.num_params = static_cast<int32_t>(Pn);
    cm.params = params.data();
    cm.lumped_mass = any_lumped ? lumped.data() : nullptr;
    cm.nodal_mass = any_nmass ? nmass.data() : nullptr;
    cm.nodal_alpha_mass = any_namass ? namass.data() : nullptr;
    cm.eq_dof = eqdof.data();
    auto* h = new fx_nbatch;
    fx::NBatch& b = h->b;
    try {
      const int rc = fx_force_create(&cm, device, &b.force);
      if (rc != FX_OK) throw fx::Error(rc, fx_last_error());
      b.device = device;
      b.count = count;
      b.total = Q;
      b.nchunks = fx::chunks_of(Q);
      b.o = o;
      b.rg_h.resize(static_cast<size_t>(count));
      std::vector<int> owner(static_cast<size_t>(b.nchunks), -1);
      for (int i = 0; i < count; ++i) {
        const int64_t nc = fx::chunks_of(meshes[i].num_equations);
        b.rg_h[i] = fx::Range{qo[i], meshes[i].num_equations, qo[i] / fx::kChunk, nc};
        for (int64_t c = 0; c < nc; ++c) owner[qo[i] / fx::kChunk + c] = i;
      }
      FX_CUDA(cudaSetDevice(device));
      FX_CUDA(cudaStreamCreateWithFlags(&b.cs, cudaStreamNonBlocking));
      FX_CUDA(cudaEventCreateWithFlags(&b.ev_in, cudaEventDisableTiming));
      FX_CUDA(cudaEventCreateWithFlags(&b.ev_out, cudaEventDisableTiming));
      b.rg.upload(b.rg_h);
      b.owner.upload(owner);
      for (auto* v : {&b.r, &b.du, &b.rr, &b.p, &b.ap, &b.d, &b.inv, &b.zero}) {
        v->alloc(static_cast<size_t>(Q));
        v->zero(nullptr);
      }
      b.part.alloc(static_cast<size_t>(b.nchunks) * 2);
      b.sc.alloc(static_cast<size_t>(count) * fx::NNS);
      b.fl.alloc(static_cast<size_t>(count) * fx::NNF);
      b.cnt.alloc(static_cast<size_t>(count));
      b.cnt.zero(nullptr);
      b.passes.alloc(1);
      FX_CUDA(cudaMallocHost(&b.fl_h, sizeof(int) * fx::NNF * count));
      FX_CUDA(cudaMallocHost(&b.sc_h, sizeof(double) * fx::NNS * count));
      // the creation's work is on the legacy stream; a device-wide synchronization would also wait
      // for (and break the capture of) another thread's graph capture on its own stream
      FX_CUDA(cudaStreamSynchronize(nullptr));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

void fx_nbatch_destroy(fx_nbatch* b) { delete b; }

int fx_nbatch_layout(const fx_nbatch* h, int64_t* offsets, int64_t* equations) {
  return guard([&] {
    if (!h || !offsets) throw fx::Error(FX_E_INVALID, "fx_nbatch_layout: bad arguments");
    for (int i = 0; i < h->b.count; ++i) {
      offsets[i] = h->b.rg_h[i].off;
      if (equations) equations[i] = h->b.rg_h[i].n;
    }
    offsets[h->b.count] = h->b.total;
  });
}

fx_force* fx_nbatch_force(fx_nbatch* h) { return h ? h->b.force : nullptr; }

int fx_nbatch_set_inner(fx_nbatch* h, int32_t method, double inner_rtol) {
  return guard([&] {
    if (!h || (method != FX_SOLVER_CG && method != FX_SOLVER_IR) || !(inner_rtol > 0.0 && inner_rtol < 1.0))
      throw fx::Error(FX_E_INVALID, "fx_nbatch_set_inner: bad arguments");
    fx::NBatch& b = h->b;
    FX_CUDA(cudaSetDevice(b.device));
    b.method = method;
    b.inner_rtol = inner_rtol;
    if (method == FX_SOLVER_IR && b.q.n == 0) {
      const size_t n = static_cast<size_t>(std::max<int64_t>(b.total, 1));
      b.q.alloc(n);
      b.q.zero(b.cs);
      for (auto* v : {&b.r32, &b.d32, &b.rr32, &b.p32, &b.ap32, &b.inv32}) {
        v->alloc(n);
        FX_CUDA(cudaMemsetAsync(v->ptr, 0, sizeof(float) * n, b.cs));
      }
      FX_CUDA(cudaStreamSynchronize(b.cs));
    }
  });
}

int fx_nbatch_step(fx_nbatch* h, const double* fext, double* u, double tol, int32_t max_newton,
                   int32_t* newton_iterations, fx_solve_result* results, void* stream) {
  return guard([&] {
    if (!h || !fext || !u || !(tol >= 0.0) || max_newton < 0)
      throw fx::Error(FX_E_INVALID, "fx_nbatch_step: bad arguments");
    fx::NBatch& b = h->b;
    FX_CUDA(cudaSetDevice(b.device));
    auto st = static_cast<cudaStream_t>(stream);
    FX_CUDA(cudaEventRecord(b.ev_in, st));
    FX_CUDA(cudaStreamWaitEvent(b.cs, b.ev_in, 0));
    b.step(fext, u, tol, max_newton);
    FX_CUDA(cudaEventRecord(b.ev_out, b.cs));
    FX_CUDA(cudaStreamWaitEvent(st, b.ev_out, 0));
    for (int i = 0; i < b.count; ++i) {
      const int* f = b.fl_h + i * fx::NNF;
      const double* c = b.sc_h + i * fx::NNS;
      if (newton_iterations) newton_iterations[i] = f[fx::G_ITERS];
      if (results) {
        fx_solve_result r{};
        r.converged = f[fx::G_CONV];
        r.iterations = f[fx::G_CG_TOTAL];
        r.refinements = f[fx::G_IR_REFS];
        r.final_residual = c[fx::N_RNORM];
        r.indefinite = f[fx::G_INDEF];
        r.status = r.converged ? FX_OK : (r.indefinite ? FX_E_NOT_SPD : FX_E_DIVERGED);
        results[i] = r;
      }
    }
  });
}

}  // extern "C"
