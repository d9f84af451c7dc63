// Linear solvers on the matrix-free operator (solvers::LinearSolver and its implementations,
// src/solvers/linear_solver.hpp:96-105, cg.cpp:24-71, gmres.cpp:32-123, krylov.cpp:25-41,
// jacobi.cpp:10-26), B200-resident.
//
// CG keeps its scalars on the device: one iteration is the operator, the p.Ap reduction, a
// one-thread kernel for alpha, one fused pass that updates x and r and forms the chunk sums of
// r.r and r.z (z = D^-1 r, never stored), the reduction levels, a one-thread kernel for the
// convergence test and beta, and the p update. The iterations run as a CUDA graph; the host
// reads the `done` flag after each block of iterations. Every kernel returns at once when the
// solve is done, so the iterate is frozen at the converged one. All reductions use the
// documented chunk/lane order (fused multiply-adds), so a solve gives the same bits every run.
#include <functional>
#include <algorithm>
#include <cstring>
#include <cmath>
#include <vector>

#include "force.hpp"
#include "vector.hpp"

// scalar slots of one solve
enum : int {
  S_RZ = 0,
  S_PAP = 1,
  S_ALPHA = 2,
  S_BETA = 3,
  S_RNORM = 4,
  S_TOL = 5,
  S_RHS = 6,
  S_RR = 7,      // r.r of the update kernel (with S_RZNEW contiguous: two columns)
  S_RZNEW = 8,
  S_INIT = 9,
  S_BB = 10,
  S_NSCALAR = 16
};
enum : int { F_DONE = 0, F_CONV = 1, F_INDEF = 2, F_ITERS = 3, F_NFLAG = 4 };

namespace fx {
namespace {

constexpr int kWarps = 8;
// A lane's sum runs over its entries in index order (the documented order), but the operands of
// kAhead consecutive iterations are fetched before their products are added, so that a warp has
// that many loads in flight per vector instead of one: the chunks are few per SM, and one load
// at a time leaves them waiting on memory latency.
constexpr int kAhead = 8;

// the scalar steps of an iteration (alpha, then the test and beta), defined below
__device__ void cg_alpha_step(double* sc, int* fl);
__device__ void cg_beta_step(double* sc, int* fl, int max_it);

// documented-order chunk sums of x.y for vectors of type T, accumulated in double
template <class T>
__global__ void __launch_bounds__(32 * kWarps) k_dot_chunks(const T* __restrict__ x, const T* __restrict__ y, int64_t n,
                                                            int lanes, int64_t nchunks, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int64_t begin = c * kChunk;
  const int64_t len = (n - begin < kChunk) ? n - begin : kChunk;
  double s = 0.0;
  if (lane < lanes) {
    int64_t k = lane;
    for (; k + (kAhead - 1) * lanes < len; k += kAhead * lanes) {
      T a[kAhead], b[kAhead];
#pragma unroll
      for (int u = 0; u < kAhead; ++u) {
        a[u] = x[begin + k + u * lanes];
        b[u] = y[begin + k + u * lanes];
      }
#pragma unroll
      for (int u = 0; u < kAhead; ++u) s = fma(static_cast<double>(a[u]), static_cast<double>(b[u]), s);
    }
    for (; k < len; k += lanes) s = fma(static_cast<double>(x[begin + k]), static_cast<double>(y[begin + k]), s);
  }
  double total = 0.0;
  for (int j = 0; j < lanes; ++j) total += __shfl_sync(0xffffffffu, s, j);
  if (lane == 0) out[c] = total;
}

// chunk sums of p.Ap; then, in the grid's last block, their levels (into S_PAP) and the alpha step
template <class T>
__global__ void __launch_bounds__(32 * kWarps) k_cg_pap(const T* __restrict__ p, const T* __restrict__ ap, int64_t n,
                                                        int lanes, int64_t nchunks, double* __restrict__ out,
                                                        double* __restrict__ out2, unsigned* __restrict__ counter,
                                                        double* __restrict__ sc, int* __restrict__ fl) {
  if (fl[F_DONE]) return;  // (the same for every block: the counter stays untouched)
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  const int64_t begin = c * kChunk;
  const int64_t len = c >= nchunks ? 0 : ((n - begin < kChunk) ? n - begin : kChunk);
  double s = 0.0;
  if (lane < lanes)
    lane_loop<kAhead>(begin, len, lane, lanes, [&](int64_t i) { return Ops<T, 2>{{p[i], ap[i]}}; },
                      [&](int64_t, const Ops<T, 2>& o) {
                        s = fma(static_cast<double>(o.v[0]), static_cast<double>(o.v[1]), s);
                      });
  double total = 0.0;
  for (int j = 0; j < lanes; ++j) total += __shfl_sync(0xffffffffu, s, j);
  if (lane == 0 && c < nchunks) out[c] = total;
  if (!last_block(counter)) return;
  block_levels(out, out2, nchunks, 1, lanes, sc + S_PAP);
  if (threadIdx.x == 0) {
    *counter = 0u;
    cg_alpha_step(sc, fl);
  }
}

// r = b - ap; z = inv r; p = z; chunk sums of r.r and r.z (columns 0 and 1 of out)
template <class T>
__global__ void __launch_bounds__(32 * kWarps) k_cg_begin(const T* __restrict__ b, const T* __restrict__ ap,
                                                          const T* __restrict__ inv, T* __restrict__ r,
                                                          T* __restrict__ p, int64_t n, int lanes, int64_t nchunks,
                                                          double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const int64_t begin = c * kChunk;
  const int64_t len = (n - begin < kChunk) ? n - begin : kChunk;
  double srr = 0.0, srz = 0.0;
  auto one = [&](int64_t i, T bi, T ai, T vi) {
    const T ri = fma(T(-1), ai, bi);
    const T zi = vi * ri;
    r[i] = ri;
    p[i] = zi;
    srr = fma(static_cast<double>(ri), static_cast<double>(ri), srr);
    srz = fma(static_cast<double>(ri), static_cast<double>(zi), srz);
  };
  if (lane < lanes) {
    constexpr int U = kAhead / 2;
    int64_t k = lane;
    for (; k + (U - 1) * lanes < len; k += U * lanes) {
      T bv[U], av[U], vv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t i = begin + k + u * lanes;
        bv[u] = b[i];
        av[u] = ap[i];
        vv[u] = inv[i];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) one(begin + k + u * lanes, bv[u], av[u], vv[u]);
    }
    for (; k < len; k += lanes) one(begin + k, b[begin + k], ap[begin + k], inv[begin + k]);
  }
  double trr = 0.0, trz = 0.0;
  for (int j = 0; j < lanes; ++j) {
    trr += __shfl_sync(0xffffffffu, srr, j);
    trz += __shfl_sync(0xffffffffu, srz, j);
  }
  if (lane == 0) {
    out[c] = trr;
    out[nchunks + c] = trz;
  }
}

// x += alpha p; r -= alpha ap; chunk sums of r.r and r.z; then, in the grid's last block, their
// levels (into S_RR, S_RZNEW) and the beta step: the convergence test, the iteration count, beta
template <class T>
__global__ void __launch_bounds__(32 * kWarps) k_cg_update(double* __restrict__ sc, int* __restrict__ fl,
                                                           const T* __restrict__ p, const T* __restrict__ ap,
                                                           const T* __restrict__ inv, T* __restrict__ x,
                                                           T* __restrict__ r, int64_t n, int lanes, int64_t nchunks,
                                                           double* __restrict__ out, double* __restrict__ out2,
                                                           unsigned* __restrict__ counter, int max_it) {
  if (fl[F_DONE]) return;  // (the same for every block: the counter stays untouched)
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
  const T alpha = static_cast<T>(sc[S_ALPHA]);
  const int64_t begin = c * kChunk;
  const int64_t len = c >= nchunks ? 0 : ((n - begin < kChunk) ? n - begin : kChunk);
  double srr = 0.0, srz = 0.0;
  auto one = [&](int64_t i, T pi, T ai, T vi, T xi, T ri0) {
    x[i] = fma(alpha, pi, xi);
    const T ri = fma(-alpha, ai, ri0);
    r[i] = ri;
    const T zi = vi * ri;
    srr = fma(static_cast<double>(ri), static_cast<double>(ri), srr);
    srz = fma(static_cast<double>(ri), static_cast<double>(zi), srz);
  };
  if (lane < lanes) {
    constexpr int U = kAhead / 2;
    int64_t k = lane;
    for (; k + (U - 1) * lanes < len; k += U * lanes) {
      T pv[U], av[U], vv[U], xv[U], rv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t i = begin + k + u * lanes;
        pv[u] = p[i];
        av[u] = ap[i];
        vv[u] = inv[i];
        xv[u] = x[i];
        rv[u] = r[i];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) one(begin + k + u * lanes, pv[u], av[u], vv[u], xv[u], rv[u]);
    }
    for (; k < len; k += lanes) {
      const int64_t i = begin + k;
      one(i, p[i], ap[i], inv[i], x[i], r[i]);
    }
  }
  double trr = 0.0, trz = 0.0;
  for (int j = 0; j < lanes; ++j) {
    trr += __shfl_sync(0xffffffffu, srr, j);
    trz += __shfl_sync(0xffffffffu, srz, j);
  }
  if (lane == 0 && c < nchunks) {
    out[c] = trr;
    out[nchunks + c] = trz;
  }
  if (!last_block(counter)) return;
  block_levels(out, out2, nchunks, 2, lanes, sc + S_RR);
  if (threadIdx.x == 0) {
    *counter = 0u;
    cg_beta_step(sc, fl, max_it);
  }
}

// k_cg_pap and k_cg_update with a block per chunk (kChunkBlock threads; the grid is the chunks):
// every entry's loads in flight at once, the chunk's sums by one warp from shared memory in the
// same order, so the same bits; used for vectors of at most kBlockChunks chunks.
template <class T>
__global__ void __launch_bounds__(kChunkBlock) k_cg_pap_b(const T* __restrict__ p, const T* __restrict__ ap, int64_t n,
                                                          int lanes, int64_t nchunks, double* __restrict__ out,
                                                          double* __restrict__ out2, unsigned* __restrict__ counter,
                                                          double* __restrict__ sc, int* __restrict__ fl) {
  if (fl[F_DONE]) return;  // (the same for every block: the counter stays untouched)
  __shared__ T sa[kChunk], sb[kChunk];
  const int64_t c = blockIdx.x;
  const int64_t begin = c * kChunk;
  const int len = static_cast<int>((n - begin < kChunk) ? n - begin : kChunk);
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
  if (threadIdx.x < 32) {
    const double total = chunk_fma_sum(sa, sb, len, lanes, static_cast<int>(threadIdx.x));
    if (threadIdx.x == 0) out[c] = total;
  }
  if (!last_block(counter)) return;
  block_levels(out, out2, nchunks, 1, lanes, sc + S_PAP);
  if (threadIdx.x == 0) {
    *counter = 0u;
    cg_alpha_step(sc, fl);
  }
}

template <class T>
__global__ void __launch_bounds__(kChunkBlock) k_cg_update_b(double* __restrict__ sc, int* __restrict__ fl,
                                                             const T* __restrict__ p, const T* __restrict__ ap,
                                                             const T* __restrict__ inv, T* __restrict__ x,
                                                             T* __restrict__ r, int64_t n, int lanes, int64_t nchunks,
                                                             double* __restrict__ out, double* __restrict__ out2,
                                                             unsigned* __restrict__ counter, int max_it) {
  if (fl[F_DONE]) return;  // (the same for every block: the counter stays untouched)
  __shared__ T sr[kChunk], sz[kChunk];
  const T alpha = static_cast<T>(sc[S_ALPHA]);
  const int64_t c = blockIdx.x;
  const int64_t begin = c * kChunk;
  const int len = static_cast<int>((n - begin < kChunk) ? n - begin : kChunk);
  T vp[kChunkPer], vap[kChunkPer], vinv[kChunkPer], vx[kChunkPer], vr[kChunkPer];
#pragma unroll
  for (int k = 0; k < kChunkPer; ++k) {
    const int j = threadIdx.x + k * kChunkBlock;
    if (j < len) {
      const int64_t i = begin + j;
      vp[k] = p[i];
      vap[k] = ap[i];
      vinv[k] = inv[i];
      vx[k] = x[i];
      vr[k] = r[i];
    }
  }
#pragma unroll
  for (int k = 0; k < kChunkPer; ++k) {
    const int j = threadIdx.x + k * kChunkBlock;
    if (j < len) {
      const int64_t i = begin + j;
      x[i] = fma(alpha, vp[k], vx[k]);
      const T ri = fma(-alpha, vap[k], vr[k]);
      r[i] = ri;
      sr[j] = ri;
      sz[j] = vinv[k] * ri;
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = static_cast<int>(threadIdx.x);
    const double trr = chunk_fma_sum(sr, sr, len, lanes, lane);
    const double trz = chunk_fma_sum(sr, sz, len, lanes, lane);
    if (lane == 0) {
      out[c] = trr;
      out[nchunks + c] = trz;
    }
  }
  if (!last_block(counter)) return;
  block_levels(out, out2, nchunks, 2, lanes, sc + S_RR);
  if (threadIdx.x == 0) {
    *counter = 0u;
    cg_beta_step(sc, fl, max_it);
  }
}

template <class T>
__global__ void k_cg_p(const double* __restrict__ sc, const int* __restrict__ fl, const T* __restrict__ inv,
                       const T* __restrict__ r, T* __restrict__ p, int64_t n) {
  if (fl[F_DONE]) return;
  const T beta = static_cast<T>(sc[S_BETA]);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[i] = fma(beta, p[i], inv[i] * r[i]);
}

__global__ void k_cg_start(double* sc, int* fl, double rtol, double atol, int max_it) {
  sc[S_RHS] = sqrt(sc[S_BB]);
  const double rn = sqrt(sc[S_RR]);
  sc[S_RNORM] = rn;
  sc[S_INIT] = rn;
  sc[S_RZ] = sc[S_RZNEW];
  const double tol = rtol * sc[S_RHS];
  sc[S_TOL] = tol > atol ? tol : atol;
  fl[F_ITERS] = 0;
  fl[F_INDEF] = 0;
  fl[F_CONV] = rn <= sc[S_TOL];
  fl[F_DONE] = fl[F_CONV] || max_it <= 0;
}

__device__ void cg_alpha_step(double* sc, int* fl) {
  if (fl[F_DONE]) return;
  const double pap = sc[S_PAP];
  if (!(pap > 0.0)) {
    fl[F_INDEF] = 1;
    fl[F_DONE] = 1;
    return;
  }
  sc[S_ALPHA] = sc[S_RZ] / pap;
}

__device__ void cg_beta_step(double* sc, int* fl, int max_it) {
  if (fl[F_DONE]) return;
  const double rn = sqrt(sc[S_RR]);
  sc[S_RNORM] = rn;
  const int it = ++fl[F_ITERS];
  if (rn <= sc[S_TOL]) {
    fl[F_CONV] = 1;
    fl[F_DONE] = 1;
    return;
  }
  if (it >= max_it) {
    fl[F_DONE] = 1;
    return;
  }
  sc[S_BETA] = sc[S_RZNEW] / sc[S_RZ];
  sc[S_RZ] = sc[S_RZNEW];
}

// CG iterations per pass of the loop graph: fewer condition kernels and body relaunches against
// at most kCgPass - 1 empty iterations after the solve ends.
constexpr int kCgPass = 4;

// The condition of the CG loop graph: another pass while the solve is not done, at most `cap`
// passes (a bound the solve's own max_it already keeps below).
__global__ void k_cg_cond(cudaGraphConditionalHandle h, const int* __restrict__ fl, int* __restrict__ passes, int cap) {
  const int c = ++*passes;
  cudaGraphSetConditional(h, (!fl[F_DONE] && c < cap) ? 1u : 0u);
}

__global__ void k_count_zero(const double* __restrict__ d, int64_t n, int* count) {
  int local = 0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    local += d[i] == 0.0;
  if (local) atomicAdd(count, local);
}

template <class T>
__global__ void k_reciprocal_t(const double* __restrict__ d, T* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = static_cast<T>(1.0 / d[i]);
}

// IR helpers: r64 = b - ax (FP64), r32 = (float) r64, x += (double) d32
__global__ void k_residual64(const double* __restrict__ b, const double* __restrict__ ax, double* __restrict__ r,
                             int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    r[i] = b[i] - ax[i];
}
// r = b - f - ma
__global__ void k_dyn_residual(const double* __restrict__ b, const double* __restrict__ ma, double* __restrict__ r,
                               int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    r[i] = b[i] - r[i] - ma[i];
}
__global__ void k_mul(const double* __restrict__ d, const double* __restrict__ x, double* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = d[i] * x[i];
}
// y = b - y
__global__ void k_sub_from(const double* __restrict__ b, double* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = b[i] - y[i];
}
__global__ void k_add64(const double* __restrict__ d, double* __restrict__ x, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] += d[i];
}
__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    b[i] = static_cast<float>(a[i]);
}
__global__ void k_add_f32(const float* __restrict__ d, double* __restrict__ x, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] += static_cast<double>(d[i]);
}
__global__ void k_zero_f32(float* __restrict__ x, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] = 0.f;
}

unsigned ew(int64_t n) {
  const int64_t blocks = (n + 255) / 256;
  const int64_t cap = static_cast<int64_t>(num_sms()) * 8;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min(blocks, cap)));
}
unsigned chunk_grid(int64_t nchunks) { return static_cast<unsigned>((nchunks + kWarps - 1) / kWarps); }

}  // namespace

// ------------------------------------------------------------------ the solver object
struct Solver {
  fx_force* f = nullptr;
  int method = FX_SOLVER_CG;
  fx_solve_opts o{};
  double inner_rtol = 1e-4;
  double k[3] = {1, 0, 0};
  bool ready = false;
  int64_t n = 0;
  cudaStream_t cs = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  ReduceWork w;
  DeviceArray<double> diag, inv, r, p, ap, x0;
  DeviceArray<float> inv32, r32, p32, ap32, d32;
  DeviceArray<double> sc;
  DeviceArray<int> fl;
  DeviceArray<int> zero_count;
  DeviceArray<int> passes;  // the CG loop graph's pass counter
  DeviceArray<unsigned> counter;  // the fused kernels' last-block counter (0 between launches)
  DeviceArray<double> V, Z, wv, hbuf;  // GMRES
  DeviceArray<double> nres, ndu;       // Newton: residual and increment
  DeviceArray<double> nut, nvt, nat;   // Newmark: the last step's u, v, a
  DeviceArray<double> cu, cv, ca, fx_t;  // recovery: the committed u, v, a of an attempt; its load
  DeviceArray<double> ct_j2, ct_pimy, ct_pdmy;  // recovery: the points' tangents before an attempt
  int* host_flags = nullptr;           // pinned
  double* host_sc = nullptr;           // pinned
  // The CG loop graph of the last solve per precision (0: FP64, 1: FP32 inner), kept for the next
  // solve on the same vectors (the Newton and Newmark loops, refinement rounds): capturing and
  // instantiating it costs as much as several iterations. Dropped when setup changes the
  // coefficients (the layered tables are kernel parameters captured with it).
  struct CgGraph {
    cudaGraphExec_t exec = nullptr;
    const void* key[5] = {};
    int max_it = 0;
  } cg_graph[2];
  void drop_graphs() {
    for (auto& g : cg_graph) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g = CgGraph{};
    }
  }
  ~Solver() {
    drop_graphs();
    if (cs) cudaStreamDestroy(cs);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (host_flags) cudaFreeHost(host_flags);
    if (host_sc) cudaFreeHost(host_sc);
  }

  void apply64(const double* x, double* y, const int* skip) {
    if (f->s.use_box()) box_apply(f->s, k, x, y, cs, skip);
    else general_apply(f->s, k, x, y, cs, skip);
  }
  void apply32(const float* x, float* y, const int* skip) {
    if (f->s.use_box()) box_apply_f32(f->s, k, x, y, cs, skip);
    else general_apply_f32(f->s, k, x, y, cs, skip);
  }

  void read_state() {
    FX_CUDA(cudaMemcpyAsync(host_flags, fl.ptr, sizeof(int) * F_NFLAG, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaMemcpyAsync(host_sc, sc.ptr, sizeof(double) * S_NSCALAR, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
  }

  // Jacobi-PCG on vectors of type T (double: the plain solve; float: the inner solve of IR).
  template <class T>
  void cg(const T* b, T* x, T* rr, T* pp, T* aa, const T* iv, double rtol, double atol, int max_it, fx_solve_result* res) {
    const int lanes = o.lanes;
    const int64_t nc = chunks_of(n);
    auto apply = [&](const T* xin, T* yout, const int* skip) {
      if constexpr (sizeof(T) == 8) apply64(xin, yout, skip);
      else apply32(xin, yout, skip);
    };
    // b.b, r = b - A x, r.r, r.z, p = z
    k_dot_chunks<T><<<chunk_grid(nc), 32 * kWarps, 0, cs>>>(b, b, n, lanes, nc, w.level[0].ptr);
    FX_LAUNCH_CHECK("cg_bb");
    reduce_partials(w, nc, 1, sc.ptr + S_BB, cs);
    apply(x, aa, nullptr);
    k_cg_begin<T><<<chunk_grid(nc), 32 * kWarps, 0, cs>>>(b, aa, iv, rr, pp, n, lanes, nc, w.level[0].ptr);
    FX_LAUNCH_CHECK("cg_begin");
    reduce_partials(w, nc, 2, sc.ptr + S_RR, cs);
    k_cg_start<<<1, 1, 0, cs>>>(sc.ptr, fl.ptr, rtol, atol, max_it);
    FX_LAUNCH_CHECK("cg_start");
    auto iteration = [&] {
      apply(pp, aa, fl.ptr + F_DONE);
      // p.Ap and alpha, then the update, r.r, r.z and beta (each with its levels in the kernel's
      // last block), then p
      if (nc <= kBlockChunks) {
        k_cg_pap_b<T><<<static_cast<unsigned>(nc), kChunkBlock, 0, cs>>>(pp, aa, n, lanes, nc, w.level[0].ptr,
                                                                         w.level[1].ptr, counter.ptr, sc.ptr, fl.ptr);
        k_cg_update_b<T><<<static_cast<unsigned>(nc), kChunkBlock, 0, cs>>>(sc.ptr, fl.ptr, pp, aa, iv, x, rr, n,
                                                                            lanes, nc, w.level[0].ptr, w.level[1].ptr,
                                                                            counter.ptr, max_it);
      } else {
        k_cg_pap<T><<<chunk_grid(nc), 32 * kWarps, 0, cs>>>(pp, aa, n, lanes, nc, w.level[0].ptr, w.level[1].ptr,
                                                           counter.ptr, sc.ptr, fl.ptr);
        k_cg_update<T><<<chunk_grid(nc), 32 * kWarps, 0, cs>>>(sc.ptr, fl.ptr, pp, aa, iv, x, rr, n, lanes, nc,
                                                              w.level[0].ptr, w.level[1].ptr, counter.ptr, max_it);
      }
      k_cg_p<T><<<ew(n), 256, 0, cs>>>(sc.ptr, fl.ptr, iv, rr, pp, n);
      FX_LAUNCH_CHECK("cg_iteration");
    };
    // The iterations run as one graph: a while node whose body is kCgPass iterations and the
    // condition kernel, so the device loops until the solve is done with no host round trip.
    // The begin above ran eagerly (its apply builds lazy state and this solver's coefficient
    // tables); a new graph is captured when the vectors differ from the last solve's.
    CgGraph& G = cg_graph[sizeof(T) == 4 ? 1 : 0];
    const void* key[5] = {x, rr, pp, aa, iv};
    if (G.exec && (std::memcmp(G.key, key, sizeof key) != 0 || G.max_it != max_it)) {
      cudaGraphExecDestroy(G.exec);
      G = CgGraph{};
    }
    if (!G.exec) {
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
          // kCgPass iterations per pass (every kernel of an iteration skips once the solve is
          // done, so the iterations of a pass after the one that ends the solve are empty)
          for (int i = 0; i < kCgPass; ++i) iteration();
          k_cg_cond<<<1, 1, 0, cs>>>(h, fl.ptr, passes.ptr, (max_it + kCgPass - 1) / kCgPass + 2);
          FX_LAUNCH_CHECK("cg_condition");
        } catch (...) {
          cudaStreamEndCapture(cs, &body);
          throw;
        }
        FX_CUDA(cudaStreamEndCapture(cs, &body));
        FX_CUDA(cudaGraphInstantiate(&G.exec, g, 0));
      } catch (...) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        G = CgGraph{};
        cudaGraphDestroy(g);
        throw;
      }
      cudaGraphDestroy(g);
      std::memcpy(G.key, key, sizeof key);
      G.max_it = max_it;
    }
    FX_CUDA(cudaMemsetAsync(passes.ptr, 0, sizeof(int), cs));
    FX_CUDA(cudaGraphLaunch(G.exec, cs));
    read_state();
    res->converged = host_flags[F_CONV];
    res->iterations = host_flags[F_ITERS];
    res->indefinite = host_flags[F_INDEF];
    res->rhs_norm = host_sc[S_RHS];
    res->initial_residual = host_sc[S_INIT];
    res->final_residual = host_sc[S_RNORM];
  }

  void gmres(const double* b, double* x, fx_solve_result* res);
  void ir(const double* b, double* x, fx_solve_result* res);
  int newton(const double* fext, double* u, int test, double tol, int max_newton, fx_solve_result* res);
  void setup_coefficients(const double kk[3], bool initial, cudaStream_t st);
  struct Recovery {
    int max_retries = 0, num_sublevels = 0, num_substeps = 2;
    int attempts = 0, failed = 0, retries = 0, substepped = 0, newton = 0;
  };
  bool newmark_recover(const double* fext0, const double* fext1, double* u, double* v, double* a, double h,
                       double beta, double gamma, int test, double tol, int max_newton, Recovery& rc,
                       fx_solve_result* res);
  bool newton_recover(const double* fext, double* u, int test, double tol, int max_newton, Recovery& rc,
                      fx_solve_result* res);
  int newmark(const double* fext, double* u, double* v, double* a, double h, double beta, double gamma, int test,
              double tol, int max_newton, fx_solve_result* res);
};

// FGMRES(m) with CGS2, host-side Hessenberg and Givens rotations, as gmres.cpp:32-123.
void Solver::gmres(const double* b, double* x, fx_solve_result* res) {
  const int m = std::max(1, std::min(o.restart, 63));
  const int64_t ld = n;
  std::vector<double> H(static_cast<size_t>((m + 1) * m)), cs_(m), sn(m), g(m + 1), h(m + 1), h2(m + 1), y(m);
  auto Hij = [&](int i, int j) -> double& { return H[static_cast<size_t>(j * (m + 1) + i)]; };
  auto dot_host = [&](const double* a, const double* c) {
    dot_device(w, a, c, n, sc.ptr + S_PAP, cs);
    FX_CUDA(cudaMemcpyAsync(host_sc, sc.ptr + S_PAP, sizeof(double), cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
    return host_sc[0];
  };
  auto dots_host = [&](int kk, const double* wvec, std::vector<double>& out) {
    multi_dot_device(w, V.ptr, ld, kk, wvec, n, hbuf.ptr, cs);
    FX_CUDA(cudaMemcpyAsync(out.data(), hbuf.ptr, sizeof(double) * kk, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
  };
  auto combine = [&](const double* M, int kk, const std::vector<double>& coef, double a, double* wvec) {
    for (int c = 0; c < kk; ++c) axpy(a * coef[c], M + static_cast<int64_t>(c) * ld, wvec, n, cs);
  };
  res->rhs_norm = std::sqrt(dot_host(b, b));
  const double tol = std::max(o.rtol * res->rhs_norm, o.atol);
  bool first = true;
  int iterations = 0;
  for (;;) {
    apply64(x, wv.ptr, nullptr);
    FX_CUDA(cudaMemcpyAsync(r.ptr, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, cs));
    axpy(-1.0, wv.ptr, r.ptr, n, cs);
    const double beta = std::sqrt(dot_host(r.ptr, r.ptr));
    if (first) res->initial_residual = beta;
    first = false;
    res->final_residual = beta;
    if (beta <= tol) {
      res->converged = 1;
      break;
    }
    if (iterations >= o.max_iterations) break;
    fill(V.ptr, 0.0, n, cs);
    axpy(1.0 / beta, r.ptr, V.ptr, n, cs);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    for (; j < m && iterations < o.max_iterations; ++j) {
      double* vj = V.ptr + static_cast<int64_t>(j) * ld;
      double* zj = Z.ptr + static_cast<int64_t>(j) * ld;
      multiply(inv.ptr, vj, zj, n, cs);
      apply64(zj, wv.ptr, nullptr);
      dots_host(j + 1, wv.ptr, h);
      combine(V.ptr, j + 1, h, -1.0, wv.ptr);
      dots_host(j + 1, wv.ptr, h2);
      combine(V.ptr, j + 1, h2, -1.0, wv.ptr);
      for (int i = 0; i <= j; ++i) Hij(i, j) = h[i] + h2[i];
      const double hn = std::sqrt(dot_host(wv.ptr, wv.ptr));
      Hij(j + 1, j) = hn;
      if (hn > 0.0) {
        double* vn = V.ptr + static_cast<int64_t>(j + 1) * ld;
        fill(vn, 0.0, n, cs);
        axpy(1.0 / hn, wv.ptr, vn, n, cs);
      }
      for (int i = 0; i < j; ++i) {
        const double a = Hij(i, j), c = Hij(i + 1, j);
        Hij(i, j) = cs_[i] * a + sn[i] * c;
        Hij(i + 1, j) = -sn[i] * a + cs_[i] * c;
      }
      const double a = Hij(j, j), c = Hij(j + 1, j);
      const double d = std::hypot(a, c);
      cs_[j] = d > 0.0 ? a / d : 1.0;
      sn[j] = d > 0.0 ? c / d : 0.0;
      Hij(j, j) = d;
      Hij(j + 1, j) = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs_[j] * g[j];
      ++iterations;
      res->final_residual = std::abs(g[j + 1]);
      if (res->final_residual <= tol || hn == 0.0) {
        ++j;
        break;
      }
    }
    for (int i = j - 1; i >= 0; --i) {
      double s = g[i];
      for (int kk = i + 1; kk < j; ++kk) s -= Hij(i, kk) * y[kk];
      y[i] = s / Hij(i, i);
    }
    combine(Z.ptr, j, y, 1.0, x);
    if (res->final_residual <= tol) {
      apply64(x, wv.ptr, nullptr);
      FX_CUDA(cudaMemcpyAsync(r.ptr, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, cs));
      axpy(-1.0, wv.ptr, r.ptr, n, cs);
      res->final_residual = std::sqrt(dot_host(r.ptr, r.ptr));
      if (res->final_residual <= tol) {
        res->converged = 1;
        break;
      }
    }
    if (iterations >= o.max_iterations) break;
  }
  res->iterations = iterations;
}

// FP32 PCG inside FP64 iterative refinement.
void Solver::ir(const double* b, double* x, fx_solve_result* res) {
  res->rhs_norm = -1.0;
  int outer = 0, inner_total = 0;
  double bnorm = 0.0, prev = 0.0;
  const int max_outer = 50;
  for (;;) {
    apply64(x, ap.ptr, nullptr);
    k_residual64<<<ew(n), 256, 0, cs>>>(b, ap.ptr, r.ptr, n);
    FX_LAUNCH_CHECK("ir_residual");
    if (outer == 0) {
      dot_device(w, b, b, n, sc.ptr + S_BB, cs);
    }
    dot_device(w, r.ptr, r.ptr, n, sc.ptr + S_RR, cs);
    FX_CUDA(cudaMemcpyAsync(host_sc, sc.ptr, sizeof(double) * S_NSCALAR, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
    if (outer == 0) {
      bnorm = std::sqrt(host_sc[S_BB]);
      res->rhs_norm = bnorm;
    }
    const double rn = std::sqrt(host_sc[S_RR]);
    if (outer == 0) res->initial_residual = rn;
    res->final_residual = rn;
    if (rn <= std::max(o.rtol * bnorm, o.atol)) {
      res->converged = 1;
      break;
    }
    // a round that did not halve the FP64 residual: it has reached what FP64 resolves for this
    // operator (the FP32 corrections now only move rounding), so more rounds gain nothing
    if (outer > 0 && rn > kIrStall * prev) break;
    prev = rn;
    if (outer >= max_outer || inner_total >= o.max_iterations) break;
    // inner: K d = r in FP32 from d = 0
    k_to_f32<<<ew(n), 256, 0, cs>>>(r.ptr, r32.ptr, n);
    k_zero_f32<<<ew(n), 256, 0, cs>>>(d32.ptr, n);
    FX_LAUNCH_CHECK("ir_inner_setup");
    fx_solve_result ri{};
    // the FP32 rhs lives in r32; the CG residual vector needs its own buffer: reuse x0 as FP32 storage
    float* rr32 = reinterpret_cast<float*>(x0.ptr);
    cg<float>(r32.ptr, d32.ptr, rr32, p32.ptr, ap32.ptr, inv32.ptr, inner_rtol, 0.0, o.max_iterations - inner_total, &ri);
    inner_total += ri.iterations;
    k_add_f32<<<ew(n), 256, 0, cs>>>(d32.ptr, x, n);
    FX_LAUNCH_CHECK("ir_correct");
    ++outer;
    if (ri.iterations == 0 && !ri.converged) break;
  }
  res->iterations = inner_total;
  res->refinements = outer;
}

// Newton iterations of one quasi-static load step (ImplicitStage's Newton loop without inertia,
// src/exec/implicit_stage.cpp:118-437): r = f_ext - f_int(u) with the material update of every
// point (which also stores the points' consistent tangents), the Jacobi diagonal of that
// tangent, K_t du = r by CG from du = 0, u += du; the convergence test is the stage's
// (implicit_stage.cpp:199, 241-242, 342): NormUnbalance ||r|| <= tol or NormDispIncr
// ||du|| <= tol, absolute. After a NormDispIncr convergence the force is evaluated once more at
// the final u, so that the trial material state is u's. The trial state is left for the caller
// to commit. Returns the Newton iterations (solves); res: converged, CG iterations in all,
// ||f_ext||, the first and last ||r||.
int Solver::newton(const double* fext, double* u, int test, double tol, int max_newton, fx_solve_result* res) {
  ForceState& fs = f->s;
  FX_CUDA(cudaMemsetAsync(x0.ptr, 0, sizeof(double) * n, cs));  // velocity 0 (quasi-static)
  auto norm = [&](const double* v) {
    dot_device(w, v, v, n, sc.ptr + S_RR, cs);
    FX_CUDA(cudaMemcpyAsync(host_sc, sc.ptr, sizeof(double) * S_NSCALAR, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
    return std::sqrt(host_sc[S_RR]);
  };
  auto residual = [&]() {  // nres = f_ext - f_int(u)
    if (fs.use_box_force()) box_force(fs, u, x0.ptr, nres.ptr, cs);
    else general_force(fs, u, x0.ptr, nres.ptr, cs);
    k_sub_from<<<ew(n), 256, 0, cs>>>(fext, nres.ptr, n);
    FX_LAUNCH_CHECK("newton_residual");
    return norm(nres.ptr);
  };
  res->rhs_norm = norm(fext);
  int it = 0;
  double rn = residual();
  res->initial_residual = rn;
  for (;;) {
    res->final_residual = rn;
    if (test == FX_TEST_NORM_UNBALANCE && rn <= tol) {
      res->converged = 1;
      break;
    }
    if (it >= max_newton) break;
    general_diagonal(fs, k, diag.ptr, cs);
    k_reciprocal_t<double><<<ew(n), 256, 0, cs>>>(diag.ptr, inv.ptr, n);
    if (method == FX_SOLVER_IR) k_reciprocal_t<float><<<ew(n), 256, 0, cs>>>(diag.ptr, inv32.ptr, n);
    FX_CUDA(cudaMemsetAsync(ndu.ptr, 0, sizeof(double) * n, cs));
    fx_solve_result lin{};
    if (method == FX_SOLVER_IR) ir(nres.ptr, ndu.ptr, &lin);  // FP32 CG on the tangent, FP64 refinement
    else cg<double>(nres.ptr, ndu.ptr, r.ptr, p.ptr, ap.ptr, inv.ptr, o.rtol, o.atol, o.max_iterations, &lin);
    k_add64<<<ew(n), 256, 0, cs>>>(ndu.ptr, u, n);
    FX_LAUNCH_CHECK("newton_update");
    res->iterations += lin.iterations;
    res->refinements += lin.refinements;
    res->indefinite |= lin.indefinite;
    ++it;
    const double dn = test == FX_TEST_NORM_DISP_INCR ? norm(ndu.ptr) : 0.0;
    rn = residual();
    if (test == FX_TEST_NORM_DISP_INCR && dn <= tol) {
      res->final_residual = rn;
      res->converged = 1;
      break;
    }
  }
  return it;
}

// One Newmark time step (Newmark::newStep with displ == 1 and ImplicitStage's Newton loop with
// inertia, src/exec/implicit_stage.cpp:29-68, 118-437): predict (v = a1 v + a2 a, a = a4 a + a3 v
// of the last step; u kept), then Newton: r = f_ext - f_int(u, v) - M a, K_eff du = r by the
// solver's method (plain FP64 CG, or FP32 CG inside FP64 refinement), u += du, v += c2 du,
// a += c3 du, with K_eff = K + c2 C + c3 M, c2 = gamma / (beta h), c3 = 1 / (beta h^2): the
// coefficients the solver must be set up with. M a is the lumped masses times a when every set
// is lumped, else the mass operator of the general path. Tests as newton().
int Solver::newmark(const double* fext, double* u, double* v, double* a, double h, double beta, double gamma,
                    int test, double tol, int max_newton, fx_solve_result* res) {
  ForceState& fs = f->s;
  const double c2 = gamma / (beta * h), c3 = 1.0 / (beta * h * h);
  if (k[0] != 1.0 || k[1] != c2 || k[2] != c3)
    throw Error(FX_E_INVALID, "newmark: set the solver up with the coefficients (1, gamma/(beta h), 1/(beta h^2))");
  const double a1 = 1.0 - gamma / beta, a2 = h * (1.0 - 0.5 * gamma / beta), a3 = -1.0 / (beta * h),
               a4 = 1.0 - 0.5 / beta;
  newmark_predict(n, u, v, a, nut.ptr, nvt.ptr, nat.ptr, a1, a2, a3, a4, cs);
  bool all_lumped = fs.lumped_mass.n > 0;
  for (const auto& q : fs.params_h) all_lumped = all_lumped && q.mass_type == 1;
  auto norm = [&](const double* x) {
    dot_device(w, x, x, n, sc.ptr + S_RR, cs);
    FX_CUDA(cudaMemcpyAsync(host_sc, sc.ptr, sizeof(double) * S_NSCALAR, cudaMemcpyDeviceToHost, cs));
    FX_CUDA(cudaStreamSynchronize(cs));
    return std::sqrt(host_sc[S_RR]);
  };
  auto residual = [&]() {  // nres = f_ext - f_int(u, v) - M a
    if (fs.use_box_force()) box_force(fs, u, v, nres.ptr, cs);
    else general_force(fs, u, v, nres.ptr, cs);
    if (all_lumped) {
      k_mul<<<ew(n), 256, 0, cs>>>(fs.lumped_mass.ptr, a, nut.ptr, n);  // nut is free after the predict
    } else if (fs.use_box()) {
      box_mass_apply(fs, a, nut.ptr, cs);
    } else {
      const double km[3] = {0.0, 0.0, 1.0};
      const bool init = fs.initial;
      general_apply(fs, km, a, nut.ptr, cs);
      fs.initial = init;
    }
    k_dyn_residual<<<ew(n), 256, 0, cs>>>(fext, nut.ptr, nres.ptr, n);
    FX_LAUNCH_CHECK("newmark_residual");
    return norm(nres.ptr);
  };
  res->rhs_norm = norm(fext);
  int it = 0;
  double rn = residual();
  res->initial_residual = rn;
  for (;;) {
    res->final_residual = rn;
    if (test == FX_TEST_NORM_UNBALANCE && rn <= tol) {
      res->converged = 1;
      break;
    }
    if (it >= max_newton) break;
    FX_CUDA(cudaMemsetAsync(ndu.ptr, 0, sizeof(double) * n, cs));
    fx_solve_result lin{};
    if (method == FX_SOLVER_IR) ir(nres.ptr, ndu.ptr, &lin);
    else cg<double>(nres.ptr, ndu.ptr, r.ptr, p.ptr, ap.ptr, inv.ptr, o.rtol, o.atol, o.max_iterations, &lin);
    newmark_update(n, ndu.ptr, u, v, a, c2, c3, cs);
    res->iterations += lin.iterations;
    res->refinements += lin.refinements;
    res->indefinite |= lin.indefinite;
    ++it;
    const double dn = test == FX_TEST_NORM_DISP_INCR ? norm(ndu.ptr) : 0.0;
    rn = residual();
    if (test == FX_TEST_NORM_DISP_INCR && dn <= tol) {
      res->final_residual = rn;
      res->converged = 1;
      break;
    }
  }
  return it;
}

// The Jacobi preconditioner and the operator tables for coefficients kk (fx_solver_setup).
void Solver::setup_coefficients(const double kk[3], bool initial, cudaStream_t st) {
  drop_graphs();
  k[0] = kk[0];
  k[1] = kk[1];
  k[2] = kk[2];
  f->s.initial = initial;
  if (n == 0) return;
  general_diagonal(f->s, k, diag.ptr, st);
  FX_CUDA(cudaMemsetAsync(zero_count.ptr, 0, sizeof(int), st));
  k_count_zero<<<ew(n), 256, 0, st>>>(diag.ptr, n, zero_count.ptr);
  int zeros = 0;
  FX_CUDA(cudaMemcpyAsync(&zeros, zero_count.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  FX_CUDA(cudaStreamSynchronize(st));
  if (zeros > 0) throw Error(FX_E_INVALID, "Jacobi: " + std::to_string(zeros) + " zero diagonal entries");
  k_reciprocal_t<double><<<ew(n), 256, 0, st>>>(diag.ptr, inv.ptr, n);
  if (method == FX_SOLVER_IR) k_reciprocal_t<float><<<ew(n), 256, 0, st>>>(diag.ptr, inv32.ptr, n);
  FX_LAUNCH_CHECK("jacobi_setup");
  if (f->s.use_box()) box_prepare(f->s, k);
  FX_CUDA(cudaStreamSynchronize(st));
}

namespace {
__global__ void k_lerp(const double* __restrict__ a, const double* __restrict__ b, double t, double* __restrict__ out,
                       int64_t n) {
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[q] = t == 1.0 ? b[q] : a[q] + t * (b[q] - a[q]);
}
void commit_materials(ForceState& fs, cudaStream_t st) {  // Domain::commit
  if (fs.has_j2)
    FX_CUDA(cudaMemcpyAsync(fs.j2_committed.ptr, fs.j2_trial.ptr, fs.j2_committed.bytes(), cudaMemcpyDeviceToDevice, st));
  pimy_commit(fs, st);
}
}  // namespace

// Femora's retry and substep recovery around one Newmark step (implicit_stage.cpp:261-402): an
// attempt that does not converge goes back to the committed state (u, v, a and the points'
// tangents; the materials' trial state is rebuilt from their committed one by the next force
// evaluation) and is retried at the
// same size up to max_retries times; then, below num_sublevels, the step is split into
// num_substeps steps one level down, each with the same recovery. Every converged attempt commits
// the materials (Domain::commit). The load of an attempt ending at the fraction theta of the step
// is fext0 + theta (fext1 - fext0). The solver is set up for each attempt's size and back for h.
bool Solver::newmark_recover(const double* fext0, const double* fext1, double* u, double* v, double* a, double h,
                             double beta, double gamma, int test, double tol, int max_newton, Recovery& rc,
                             fx_solve_result* res) {
  const size_t nn = static_cast<size_t>(n);
  if (cu.n < nn) {
    cu.alloc(nn);
    cv.alloc(nn);
    ca.alloc(nn);
    fx_t.alloc(nn);
  }
  const double k0[3] = {k[0], k[1], k[2]};
  const bool init0 = f->s.initial;
  const size_t bytes = sizeof(double) * nn;
  // The points' tangents of the last force evaluation feed the Jacobi preconditioner set up for an
  // attempt's size: a failed attempt gives them back with u, v, a, so that every attempt starts
  // from the state the step started from.
  ForceState& fs = f->s;
  std::pair<DeviceArray<double>*, DeviceArray<double>*> tangents[3] = {
      {&fs.j2_tan, &ct_j2}, {&fs.pimy_tan, &ct_pimy}, {&fs.pdmy_tan, &ct_pdmy}};
  for (auto& t : tangents)
    if (t.first->n > 0 && t.second->n != t.first->n) t.second->alloc(t.first->n);
  auto keep = [&](bool restore) {
    for (auto& t : tangents)
      if (t.first->n > 0)
        FX_CUDA(cudaMemcpyAsync(restore ? t.first->ptr : t.second->ptr, restore ? t.second->ptr : t.first->ptr,
                                t.first->bytes(), cudaMemcpyDeviceToDevice, cs));
  };
  double theta = 0.0;
  auto attempt = [&](double hs) -> bool {
    ++rc.attempts;
    FX_CUDA(cudaMemcpyAsync(cu.ptr, u, bytes, cudaMemcpyDeviceToDevice, cs));
    FX_CUDA(cudaMemcpyAsync(cv.ptr, v, bytes, cudaMemcpyDeviceToDevice, cs));
    FX_CUDA(cudaMemcpyAsync(ca.ptr, a, bytes, cudaMemcpyDeviceToDevice, cs));
    keep(false);
    const double end = hs == h ? 1.0 : std::min(1.0, theta + hs / h);
    k_lerp<<<ew(n), 256, 0, cs>>>(fext0 ? fext0 : fext1, fext1, end, fx_t.ptr, n);
    FX_LAUNCH_CHECK("recovery_load");
    const double kk[3] = {1.0, gamma / (beta * hs), 1.0 / (beta * hs * hs)};
    if (kk[0] != k[0] || kk[1] != k[1] || kk[2] != k[2]) setup_coefficients(kk, init0, cs);
    fx_solve_result one{};
    rc.newton += newmark(fx_t.ptr, u, v, a, hs, beta, gamma, test, tol, max_newton, &one);
    res->iterations += one.iterations;
    res->refinements += one.refinements;
    res->indefinite |= one.indefinite;
    res->rhs_norm = one.rhs_norm;
    res->initial_residual = one.initial_residual;
    res->final_residual = one.final_residual;
    if (one.converged) {
      commit_materials(f->s, cs);
      theta = end;
      return true;
    }
    ++rc.failed;
    FX_CUDA(cudaMemcpyAsync(u, cu.ptr, bytes, cudaMemcpyDeviceToDevice, cs));
    FX_CUDA(cudaMemcpyAsync(v, cv.ptr, bytes, cudaMemcpyDeviceToDevice, cs));
    FX_CUDA(cudaMemcpyAsync(a, ca.ptr, bytes, cudaMemcpyDeviceToDevice, cs));
    keep(true);
    return false;
  };
  std::function<bool(double, int)> recover = [&](double hs, int level) -> bool {
    if (attempt(hs)) return true;
    for (int r = 1; r <= rc.max_retries; ++r) {
      ++rc.retries;
      if (attempt(hs)) return true;
    }
    if (level >= rc.num_sublevels) return false;
    ++rc.substepped;
    const double sub = hs / static_cast<double>(rc.num_substeps);
    for (int i = 0; i < rc.num_substeps; ++i)
      if (!recover(sub, level + 1)) return false;
    return true;
  };
  const bool ok = recover(h, 0);
  if (k[0] != k0[0] || k[1] != k0[1] || k[2] != k0[2]) setup_coefficients(k0, init0, cs);
  res->converged = ok ? 1 : 0;
  return ok;
}

// The same recovery for a quasi-static load step: a failed step returns to the committed
// displacement and is retried, up to max_retries times (static stages retry only,
// implicit_stage.cpp:263-266); a converged one commits the materials.
bool Solver::newton_recover(const double* fext, double* u, int test, double tol, int max_newton, Recovery& rc,
                            fx_solve_result* res) {
  const size_t nn = static_cast<size_t>(n);
  if (cu.n < nn) {
    cu.alloc(nn);
    cv.alloc(nn);
    ca.alloc(nn);
    fx_t.alloc(nn);
  }
  const size_t bytes = sizeof(double) * nn;
  for (int r = 0; r <= rc.max_retries; ++r) {
    if (r > 0) ++rc.retries;
    ++rc.attempts;
    FX_CUDA(cudaMemcpyAsync(cu.ptr, u, bytes, cudaMemcpyDeviceToDevice, cs));
    fx_solve_result one{};
    rc.newton += newton(fext, u, test, tol, max_newton, &one);
    res->iterations += one.iterations;
    res->refinements += one.refinements;
    res->indefinite |= one.indefinite;
    res->rhs_norm = one.rhs_norm;
    res->initial_residual = one.initial_residual;
    res->final_residual = one.final_residual;
    if (one.converged) {
      commit_materials(f->s, cs);
      res->converged = 1;
      return true;
    }
    ++rc.failed;
    FX_CUDA(cudaMemcpyAsync(u, cu.ptr, bytes, cudaMemcpyDeviceToDevice, cs));
  }
  res->converged = 0;
  return false;
}

}  // namespace fx

struct fx_solver {
  fx::Solver s;
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

int fx_solver_create(fx_force* f, int32_t method, fx_solve_opts o, fx_solver** out) {
  return guard([&] {
    if (!f || !out) throw fx::Error(FX_E_INVALID, "fx_solver_create: bad arguments");
    if (method < FX_SOLVER_CG || method > FX_SOLVER_IR) throw fx::Error(FX_E_INVALID, "fx_solver_create: unknown method");
    if (o.lanes <= 0) o.lanes = 32;
    if (o.lanes > 32) throw fx::Error(FX_E_INVALID, "lanes must be in 1..32");
    if (o.restart <= 0) o.restart = 30;
    if (o.max_iterations < 0) throw fx::Error(FX_E_INVALID, "max_iterations must be >= 0");
    FX_CUDA(cudaSetDevice(f->s.device));
    auto* h = new fx_solver;
    fx::Solver& s = h->s;
    try {
      s.f = f;
      s.method = method;
      s.o = o;
      s.n = f->s.neq;
      const size_t n = static_cast<size_t>(std::max<int64_t>(s.n, 1));
      FX_CUDA(cudaStreamCreateWithFlags(&s.cs, cudaStreamNonBlocking));
      FX_CUDA(cudaEventCreateWithFlags(&s.ev_in, cudaEventDisableTiming));
      FX_CUDA(cudaEventCreateWithFlags(&s.ev_out, cudaEventDisableTiming));
      FX_CUDA(cudaMallocHost(&s.host_flags, sizeof(int) * F_NFLAG));
      FX_CUDA(cudaMallocHost(&s.host_sc, sizeof(double) * S_NSCALAR));
      s.w.init(std::max<int64_t>(s.n, 1), o.lanes);
      s.diag.alloc(n);
      s.inv.alloc(n);
      s.r.alloc(n);
      s.p.alloc(n);
      s.ap.alloc(n);
      s.x0.alloc(n);
      s.sc.alloc(S_NSCALAR);
      s.fl.alloc(F_NFLAG);
      s.zero_count.alloc(1);
      s.passes.alloc(1);
      s.counter.alloc(1);
      FX_CUDA(cudaMemset(s.counter.ptr, 0, sizeof(unsigned)));
      s.hbuf.alloc(64);
      s.nres.alloc(n);
      s.ndu.alloc(n);
      s.nut.alloc(n);
      s.nvt.alloc(n);
      s.nat.alloc(n);
      if (method == FX_SOLVER_GMRES || method == FX_SOLVER_KRYLOV) {
        const int m = std::max(1, std::min(o.restart, 63));
        s.V.alloc(n * static_cast<size_t>(m + 1));
        s.Z.alloc(n * static_cast<size_t>(m));
        s.wv.alloc(n);
      }
      if (method == FX_SOLVER_IR) {
        s.inv32.alloc(n);
        s.r32.alloc(n);
        s.p32.alloc(n);
        s.ap32.alloc(n);
        s.d32.alloc(n);
      }
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

void fx_solver_destroy(fx_solver* s) { delete s; }

int fx_solver_set_inner_tolerance(fx_solver* s, double inner_rtol) {
  return guard([&] {
    if (!s || !(inner_rtol > 0.0 && inner_rtol < 1.0)) throw fx::Error(FX_E_INVALID, "inner tolerance must be in (0, 1)");
    s->s.inner_rtol = inner_rtol;
  });
}

int fx_solver_setup(fx_solver* h, fx_coeffs k, void* stream) {
  return guard([&] {
    if (!h) throw fx::Error(FX_E_INVALID, "fx_solver_setup: null handle");
    fx::Solver& s = h->s;
    const double kk[3] = {k.stiffness, k.damping, k.mass};
    s.setup_coefficients(kk, k.initial != 0, static_cast<cudaStream_t>(stream));
    s.ready = true;
  });
}

int fx_solver_solve(fx_solver* h, const double* b, double* x, fx_solve_result* r, void* stream) {
  return guard([&] {
    if (!h || !r || (h->s.n > 0 && (!b || !x))) throw fx::Error(FX_E_INVALID, "fx_solver_solve: bad arguments");
    fx::Solver& s = h->s;
    if (!s.ready) throw fx::Error(FX_E_INVALID, "fx_solver_solve: call fx_solver_setup first");
    *r = fx_solve_result{};
    if (s.n == 0) {
      r->converged = 1;
      return;
    }
    auto st = static_cast<cudaStream_t>(stream);
    FX_CUDA(cudaEventRecord(s.ev_in, st));
    FX_CUDA(cudaStreamWaitEvent(s.cs, s.ev_in, 0));
    switch (s.method) {
      case FX_SOLVER_CG:
        s.cg<double>(b, x, s.r.ptr, s.p.ptr, s.ap.ptr, s.inv.ptr, s.o.rtol, s.o.atol, s.o.max_iterations, r);
        break;
      case FX_SOLVER_GMRES:
        s.gmres(b, x, r);
        break;
      case FX_SOLVER_KRYLOV: {
        FX_CUDA(cudaMemcpyAsync(s.x0.ptr, x, sizeof(double) * s.n, cudaMemcpyDeviceToDevice, s.cs));
        s.cg<double>(b, x, s.r.ptr, s.p.ptr, s.ap.ptr, s.inv.ptr, s.o.rtol, s.o.atol, s.o.max_iterations, r);
        if (r->indefinite) {
          const int cg_it = r->iterations;
          FX_CUDA(cudaMemcpyAsync(x, s.x0.ptr, sizeof(double) * s.n, cudaMemcpyDeviceToDevice, s.cs));
          *r = fx_solve_result{};
          s.gmres(b, x, r);
          r->iterations += cg_it;
          r->indefinite = 1;
        }
        break;
      }
      case FX_SOLVER_IR:
        s.ir(b, x, r);
        break;
    }
    FX_CUDA(cudaEventRecord(s.ev_out, s.cs));
    FX_CUDA(cudaStreamWaitEvent(st, s.ev_out, 0));
    r->status = r->converged ? FX_OK : (r->indefinite ? FX_E_NOT_SPD : FX_E_DIVERGED);
  });
}

int fx_solver_newton(fx_solver* h, const double* fext, double* u, int32_t test, double tol, int32_t max_newton,
                     int32_t* newton_iterations, fx_solve_result* r, void* stream) {
  return guard([&] {
    if (!h || !r || !newton_iterations || (h->s.n > 0 && (!fext || !u)) || max_newton < 0 || !(tol >= 0.0))
      throw fx::Error(FX_E_INVALID, "fx_solver_newton: bad arguments");
    if (test != FX_TEST_NORM_UNBALANCE && test != FX_TEST_NORM_DISP_INCR)
      throw fx::Error(FX_E_INVALID, "fx_solver_newton: unknown convergence test");
    fx::Solver& s = h->s;
    if (!s.ready) throw fx::Error(FX_E_INVALID, "fx_solver_newton: call fx_solver_setup first");
    if (s.method != FX_SOLVER_CG && s.method != FX_SOLVER_IR)
      throw fx::Error(FX_E_UNSUPPORTED, "fx_solver_newton: CG or refined FP32 CG solvers only");
    *r = fx_solve_result{};
    *newton_iterations = 0;
    if (s.n == 0) {
      r->converged = 1;
      return;
    }
    auto st = static_cast<cudaStream_t>(stream);
    FX_CUDA(cudaEventRecord(s.ev_in, st));
    FX_CUDA(cudaStreamWaitEvent(s.cs, s.ev_in, 0));
    *newton_iterations = s.newton(fext, u, test, tol, max_newton, r);
    FX_CUDA(cudaEventRecord(s.ev_out, s.cs));
    FX_CUDA(cudaStreamWaitEvent(st, s.ev_out, 0));
    r->status = r->converged ? FX_OK : (r->indefinite ? FX_E_NOT_SPD : FX_E_DIVERGED);
  });
}

int fx_solver_newmark(fx_solver* h, const double* fext, double* u, double* v, double* a, double dt, double beta,
                      double gamma, int32_t test, double tol, int32_t max_newton, int32_t* newton_iterations,
                      fx_solve_result* r, void* stream) {
  return guard([&] {
    if (!h || !r || !newton_iterations || (h->s.n > 0 && (!fext || !u || !v || !a)) || max_newton < 0 ||
        !(tol >= 0.0) || !(dt > 0.0) || !(beta > 0.0) || !(gamma > 0.0))
      throw fx::Error(FX_E_INVALID, "fx_solver_newmark: bad arguments");
    if (test != FX_TEST_NORM_UNBALANCE && test != FX_TEST_NORM_DISP_INCR)
      throw fx::Error(FX_E_INVALID, "fx_solver_newmark: unknown convergence test");
    fx::Solver& s = h->s;
    if (!s.ready) throw fx::Error(FX_E_INVALID, "fx_solver_newmark: call fx_solver_setup first");
    if (s.method != FX_SOLVER_CG && s.method != FX_SOLVER_IR)
      throw fx::Error(FX_E_UNSUPPORTED, "fx_solver_newmark: CG or IR solvers only");
    *r = fx_solve_result{};
    *newton_iterations = 0;
    if (s.n == 0) {
      r->converged = 1;
      return;
    }
    auto st = static_cast<cudaStream_t>(stream);
    FX_CUDA(cudaEventRecord(s.ev_in, st));
    FX_CUDA(cudaStreamWaitEvent(s.cs, s.ev_in, 0));
    *newton_iterations = s.newmark(fext, u, v, a, dt, beta, gamma, test, tol, max_newton, r);
    FX_CUDA(cudaEventRecord(s.ev_out, s.cs));
    FX_CUDA(cudaStreamWaitEvent(st, s.ev_out, 0));
    r->status = r->converged ? FX_OK : (r->indefinite ? FX_E_NOT_SPD : FX_E_DIVERGED);
  });
}

int fx_solver_newmark_recover(fx_solver* h, const double* fext0, const double* fext1, double* u, double* v, double* a,
                              double dt, double beta, double gamma, int32_t test, double tol, int32_t max_newton,
                              int32_t max_retries, int32_t num_sublevels, int32_t num_substeps, int32_t* stats,
                              fx_solve_result* r, void* stream) {
  return guard([&] {
    if (!h || !r || !stats || (h->s.n > 0 && (!fext1 || !u || !v || !a)) || max_newton < 0 || !(tol >= 0.0) ||
        !(dt > 0.0) || !(beta > 0.0) || !(gamma > 0.0) || max_retries < 0 || num_sublevels < 0 || num_substeps < 1)
      throw fx::Error(FX_E_INVALID, "fx_solver_newmark_recover: bad arguments");
    if (test != FX_TEST_NORM_UNBALANCE && test != FX_TEST_NORM_DISP_INCR)
      throw fx::Error(FX_E_INVALID, "fx_solver_newmark_recover: unknown convergence test");
    fx::Solver& s = h->s;
    if (!s.ready) throw fx::Error(FX_E_INVALID, "fx_solver_newmark_recover: call fx_solver_setup first");
    if (s.method != FX_SOLVER_CG && s.method != FX_SOLVER_IR)
      throw fx::Error(FX_E_UNSUPPORTED, "fx_solver_newmark_recover: CG or IR solvers only");
    *r = fx_solve_result{};
    for (int i = 0; i < 5; ++i) stats[i] = 0;
    if (s.n == 0) {
      r->converged = 1;
      return;
    }
    auto st = static_cast<cudaStream_t>(stream);
    FX_CUDA(cudaEventRecord(s.ev_in, st));
    FX_CUDA(cudaStreamWaitEvent(s.cs, s.ev_in, 0));
    fx::Solver::Recovery rc;
    rc.max_retries = max_retries;
    rc.num_sublevels = num_sublevels;
    rc.num_substeps = num_substeps;
    s.newmark_recover(fext0, fext1, u, v, a, dt, beta, gamma, test, tol, max_newton, rc, r);
    stats[0] = rc.attempts;
    stats[1] = rc.failed;
    stats[2] = rc.retries;
    stats[3] = rc.substepped;
    stats[4] = rc.newton;
    FX_CUDA(cudaEventRecord(s.ev_out, s.cs));
    FX_CUDA(cudaStreamWaitEvent(st, s.ev_out, 0));
    r->status = r->converged ? FX_OK : (r->indefinite ? FX_E_NOT_SPD : FX_E_DIVERGED);
  });
}

int fx_solver_newton_recover(fx_solver* h, const double* fext, double* u, int32_t test, double tol, int32_t max_newton,
                             int32_t max_retries, int32_t* stats, fx_solve_result* r, void* stream) {
  return guard([&] {
    if (!h || !r || !stats || (h->s.n > 0 && (!fext || !u)) || max_newton < 0 || !(tol >= 0.0) || max_retries < 0)
      throw fx::Error(FX_E_INVALID, "fx_solver_newton_recover: bad arguments");
    if (test != FX_TEST_NORM_UNBALANCE && test != FX_TEST_NORM_DISP_INCR)
      throw fx::Error(FX_E_INVALID, "fx_solver_newton_recover: unknown convergence test");
    fx::Solver& s = h->s;
    if (!s.ready) throw fx::Error(FX_E_INVALID, "fx_solver_newton_recover: call fx_solver_setup first");
    if (s.method != FX_SOLVER_CG && s.method != FX_SOLVER_IR)
      throw fx::Error(FX_E_UNSUPPORTED, "fx_solver_newton_recover: CG or refined FP32 CG solvers only");
    *r = fx_solve_result{};
    for (int i = 0; i < 5; ++i) stats[i] = 0;
    if (s.n == 0) {
      r->converged = 1;
      return;
    }
    auto st = static_cast<cudaStream_t>(stream);
    FX_CUDA(cudaEventRecord(s.ev_in, st));
    FX_CUDA(cudaStreamWaitEvent(s.cs, s.ev_in, 0));
    fx::Solver::Recovery rc;
    rc.max_retries = max_retries;
    s.newton_recover(fext, u, test, tol, max_newton, rc, r);
    stats[0] = rc.attempts;
    stats[1] = rc.failed;
    stats[2] = rc.retries;
    stats[4] = rc.newton;
    FX_CUDA(cudaEventRecord(s.ev_out, s.cs));
    FX_CUDA(cudaStreamWaitEvent(st, s.ev_out, 0));
    r->status = r->converged ? FX_OK : (r->indefinite ? FX_E_NOT_SPD : FX_E_DIVERGED);
  });
}

}  // extern "C"
