// Deterministic reductions and element-wise kernels (vector.cu), shared by the solvers.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace fx {

constexpr int64_t kChunk = 2048;
// Iterative refinement (FP32 inner solves, FP64 residuals) ends a linear solve when a round
// leaves the FP64 residual above this fraction of the previous round's: the residual has then
// reached the level that FP64 resolves for the operator, and further FP32 corrections only move
// rounding (the stagnation test of mixed-precision refinement, Carson & Higham 2018).
constexpr double kIrStall = 0.5;
__host__ __device__ inline int64_t chunks_of(int64_t n) { return (n + kChunk - 1) / kChunk; }

// A lane's pass over a chunk in the documented order: use(i, load(i)) for i = begin + k,
// k = lane, lane + lanes, ... < len, in that order, with the loads of U consecutive iterations
// issued before their uses. A chunk is one warp's work and few warps share an SM, so one load in
// flight at a time would leave the pass waiting on memory latency; the order of the uses (and so
// of every sum) is unchanged.
// the operands of one iteration of a lane_loop
template <class T, int N>
struct Ops {
  T v[N];
};

template <int U, class Load, class Use>
__device__ __forceinline__ void lane_loop(int64_t begin, int64_t len, int lane, int lanes, Load load, Use use) {
  int64_t k = lane;
  for (; k + (U - 1) * static_cast<int64_t>(lanes) < len; k += U * static_cast<int64_t>(lanes)) {
    decltype(load(begin)) v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) v[u] = load(begin + k + u * static_cast<int64_t>(lanes));
#pragma unroll
    for (int u = 0; u < U; ++u) use(begin + k + u * static_cast<int64_t>(lanes), v[u]);
  }
  for (; k < len; k += lanes) use(begin + k, load(begin + k));
}

// Block-per-chunk kernels (vectors of few chunks, where one warp per chunk leaves the GPU waiting on
// memory latency): a block of kChunkBlock threads loads and updates a chunk's entries, kChunkPer
// each, all loads issued before their uses, and one warp then sums the chunk in the documented
// order from shared memory, so the sums are those of the warp-per-chunk kernels.
constexpr int kChunkBlock = 256;
constexpr int kChunkPer = static_cast<int>(kChunk) / kChunkBlock;
// Vectors of at most this many chunks use the block-per-chunk forms; longer ones keep a warp per
// chunk (enough warps in flight already; measured on a B200: the block forms 1.4x faster at 64 and
// 51 chunks, equal at 1,495, 4-7 % slower at the served engine's thousands of chunks).
constexpr int64_t kBlockChunks = 1024;

// A chunk's sum of a[j] * b[j], j < len (a, b in shared memory), by one warp: lane l accumulates
// j = l, l + lanes, ... with fused multiply-adds in double, then the lanes' sums in lane order (the
// order of lane_loop over the chunk); the sum in every lane.
template <class T>
__device__ __forceinline__ double chunk_fma_sum(const T* a, const T* b, int len, int lanes, int lane) {
  double acc = 0.0;
  if (lane < lanes)
    for (int j = lane; j < len; j += lanes) acc = fma(static_cast<double>(a[j]), static_cast<double>(b[j]), acc);
  double total = 0.0;
  for (int l = 0; l < lanes; ++l) total += __shfl_sync(0xffffffffu, acc, l);
  return total;
}

// True in the last block of the grid to get here (a grid-wide counter, which that block resets
// to 0 when it is done); every block's writes before the call are visible to it. Every thread of
// the block must call it.
__device__ __forceinline__ bool last_block(unsigned* counter) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  return last;
}

// The levels above a level of chunk sums, by one block, in the order of the level kernels
// (k_reduce_chunks without y): `ncol` columns of n values at stride n in a, alternating with b
// (each holding at least ncol * chunks_of(n) values), the sums in out[0 .. ncol). The values
// were written by other blocks: read through L2.
__device__ __forceinline__ void block_levels(double* a, double* b, int64_t n, int ncol, int lanes, double* out) {
  const int warp = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31);
  const int nw = static_cast<int>(blockDim.x >> 5);
  double* src = a;
  double* dst = b;
  for (;;) {
    const int64_t nc = chunks_of(n);
    for (int64_t item = warp; item < ncol * nc; item += nw) {
      const int col = static_cast<int>(item / nc);
      const int64_t c = item % nc;
      const int64_t begin = c * kChunk;
      const int64_t len = (n - begin < kChunk) ? n - begin : kChunk;
      const double* x = src + col * n;
      double s = 0.0;
      if (lane < lanes)
        lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<double, 1>{{__ldcg(x + i)}}; },
                     [&](int64_t, const Ops<double, 1>& o) { s += o.v[0]; });
      double total = 0.0;
      for (int j = 0; j < lanes; ++j) {
        const double v = __shfl_sync(0xffffffffu, s, j);
        total += v;
      }
      if (lane == 0) {
        if (nc == 1) out[col] = total;
        else dst[col * nc + c] = total;
      }
    }
    __syncthreads();
    if (nc == 1) return;
    double* t = src;
    src = dst;
    dst = t;
    n = nc;
  }
}

// Partial sums for vectors of up to `capacity` entries (VectorOps' partial_[2]).
struct ReduceWork {
  int lanes = 32;
  int64_t capacity = 0;
  DeviceArray<double> level[2];
  void init(int64_t cap, int ln);
};

// One level: out[c] = sum over chunk c of x*y (or of x if y == nullptr) in the documented order.
void reduce_chunks(const double* x, const double* y, int64_t n, int lanes, double* out, cudaStream_t st);
// x.y into *result (device) through the levels of w.
void dot_device(ReduceWork& w, const double* x, const double* y, int64_t n, double* result, cudaStream_t st);
// Reduces k columns of n_partial level-1 chunk sums held in w.level[0] (column c at
// c * n_partial) into result[c] (device), by the levels above.
void reduce_partials(ReduceWork& w, int64_t n_partial, int k, double* result, cudaStream_t st);
// Several dots x_c . y (columns c < k of V, leading dimension ld) into result[c] (device).
void multi_dot_device(ReduceWork& w, const double* V, int64_t ld, int k, const double* y, int64_t n, double* result,
                      cudaStream_t st);

void axpy(double a, const double* x, double* y, int64_t n, cudaStream_t st);
void xpay(const double* x, double a, double* y, int64_t n, cudaStream_t st);
void multiply(const double* d, const double* x, double* y, int64_t n, cudaStream_t st);
void reciprocal(const double* d, double* y, int64_t n, cudaStream_t st);
void fill(double* y, double a, int64_t n, cudaStream_t st);

}  // namespace fx

struct fx_vops {
  int device = 0;
  fx::ReduceWork w;
  fx::DeviceArray<double> result;
};
