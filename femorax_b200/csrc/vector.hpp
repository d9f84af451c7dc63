// Deterministic reductions and element-wise kernels (vector.cu), shared by the solvers.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace fx {

constexpr int64_t kChunk = 2048;
inline int64_t chunks_of(int64_t n) { return (n + kChunk - 1) / kChunk; }

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
