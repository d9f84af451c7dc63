// Deterministic reductions in the reference's documented order and the element-wise kernels
// (solvers::VectorOps, src/solvers/vector_ops.cpp:19-103; BlockOps, block_ops.cpp:19-90).
//
// One warp reduces one chunk of 2048 entries: lane l (l < lanes) sums entries l, l + lanes, ...
// of the chunk in index order (fused multiply-add for products), then lane 0 adds the lane sums
// in lane order. Levels of chunk sums repeat this until one value is left. The order depends
// only on n and lanes, so the bits are the same run after run and for any launch shape.
#include <mutex>
#include <string>

#include "vector.hpp"

namespace fx {
namespace {

constexpr int kWarpsPerBlock = 8;

// grid.x: chunk, grid.y: column (multi-dot); x has leading dimension ld per column.
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_reduce_chunks(const double* __restrict__ x, int64_t ld,
                                                                         const double* __restrict__ y, int64_t n,
                                                                         int lanes, int64_t nchunks,
                                                                         double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * kWarpsPerBlock + (threadIdx.x >> 5);
  if (c >= nchunks) return;
  const double* xc = x + static_cast<int64_t>(blockIdx.y) * ld;
  const int64_t begin = c * kChunk;
  const int64_t len = (n - begin < kChunk) ? n - begin : kChunk;
  double s = 0.0;
  if (lane < lanes) {
    if (y)
      lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<double, 2>{{xc[i], y[i]}}; },
                   [&](int64_t, const Ops<double, 2>& o) { s = fma(o.v[0], o.v[1], s); });
    else
      lane_loop<8>(begin, len, lane, lanes, [&](int64_t i) { return Ops<double, 1>{{xc[i]}}; },
                   [&](int64_t, const Ops<double, 1>& o) { s += o.v[0]; });
  }
  // lane 0 adds the lane sums in lane order
  double total = 0.0;
  for (int j = 0; j < lanes; ++j) {
    const double v = __shfl_sync(0xffffffffu, s, j);
    total += v;
  }
  if (lane == 0) out[static_cast<int64_t>(blockIdx.y) * nchunks + c] = total;
}

__global__ void k_axpy(double a, const double* __restrict__ x, double* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}
__global__ void k_xpay(const double* __restrict__ x, double a, double* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = fma(a, y[i], x[i]);
}
__global__ void k_multiply(const double* __restrict__ d, const double* __restrict__ x, double* __restrict__ y,
                           int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = d[i] * x[i];
}
__global__ void k_reciprocal(const double* __restrict__ d, double* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = 1.0 / d[i];
}
__global__ void k_fill(double* __restrict__ y, double a, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = a;
}

unsigned ew_grid(int64_t n) {
  const int64_t blocks = (n + 255) / 256;
  const int64_t cap = static_cast<int64_t>(num_sms()) * 16;
  return static_cast<unsigned>(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

void check_lanes(int lanes) {
  if (lanes < 1 || lanes > 32) throw Error(FX_E_INVALID, "lanes must be in 1..32");
}

}  // namespace

void ReduceWork::init(int64_t cap, int ln) {
  check_lanes(ln);
  lanes = ln;
  capacity = cap;
  const int64_t l1 = std::max<int64_t>(1, chunks_of(cap));
  level[0].alloc(static_cast<size_t>(l1) * 64);  // up to 64 columns (GMRES restart + 1)
  level[1].alloc(static_cast<size_t>(std::max<int64_t>(1, chunks_of(l1))) * 64);
}

void reduce_chunks(const double* x, const double* y, int64_t n, int lanes, double* out, cudaStream_t st) {
  const int64_t nc = chunks_of(n);
  dim3 grid(static_cast<unsigned>((nc + kWarpsPerBlock - 1) / kWarpsPerBlock), 1);
  k_reduce_chunks<<<grid, 32 * kWarpsPerBlock, 0, st>>>(x, 0, y, n, lanes, nc, out);
  FX_LAUNCH_CHECK("reduce_chunks");
}

// Levels of one or several columns (k) of partials of length n each, ending in result[c].
static void reduce_levels(ReduceWork& w, int64_t n, int k, double* result, cudaStream_t st) {
  int cur = 0;
  while (n > 1) {
    const int64_t nc = chunks_of(n);
    double* dst = (nc == 1) ? result : w.level[cur ^ 1].ptr;
    dim3 grid(static_cast<unsigned>((nc + kWarpsPerBlock - 1) / kWarpsPerBlock), static_cast<unsigned>(k));
    k_reduce_chunks<<<grid, 32 * kWarpsPerBlock, 0, st>>>(w.level[cur].ptr, n, nullptr, n, w.lanes, nc, dst);
    FX_LAUNCH_CHECK("reduce_levels");
    if (nc == 1) return;
    n = nc;
    cur ^= 1;
  }
  // a single chunk at level 1: its partials are already the results
  FX_CUDA(cudaMemcpyAsync(result, w.level[cur].ptr, sizeof(double) * static_cast<size_t>(k), cudaMemcpyDeviceToDevice, st));
}

void reduce_partials(ReduceWork& w, int64_t n_partial, int k, double* result, cudaStream_t st) {
  if (n_partial <= 1) {
    // one chunk: its sums are the results (columns at stride 1)
    FX_CUDA(cudaMemcpyAsync(result, w.level[0].ptr, sizeof(double) * static_cast<size_t>(k), cudaMemcpyDeviceToDevice,
                            st));
    return;
  }
  reduce_levels(w, n_partial, k, result, st);
}

void dot_device(ReduceWork& w, const double* x, const double* y, int64_t n, double* result, cudaStream_t st) {
  if (n > w.capacity) throw Error(FX_E_INVALID, "vector longer than the reduction capacity");
  if (n == 0) {
    FX_CUDA(cudaMemsetAsync(result, 0, sizeof(double), st));
    return;
  }
  const int64_t nc = chunks_of(n);
  dim3 grid(static_cast<unsigned>((nc + kWarpsPerBlock - 1) / kWarpsPerBlock), 1);
  k_reduce_chunks<<<grid, 32 * kWarpsPerBlock, 0, st>>>(x, 0, y, n, w.lanes, nc, nc == 1 ? result : w.level[0].ptr);
  FX_LAUNCH_CHECK("dot");
  if (nc > 1) reduce_levels(w, nc, 1, result, st);
}

void multi_dot_device(ReduceWork& w, const double* V, int64_t ld, int k, const double* y, int64_t n, double* result,
                      cudaStream_t st) {
  if (k <= 0) return;
  if (k > 64) throw Error(FX_E_INVALID, "too many columns");
  if (n > w.capacity) throw Error(FX_E_INVALID, "vector longer than the reduction capacity");
  const int64_t nc = chunks_of(n);
  dim3 grid(static_cast<unsigned>((nc + kWarpsPerBlock - 1) / kWarpsPerBlock), static_cast<unsigned>(k));
  k_reduce_chunks<<<grid, 32 * kWarpsPerBlock, 0, st>>>(V, ld, y, n, w.lanes, nc, nc == 1 ? result : w.level[0].ptr);
  FX_LAUNCH_CHECK("multi_dot");
  if (nc > 1) reduce_levels(w, nc, k, result, st);
}

void axpy(double a, const double* x, double* y, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  k_axpy<<<ew_grid(n), 256, 0, st>>>(a, x, y, n);
  FX_LAUNCH_CHECK("axpy");
}
void xpay(const double* x, double a, double* y, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  k_xpay<<<ew_grid(n), 256, 0, st>>>(x, a, y, n);
  FX_LAUNCH_CHECK("xpay");
}
void multiply(const double* d, const double* x, double* y, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  k_multiply<<<ew_grid(n), 256, 0, st>>>(d, x, y, n);
  FX_LAUNCH_CHECK("multiply");
}
void reciprocal(const double* d, double* y, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  k_reciprocal<<<ew_grid(n), 256, 0, st>>>(d, y, n);
  FX_LAUNCH_CHECK("reciprocal");
}
void fill(double* y, double a, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  k_fill<<<ew_grid(n), 256, 0, st>>>(y, a, n);
  FX_LAUNCH_CHECK("fill");
}

// ------------------------------------------------------------------ dot without allocation
// The same reduction as dot_device, with its partial sums in one file-scope device array
// instead of memory allocated by a handle. The array is shared by every call in the process:
// each level writes every partial it later reads, so nothing has to start at zero, and it keeps
// the last call's partials afterwards. Calls whose kernels overlap on the GPU race on it.
namespace {
constexpr int64_t kNoAllocMaxN = int64_t(1) << 27;                     // entries per vector
constexpr int64_t kNoAllocL0 = (kNoAllocMaxN + kChunk - 1) / kChunk;  // 65536 chunk sums
constexpr int64_t kNoAllocL1 = (kNoAllocL0 + kChunk - 1) / kChunk;    // 32 sums of those
constexpr int kNoAllocDevices = 64;
static_assert((kNoAllocL0 + kChunk - 1) / kChunk <= kNoAllocL1, "level 1 holds the sums of level 0's chunks");
static_assert((kNoAllocL1 + kChunk - 1) / kChunk <= kNoAllocL0, "level 0 holds the sums of level 1's chunks");
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocL0 + kNoAllocL1 + 1];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocDevices] = {};

// Device memory on `dev` (or managed memory): the vectors a kernel on the current device reads.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();  // clear the query's error state
    return false;
  }
  return a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
}

// The scratch array's address on the current device, looked up on the first call there. The
// vectors must live on that device: the address is only valid there.
double* noalloc_scratch(const double* x, const double* y, int64_t n) {
  int dev = 0;
  FX_CUDA(cudaGetDevice(&dev));
  if (n > 0 && (!on_device(x, dev) || !on_device(y, dev)))
    throw Error(FX_E_INVALID, "fx_dot_noalloc: x and y must be device memory of the current device (" +
                                  std::to_string(dev) + ")");
  if (dev < 0 || dev >= kNoAllocDevices) throw Error(FX_E_UNSUPPORTED, "fx_dot_noalloc: device index above 63");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw Error(FX_E_CUDA, std::string("fx_dot_noalloc: cudaGetSymbolAddress of the scratch array failed: ") +
                                 cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  return g_noalloc_ptr[dev];
}
}  // namespace

void dot_noalloc(const double* x, const double* y, int64_t n, int lanes, double* result, double* result_host,
                 cudaStream_t st) {
  check_lanes(lanes);
  if (n < 0 || (n > 0 && (!x || !y))) throw Error(FX_E_INVALID, "fx_dot_noalloc: bad arguments");
  if (n > kNoAllocMaxN)
    throw Error(FX_E_INVALID, "fx_dot_noalloc: n = " + std::to_string(n) + " exceeds the scratch limit of " +
                                  std::to_string(kNoAllocMaxN) + " entries");
  if (!result && !result_host) throw Error(FX_E_INVALID, "fx_dot_noalloc: no result pointer given");
  double* scratch = noalloc_scratch(x, y, n);
  double* level[2] = {scratch, scratch + kNoAllocL0};
  double* r = result ? result : scratch + kNoAllocL0 + kNoAllocL1;
  if (n == 0) {
    FX_CUDA(cudaMemsetAsync(r, 0, sizeof(double), st));
  } else {
    int64_t nc = chunks_of(n);
    dim3 grid(static_cast<unsigned>((nc + kWarpsPerBlock - 1) / kWarpsPerBlock), 1);
    k_reduce_chunks<<<grid, 32 * kWarpsPerBlock, 0, st>>>(x, 0, y, n, lanes, nc, nc == 1 ? r : level[0]);
    FX_LAUNCH_CHECK("dot_noalloc");
    int cur = 0;
    while (nc > 1) {
      const int64_t m = chunks_of(nc);
      if (m > (cur ? kNoAllocL0 : kNoAllocL1)) throw Error(FX_E_INVALID, "fx_dot_noalloc: level overflow");
      dim3 g(static_cast<unsigned>((m + kWarpsPerBlock - 1) / kWarpsPerBlock), 1);
      k_reduce_chunks<<<g, 32 * kWarpsPerBlock, 0, st>>>(level[cur], 0, nullptr, nc, lanes, m,
                                                         m == 1 ? r : level[cur ^ 1]);
      FX_LAUNCH_CHECK("dot_noalloc levels");
      nc = m;
      cur ^= 1;
    }
  }
  if (result_host) {
    FX_CUDA(cudaMemcpyAsync(result_host, r, sizeof(double), cudaMemcpyDeviceToHost, st));
    FX_CUDA(cudaStreamSynchronize(st));
  }
}

}  // namespace fx

// ------------------------------------------------------------------ C ABI
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

int fx_vops_create(int64_t capacity, int32_t lanes, int32_t device, fx_vops** out) {
  return guard([&] {
    if (!out || capacity < 0) throw fx::Error(FX_E_INVALID, "fx_vops_create: bad arguments");
    FX_CUDA(cudaSetDevice(device));
    auto* v = new fx_vops;
    try {
      v->device = device;
      v->w.init(capacity, lanes);
      v->result.alloc(1);
    } catch (...) {
      delete v;
      throw;
    }
    *out = v;
  });
}

void fx_vops_destroy(fx_vops* v) { delete v; }

int fx_vops_dot(fx_vops* v, const double* x, const double* y, int64_t n, double* result_dev, double* result_host,
                void* stream) {
  return guard([&] {
    if (!v || n < 0 || (n > 0 && (!x || !y))) throw fx::Error(FX_E_INVALID, "fx_vops_dot: bad arguments");
    auto st = static_cast<cudaStream_t>(stream);
    double* r = result_dev ? result_dev : v->result.ptr;
    fx::dot_device(v->w, x, y, n, r, st);
    if (result_host) {
      FX_CUDA(cudaMemcpyAsync(result_host, r, sizeof(double), cudaMemcpyDeviceToHost, st));
      FX_CUDA(cudaStreamSynchronize(st));
    }
  });
}

int fx_dot_noalloc(const double* x, const double* y, int64_t n, int32_t lanes, double* result_dev,
                   double* result_host, void* stream) {
  return guard([&] { fx::dot_noalloc(x, y, n, lanes, result_dev, result_host, static_cast<cudaStream_t>(stream)); });
}

int fx_axpy(double a, const double* x, double* y, int64_t n, void* stream) {
  return guard([&] { fx::axpy(a, x, y, n, static_cast<cudaStream_t>(stream)); });
}
int fx_xpay(const double* x, double a, double* y, int64_t n, void* stream) {
  return guard([&] { fx::xpay(x, a, y, n, static_cast<cudaStream_t>(stream)); });
}
int fx_multiply(const double* d, const double* x, double* y, int64_t n, void* stream) {
  return guard([&] { fx::multiply(d, x, y, n, static_cast<cudaStream_t>(stream)); });
}

}  // extern "C"
