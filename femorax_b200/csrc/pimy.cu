// PressureIndependMultiYield material points on the device (and the same arithmetic on the host):
// the C ABI fx_pimy_* over pimy.cuh. One thread per point; a point's state values, strains, stresses
// and tangent entries lie `npoints` apart (value-major), so a warp reads and writes every value of 32
// points as whole cache lines. Built with --fmad=false, like the Gauss-point path: the update is the
// reference's sequence of operations (pressure_independ_multi_yield.hpp), uncontracted.
#include <cuda_runtime.h>

#include <cmath>
#include <exception>
#include <string>

#include "common.cuh"
#include "host.hpp"
#include "pimy.cuh"

struct fx_pimy {
  fx::pimy::Params p{};
  fx::DeviceArray<fx::pimy::Params> dev;  // uploaded at the first device update
};

namespace fx {
namespace {

template <class F>
int guard(F&& f) {
  try {
    f();
    return FX_OK;
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_error(e.what());
    return FX_E_INVALID;
  }
}

__global__ void k_pimy_init(const pimy::Params* __restrict__ p, int64_t n, double* __restrict__ s) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  pimy::initial_state(*p, pimy::Slab<double>{s + i, n});
}

// Point i: strain eps[c n + i], stress sig[c n + i], tangent D[(6 r + c) n + i] (NULL: not stored),
// failures counted in *failed (NULL: not counted).
__global__ void __launch_bounds__(128) k_pimy_update(const pimy::Params* __restrict__ pp, int stage, int64_t n,
                                                     const double* __restrict__ committed, double* __restrict__ trial,
                                                     const double* __restrict__ eps, double* __restrict__ sig,
                                                     double* __restrict__ D, int* __restrict__ failed) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const pimy::Params& p = *pp;
  double e[6], s[6], d[36];
  for (int c = 0; c < 6; ++c) e[c] = eps[c * n + i];
  const bool ok = pimy::update(p, stage, pimy::Slab<const double>{committed + i, n}, pimy::Slab<double>{trial + i, n},
                               e, s, d);
  for (int c = 0; c < 6; ++c) sig[c * n + i] = s[c];
  if (D)
    for (int k = 0; k < 36; ++k) D[k * n + i] = d[k];
  if (!ok && failed) atomicAdd(failed, 1);
}

unsigned blocks_for(int64_t n, int threads) { return static_cast<unsigned>((n + threads - 1) / threads); }

}  // namespace
}  // namespace fx

extern "C" {

int fx_pimy_create(const double* in9, const double* pairs, fx_pimy** out) {
  return fx::guard([&] {
    if (!in9 || !out) throw fx::Error(FX_E_INVALID, "fx_pimy_create: bad arguments");
    auto* h = new fx_pimy;
    const int rc = fx::pimy::setup(in9, pairs, h->p);
    if (rc != fx::pimy::kOk) {
      delete h;
      static const char* why[] = {"", "more yield surfaces than the 40 this build holds",
                                  "the backbone gives a friction angle outside [0, 90] degrees",
                                  "the backbone gives a non-positive plastic modulus",
                                  "a user backbone needs at least 2 pairs",
                                  "a modulus, the peak shear strain or the reference pressure is not positive"};
      throw fx::Error(rc == fx::pimy::kTooManySurfaces ? FX_E_UNSUPPORTED : FX_E_INVALID,
                      std::string("PressureIndependMultiYield: ") + why[rc]);
    }
    *out = h;
  });
}

void fx_pimy_destroy(fx_pimy* h) { delete h; }

int fx_pimy_info(const fx_pimy* h, int32_t* nstate, int32_t* surfaces) {
  return fx::guard([&] {
    if (!h) throw fx::Error(FX_E_INVALID, "fx_pimy_info: bad arguments");
    if (nstate) *nstate = fx::pimy::nstate(h->p.ns);
    if (surfaces) *surfaces = h->p.ns;
  });
}

int fx_pimy_setup_values(const fx_pimy* h, double* out) {
  return fx::guard([&] {
    if (!h || !out) throw fx::Error(FX_E_INVALID, "fx_pimy_setup_values: bad arguments");
    out[0] = h->p.p_res;
    out[1] = h->p.phi;
    out[2] = h->p.cohesion;
    for (int i = 1; i <= fx::pimy::kMaxSurfaces; ++i) {
      out[2 + i] = h->p.size[i];
      out[2 + fx::pimy::kMaxSurfaces + i] = h->p.modulus[i];
    }
  });
}

int fx_pimy_init(fx_pimy* h, int64_t npoints, double* state, void* stream) {
  return fx::guard([&] {
    if (!h || npoints < 0 || (npoints > 0 && !state)) throw fx::Error(FX_E_INVALID, "fx_pimy_init: bad arguments");
    if (!h->dev.ptr) h->dev.upload(&h->p, 1);
    if (npoints == 0) return;
    fx::k_pimy_init<<<fx::blocks_for(npoints, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(h->dev.ptr, npoints,
                                                                                                   state);
    FX_LAUNCH_CHECK("pimy_init");
  });
}

int fx_pimy_update(fx_pimy* h, int32_t stage, int64_t npoints, const double* committed, double* trial,
                   const double* strain, double* stress, double* tangent, int32_t* failed, void* stream) {
  return fx::guard([&] {
    if (!h || npoints < 0 || (stage != 0 && stage != 1) ||
        (npoints > 0 && (!committed || !trial || !strain || !stress)))
      throw fx::Error(FX_E_INVALID, "fx_pimy_update: bad arguments");
    if (!h->dev.ptr) h->dev.upload(&h->p, 1);
    if (npoints == 0) return;
    fx::k_pimy_update<<<fx::blocks_for(npoints, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        h->dev.ptr, stage, npoints, committed, trial, strain, stress, tangent, failed);
    FX_LAUNCH_CHECK("pimy_update");
  });
}

int fx_pimy_init_host(const fx_pimy* h, int64_t npoints, double* state) {
  return fx::guard([&] {
    if (!h || npoints < 0 || (npoints > 0 && !state)) throw fx::Error(FX_E_INVALID, "fx_pimy_init_host: bad arguments");
    for (int64_t i = 0; i < npoints; ++i) fx::pimy::initial_state(h->p, fx::pimy::Slab<double>{state + i, npoints});
  });
}

int fx_pimy_update_host(const fx_pimy* h, int32_t stage, int64_t npoints, const double* committed, double* trial,
                        const double* strain, double* stress, double* tangent, int32_t* failed) {
  return fx::guard([&] {
    if (!h || npoints < 0 || (stage != 0 && stage != 1) ||
        (npoints > 0 && (!committed || !trial || !strain || !stress)))
      throw fx::Error(FX_E_INVALID, "fx_pimy_update_host: bad arguments");
    int32_t bad = 0;
    for (int64_t i = 0; i < npoints; ++i) {
      double e[6], s[6], d[36];
      for (int c = 0; c < 6; ++c) e[c] = strain[c * npoints + i];
      const bool ok = fx::pimy::update(h->p, stage, fx::pimy::Slab<const double>{committed + i, npoints},
                                       fx::pimy::Slab<double>{trial + i, npoints}, e, s, d);
      for (int c = 0; c < 6; ++c) stress[c * npoints + i] = s[c];
      if (tangent)
        for (int k = 0; k < 36; ++k) tangent[k * npoints + i] = d[k];
      bad += !ok;
    }
    if (failed) *failed += bad;
  });
}

}  // extern "C"
