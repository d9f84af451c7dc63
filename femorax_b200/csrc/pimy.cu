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
#include "force.hpp"
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
__global__ void __launch_bounds__(128, 6) k_pimy_update(const pimy::Params* __restrict__ pp, int stage, int64_t n,
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

// The points of the elements of parameter set `set` (bound to table entry m): the material's new
// state in both buffers and the elastic compact tangent of the material's moduli.
__global__ void k_pimy_elements_init(const int32_t* __restrict__ param, int32_t count, int32_t P, int32_t set,
                                     const PimySet* __restrict__ m, double* __restrict__ committed,
                                     double* __restrict__ trial, double* __restrict__ tan) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count || param[e] != set) return;
  const pimy::Params& p = m->p;
  for (int gp = 0; gp < 8; ++gp) {
    pimy::initial_state(p, pimy::Slab<double>{committed + static_cast<int64_t>(gp) * P + e, 8 * static_cast<int64_t>(P)});
    pimy::initial_state(p, pimy::Slab<double>{trial + static_cast<int64_t>(gp) * P + e, 8 * static_cast<int64_t>(P)});
    const double t[pimy::kTan] = {0.0, p.G0, p.K0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int c = 0; c < pimy::kTan; ++c) tan[(static_cast<int64_t>(c) * 8 + gp) * P + e] = t[c];
  }
}

// host table -> device, in place (kernels and captured graphs keep the pointer)
void upload_table(ForceState& s) {
  FX_CUDA(cudaMemcpy(s.pimy_dev.ptr, s.pimy_h.data(), sizeof(PimySet) * s.pimy_h.size(), cudaMemcpyHostToDevice));
}

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

int fx_force_set_pimy(fx_force* f, int32_t set, const fx_pimy* m) {
  return fx::guard([&] {
    if (!f || !m) throw fx::Error(FX_E_INVALID, "fx_force_set_pimy: bad arguments");
    fx::ForceState& s = f->s;
    if (set < 0 || set >= s.nparams) throw fx::Error(FX_E_INVALID, "fx_force_set_pimy: no such parameter set");
    fx::ParamGP& q = s.params_h[set];
    if (q.kind == FX_MAT_J2 || q.kind == 3) throw fx::Error(FX_E_INVALID, "fx_force_set_pimy: the set has another material");
    if (q.betaKinit != 0.0)
      throw fx::Error(FX_E_UNSUPPORTED, "betaKinit Rayleigh damping on a PressureIndependMultiYield set");
    if ((q.betaK != 0.0 || q.betaKcomm != 0.0) && !s.soil_sd.ptr)
      s.soil_sd.alloc(static_cast<size_t>(6) * 8 * s.P);
    if (q.rho != m->p.rho)
      throw fx::Error(FX_E_INVALID, "fx_force_set_pimy: the set's density (its masses) differs from the material's");
    const int need = fx::pimy::nstate(m->p.ns);
    const int64_t P = s.P;
    if (need > s.pimy_nstate) {  // (re)allocate the point arrays; earlier bindings start again
      s.pimy_committed.alloc(static_cast<size_t>(need) * 8 * P);
      s.pimy_trial.alloc(static_cast<size_t>(need) * 8 * P);
      if (!s.pimy_tan.ptr) s.pimy_tan.alloc(static_cast<size_t>(fx::pimy::kTan) * 8 * P);
      if (!s.pimy_sig.ptr) s.pimy_sig.alloc(static_cast<size_t>(6) * 8 * P);
      s.pimy_nstate = need;
    }
    if (!s.pimy_dev.ptr) s.pimy_dev.alloc(static_cast<size_t>(s.nparams));  // one entry per set at most
    if (!s.plastic_dev.ptr) {
      s.plastic_dev.alloc(1);
      FX_CUDA(cudaMemset(s.plastic_dev.ptr, 0, sizeof(int)));
    }
    if (!s.pimy_failed.ptr) {
      s.pimy_failed.alloc(1);
      FX_CUDA(cudaMemset(s.pimy_failed.ptr, 0, sizeof(int)));
    }
    if (q.kind != 2) {
      q.table = static_cast<int>(s.pimy_h.size());
      s.pimy_h.push_back(fx::PimySet{m->p, 0});
    } else {
      s.pimy_h[q.table] = fx::PimySet{m->p, 0};
    }
    q.kind = 2;
    fx::upload_table(s);
    FX_CUDA(cudaMemcpy(s.params.ptr, s.params_h.data(), sizeof(fx::ParamGP) * s.params_h.size(), cudaMemcpyHostToDevice));
    s.has_pimy = true;
    s.box.qualifies = false;
    s.box.why_not = "the mesh has PressureIndependMultiYield sets";
    // every bound set's points start from their material's state (after a reallocation too)
    for (int32_t k = 0; k < s.nparams; ++k)
      if (s.params_h[k].kind == 2 && s.count > 0) {
        fx::k_pimy_elements_init<<<fx::blocks_for(s.count, 128), 128>>>(s.param.ptr, s.count, s.P, k,
                                                                        s.pimy_dev.ptr + s.params_h[k].table,
                                                                        s.pimy_committed.ptr, s.pimy_trial.ptr,
                                                                        s.pimy_tan.ptr);
        FX_LAUNCH_CHECK("pimy_elements_init");
      }
    FX_CUDA(cudaStreamSynchronize(nullptr));
  });
}

int fx_force_set_material_stage(fx_force* f, int32_t set, int32_t stage) {
  return fx::guard([&] {
    if (!f || (stage != 0 && stage != 1)) throw fx::Error(FX_E_INVALID, "fx_force_set_material_stage: bad arguments");
    fx::ForceState& s = f->s;
    if (set < 0 || set >= s.nparams || (s.params_h[set].kind != 2 && s.params_h[set].kind != 3))
      throw fx::Error(FX_E_INVALID, "fx_force_set_material_stage: not a multi-yield soil set");
    if (s.params_h[set].kind == 2) {
      s.pimy_h[s.params_h[set].table].stage = stage;
      fx::upload_table(s);
    } else {
      s.pdmy_h[s.params_h[set].table].stage = stage;
      FX_CUDA(cudaMemcpy(s.pdmy_dev.ptr, s.pdmy_h.data(), sizeof(fx::PdmySet) * s.pdmy_h.size(),
                         cudaMemcpyHostToDevice));
    }
  });
}

int fx_force_pimy_failed(const fx_force* f, int64_t* count) {
  return fx::guard([&] {
    if (!f || !count) throw fx::Error(FX_E_INVALID, "fx_force_pimy_failed: bad arguments");
    int n = 0;
    if (f->s.pimy_failed.ptr) FX_CUDA(cudaMemcpy(&n, f->s.pimy_failed.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    *count = n;
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
