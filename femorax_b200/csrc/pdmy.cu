// PressureDependMultiYield material points on the device (and the same arithmetic on the host): the
// C ABI fx_pdmy_* over pdmy.cuh, laid out as fx_pimy_* (one thread per point, value-major arrays).
// Built with --fmad=false: the update is the reference's sequence of operations, uncontracted.
#include <cuda_runtime.h>

#include <algorithm>
#include <exception>
#include <string>

#include "common.cuh"
#include "force.hpp"
#include "host.hpp"
#include "pdmy.cuh"

struct fx_pdmy {
  fx::pdmy::Params p{};
  fx::DeviceArray<fx::pdmy::Params> dev;  // uploaded at the first device call
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

__global__ void k_pdmy_init(const pdmy::Params* __restrict__ p, int64_t n, double* __restrict__ s) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  pdmy::initial_state(*p, pimy::Slab<double>{s + i, n});
}

__global__ void __launch_bounds__(128, 4) k_pdmy_update(const pdmy::Params* __restrict__ pp, int stage, int64_t n,
                                                     const double* __restrict__ committed, double* __restrict__ trial,
                                                     const double* __restrict__ eps, double* __restrict__ sig,
                                                     double* __restrict__ D, int* __restrict__ failed) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  double e[6], s[6], d[36];
  for (int c = 0; c < 6; ++c) e[c] = eps[c * n + i];
  const bool ok = pdmy::update(*pp, stage, pimy::Slab<const double>{committed + i, n}, pimy::Slab<double>{trial + i, n},
                               e, s, D ? d : nullptr);
  for (int c = 0; c < 6; ++c) sig[c * n + i] = s[c];
  if (D)
    for (int k = 0; k < 36; ++k) D[k * n + i] = d[k];
  if (!ok && failed) atomicAdd(failed, 1);
}

unsigned blocks_for(int64_t n, int threads) { return static_cast<unsigned>((n + threads - 1) / threads); }

// The points of the elements of parameter set `set` (table entry m): the material's new state in both
// buffers and the elastic compact tangent.
__global__ void k_pdmy_elements_init(const int32_t* __restrict__ param, int32_t count, int32_t P, int32_t set,
                                     const PdmySet* __restrict__ m, double* __restrict__ committed,
                                     double* __restrict__ trial, double* __restrict__ tan) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count || param[e] != set) return;
  for (int gp = 0; gp < 8; ++gp) {
    const int64_t base = static_cast<int64_t>(gp) * P + e, ld = 8 * static_cast<int64_t>(P);
    pdmy::initial_state(m->p, pimy::Slab<double>{committed + base, ld});
    pdmy::initial_state(m->p, pimy::Slab<double>{trial + base, ld});
    for (int c = 0; c < pdmy::kTan; ++c) tan[base + c * ld] = 0.0;  // stage 0: the elastic tangent
  }
}

// fx_math.h's function `fn` (FX_MATH_*) of x (and y for pow), element by element
FX_HD double math_of(int fn, double x, double y) {
  return fn == FX_MATH_EXP ? fxm_exp(x) : fn == FX_MATH_LOG ? fxm_log(x) : fn == FX_MATH_POW ? fxm_pow(x, y) : fxm_cos(x);
}
__global__ void k_math_eval(int fn, const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ out,
                            int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = math_of(fn, x[i], y ? y[i] : 0.0);
}
void check_math(int32_t fn, const double* x, const double* y, const double* out, int64_t n, const char* who) {
  if (fn < FX_MATH_EXP || fn > FX_MATH_COS || n < 0 || (n > 0 && (!x || !out || (fn == FX_MATH_POW && !y))))
    throw Error(FX_E_INVALID, std::string(who) + ": bad arguments");
}

void check_update(const fx_pdmy* h, int32_t stage, int64_t n, const double* c, const double* t, const double* e,
                  const double* s, const char* who) {
  if (!h || n < 0 || (stage != 0 && stage != 1) || (n > 0 && (!c || !t || !e || !s)))
    throw Error(FX_E_INVALID, std::string(who) + ": bad arguments");
}

}  // namespace
}  // namespace fx

extern "C" {

int fx_pdmy_create(const double* in23, const double* pairs, fx_pdmy** out) {
  return fx::guard([&] {
    if (!in23 || !out) throw fx::Error(FX_E_INVALID, "fx_pdmy_create: bad arguments");
    auto* h = new fx_pdmy;
    const int rc = fx::pdmy::setup(in23, pairs, h->p);
    if (rc != fx::pimy::kOk) {
      delete h;
      static const char* why[] = {"", "more yield surfaces than the 40 this build holds",
                                  "the backbone gives a friction angle outside [0, 90] degrees",
                                  "the backbone gives a non-positive plastic modulus",
                                  "a user backbone needs at least 2 pairs",
                                  "a modulus, an angle, the peak shear strain, the reference pressure, the density or "
                                  "the void ratio is out of range"};
      throw fx::Error(rc == fx::pimy::kTooManySurfaces ? FX_E_UNSUPPORTED : FX_E_INVALID,
                      std::string("PressureDependMultiYield: ") + why[rc]);
    }
    *out = h;
  });
}

void fx_pdmy_destroy(fx_pdmy* h) { delete h; }

int fx_pdmy_info(const fx_pdmy* h, int32_t* nstate, int32_t* surfaces) {
  return fx::guard([&] {
    if (!h) throw fx::Error(FX_E_INVALID, "fx_pdmy_info: bad arguments");
    if (nstate) *nstate = fx::pdmy::nstate(h->p.ns);
    if (surfaces) *surfaces = h->p.ns;
  });
}

int fx_pdmy_setup_values(const fx_pdmy* h, double* out) {
  return fx::guard([&] {
    if (!h || !out) throw fx::Error(FX_E_INVALID, "fx_pdmy_setup_values: bad arguments");
    out[0] = h->p.p_res;
    out[1] = h->p.phi;
    out[2] = h->p.phi_pt;
    out[3] = h->p.ratio_pt;
    out[4] = h->p.strain_pt;
    for (int i = 1; i <= fx::pimy::kMaxSurfaces; ++i) {
      out[4 + i] = h->p.size[i];
      out[4 + fx::pimy::kMaxSurfaces + i] = h->p.modulus[i];
    }
  });
}

int fx_pdmy_init(fx_pdmy* h, int64_t npoints, double* state, void* stream) {
  return fx::guard([&] {
    if (!h || npoints < 0 || (npoints > 0 && !state)) throw fx::Error(FX_E_INVALID, "fx_pdmy_init: bad arguments");
    if (!h->dev.ptr) h->dev.upload(&h->p, 1);
    if (npoints == 0) return;
    fx::k_pdmy_init<<<fx::blocks_for(npoints, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(h->dev.ptr, npoints,
                                                                                                   state);
    FX_LAUNCH_CHECK("pdmy_init");
  });
}

int fx_pdmy_update(fx_pdmy* h, int32_t stage, int64_t npoints, const double* committed, double* trial,
                   const double* strain, double* stress, double* tangent, int32_t* failed, void* stream) {
  return fx::guard([&] {
    fx::check_update(h, stage, npoints, committed, trial, strain, stress, "fx_pdmy_update");
    if (!h->dev.ptr) h->dev.upload(&h->p, 1);
    if (npoints == 0) return;
    fx::k_pdmy_update<<<fx::blocks_for(npoints, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        h->dev.ptr, stage, npoints, committed, trial, strain, stress, tangent, failed);
    FX_LAUNCH_CHECK("pdmy_update");
  });
}

int fx_force_set_pdmy(fx_force* f, int32_t set, const fx_pdmy* m) {
  return fx::guard([&] {
    if (!f || !m) throw fx::Error(FX_E_INVALID, "fx_force_set_pdmy: bad arguments");
    fx::ForceState& s = f->s;
    if (set < 0 || set >= s.nparams) throw fx::Error(FX_E_INVALID, "fx_force_set_pdmy: no such parameter set");
    fx::ParamGP& q = s.params_h[set];
    if (q.kind == FX_MAT_J2 || q.kind == 2) throw fx::Error(FX_E_INVALID, "fx_force_set_pdmy: the set has another material");
    if (q.betaKinit != 0.0)
      throw fx::Error(FX_E_UNSUPPORTED, "betaKinit Rayleigh damping on a PressureDependMultiYield set");
    if ((q.betaK != 0.0 || q.betaKcomm != 0.0) && !s.soil_sd.ptr)
      s.soil_sd.alloc(static_cast<size_t>(6) * 8 * s.P);
    if (q.rho != m->p.rho)
      throw fx::Error(FX_E_INVALID, "fx_force_set_pdmy: the set's density (its masses) differs from the material's");
    const int need = fx::pdmy::nstate(m->p.ns);
    const int64_t P = s.P;
    if (need > s.pdmy_nstate) {  // (re)allocate the point arrays; earlier bindings start again
      s.pdmy_committed.alloc(static_cast<size_t>(need) * 8 * P);
      s.pdmy_trial.alloc(static_cast<size_t>(need) * 8 * P);
      if (!s.pdmy_tan.ptr) s.pdmy_tan.alloc(static_cast<size_t>(fx::pdmy::kTan) * 8 * P);
      if (!s.pdmy_sig.ptr) s.pdmy_sig.alloc(static_cast<size_t>(6) * 8 * P);
      s.pdmy_nstate = need;
    }
    if (!s.pdmy_dev.ptr) s.pdmy_dev.alloc(static_cast<size_t>(s.nparams));
    if (!s.plastic_dev.ptr) {
      s.plastic_dev.alloc(1);
      FX_CUDA(cudaMemset(s.plastic_dev.ptr, 0, sizeof(int)));
    }
    if (!s.pimy_failed.ptr) {
      s.pimy_failed.alloc(1);
      FX_CUDA(cudaMemset(s.pimy_failed.ptr, 0, sizeof(int)));
    }
    if (q.kind != 3) {
      q.table = static_cast<int>(s.pdmy_h.size());
      s.pdmy_h.push_back(fx::PdmySet{m->p, 0});
    } else {
      s.pdmy_h[q.table] = fx::PdmySet{m->p, 0};
    }
    q.kind = 3;
    FX_CUDA(cudaMemcpy(s.pdmy_dev.ptr, s.pdmy_h.data(), sizeof(fx::PdmySet) * s.pdmy_h.size(), cudaMemcpyHostToDevice));
    FX_CUDA(cudaMemcpy(s.params.ptr, s.params_h.data(), sizeof(fx::ParamGP) * s.params_h.size(), cudaMemcpyHostToDevice));
    s.has_pdmy = true;
    s.box.qualifies = false;
    s.box.why_not = "the mesh has PressureDependMultiYield sets";
    for (int32_t k = 0; k < s.nparams; ++k)
      if (s.params_h[k].kind == 3 && s.count > 0) {
        fx::k_pdmy_elements_init<<<fx::blocks_for(s.count, 128), 128>>>(s.param.ptr, s.count, s.P, k,
                                                                        s.pdmy_dev.ptr + s.params_h[k].table,
                                                                        s.pdmy_committed.ptr, s.pdmy_trial.ptr,
                                                                        s.pdmy_tan.ptr);
        FX_LAUNCH_CHECK("pdmy_elements_init");
      }
    FX_CUDA(cudaStreamSynchronize(nullptr));
  });
}

int fx_pdmy_init_host(const fx_pdmy* h, int64_t npoints, double* state) {
  return fx::guard([&] {
    if (!h || npoints < 0 || (npoints > 0 && !state)) throw fx::Error(FX_E_INVALID, "fx_pdmy_init_host: bad arguments");
    for (int64_t i = 0; i < npoints; ++i) fx::pdmy::initial_state(h->p, fx::pimy::Slab<double>{state + i, npoints});
  });
}

int fx_pdmy_update_host(const fx_pdmy* h, int32_t stage, int64_t npoints, const double* committed, double* trial,
                        const double* strain, double* stress, double* tangent, int32_t* failed) {
  return fx::guard([&] {
    fx::check_update(h, stage, npoints, committed, trial, strain, stress, "fx_pdmy_update_host");
    int32_t bad = 0;
    for (int64_t i = 0; i < npoints; ++i) {
      double e[6], s[6], d[36];
      for (int c = 0; c < 6; ++c) e[c] = strain[c * npoints + i];
      const bool ok = fx::pdmy::update(h->p, stage, fx::pimy::Slab<const double>{committed + i, npoints},
                                       fx::pimy::Slab<double>{trial + i, npoints}, e, s, tangent ? d : nullptr);
      for (int c = 0; c < 6; ++c) stress[c * npoints + i] = s[c];
      if (tangent)
        for (int k = 0; k < 36; ++k) tangent[k * npoints + i] = d[k];
      bad += !ok;
    }
    if (failed) *failed += bad;
  });
}

int fx_math_eval(int32_t fn, const double* x, const double* y, double* out, int64_t n, void* stream) {
  return fx::guard([&] {
    fx::check_math(fn, x, y, out, n, "fx_math_eval");
    if (n == 0) return;
    const unsigned grid = static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 148 * 16));
    fx::k_math_eval<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(fn, x, fn == FX_MATH_POW ? y : nullptr, out, n);
    FX_LAUNCH_CHECK("math_eval");
  });
}

int fx_math_eval_host(int32_t fn, const double* x, const double* y, double* out, int64_t n) {
  return fx::guard([&] {
    fx::check_math(fn, x, y, out, n, "fx_math_eval_host");
    for (int64_t i = 0; i < n; ++i) out[i] = fx::math_of(fn, x[i], fn == FX_MATH_POW ? y[i] : 0.0);
  });
}

}  // extern "C"
