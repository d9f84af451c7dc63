// The C ABI (include/femorax_b200.h): argument checks, error capture, dispatch to the host
// compile step and the device paths. No exception leaves this file.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>

#include "force.hpp"
#include "host.hpp"
#include "ssp_brick.cuh"

namespace fx {
namespace {
thread_local std::string g_error;
}
void set_error(const std::string& msg) { g_error = msg; }

template <class F>
int guarded(F&& f) {
  try {
    f();
    return FX_OK;
  } catch (const Error& e) {
    g_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_error = "host allocation failed";
    return FX_E_NOMEM;
  } catch (const std::exception& e) {
    g_error = e.what();
    return FX_E_INVALID;
  }
}

#define FX_REQUIRE(cond, msg) \
  if (!(cond)) throw ::fx::Error(FX_E_INVALID, msg)

int64_t ForceState::device_bytes() const {
  int64_t b = coords.bytes() + node.bytes() + eq.bytes() + param.bytes() + params.bytes() + gstart.bytes() +
              glist.bytes() + slots.bytes() + nodal_mass.bytes() + nodal_alpha_mass.bytes() + lumped_mass.bytes() +
              eq_dof.bytes() + wx.bytes() + wy.bytes() + scratch.bytes();
  b += box.node_eq.bytes() + box.elem_param.bytes() + box.escale.bytes() + box.escale32.bytes() + box.la.bytes();
  for (const auto& cs : box.cset) b += cs.coef.bytes() + cs.coef32.bytes() + cs.scoef.bytes() + cs.scoef32.bytes();
  b += j2_committed.bytes() + j2_trial.bytes() + j2_tan.bytes() + plastic_dev.bytes();
  b += geom32.bytes() + nshape32.bytes() + slots32.bytes();
  b += pimy_dev.bytes() + pimy_committed.bytes() + pimy_trial.bytes() + pimy_tan.bytes() + pimy_failed.bytes() + pimy_sig.bytes();
  b += pdmy_dev.bytes() + pdmy_committed.bytes() + pdmy_trial.bytes() + pdmy_tan.bytes() + pdmy_sig.bytes();
  b += soil_sd.bytes();
  return b;
}

}  // namespace fx

using fx::guarded;

extern "C" {

const char* fx_last_error(void) { return fx::g_error.c_str(); }
const char* fx_version(void) { return "femorax_b200 0.1 (sm_100a)"; }

int fx_device_memory(int32_t device, int64_t* free_bytes, int64_t* total_bytes) {
  return guarded([&] {
    FX_REQUIRE(free_bytes && total_bytes && device >= 0, "fx_device_memory: bad arguments");
    int cur = 0;
    FX_CUDA(cudaGetDevice(&cur));
    FX_CUDA(cudaSetDevice(device));
    size_t fr = 0, tot = 0;
    const cudaError_t e = cudaMemGetInfo(&fr, &tot);
    cudaSetDevice(cur);
    FX_CUDA(e);
    *free_bytes = static_cast<int64_t>(fr);
    *total_bytes = static_cast<int64_t>(tot);
  });
}

// ------------------------------------------------------------------ model
int fx_model_create(int32_t num_nodes, const int32_t* tags, const double* coords, fx_model** out) {
  return guarded([&] {
    FX_REQUIRE(out && num_nodes >= 0 && (num_nodes == 0 || (tags && coords)), "fx_model_create: bad arguments");
    auto* m = new fx_model;
    m->tags.assign(tags, tags + num_nodes);
    m->coords.assign(coords, coords + 3 * static_cast<size_t>(num_nodes));
    *out = m;
  });
}
void fx_model_destroy(fx_model* m) { delete m; }

int fx_model_add_group(fx_model* m, const fx_material* mat, const double* b, int32_t lumped, int32_t count,
                       const int32_t* element_tags, const int32_t* connectivity) {
  return guarded([&] {
    FX_REQUIRE(m && mat && b && count >= 0 && (count == 0 || (element_tags && connectivity)),
               "fx_model_add_group: bad arguments");
    FX_REQUIRE(mat->kind == FX_MAT_ELASTIC || mat->kind == FX_MAT_J2, "fx_model_add_group: unknown material kind");
    FX_REQUIRE(mat->element == FX_ELEM_STDBRICK || mat->element == FX_ELEM_SSPBRICK,
               "fx_model_add_group: unknown element type");
    if (mat->element == FX_ELEM_SSPBRICK && mat->kind != FX_MAT_ELASTIC)
      throw fx::Error(FX_E_UNSUPPORTED, "fx_model_add_group: SSPbrick groups take the elastic material");
    FX_REQUIRE(mat->E > 0 && mat->nu > -1.0 && mat->nu < 0.5, "fx_model_add_group: E > 0 and -1 < nu < 0.5 required");
    fx::Group g;
    g.mat = *mat;
    for (int q = 0; q < 3; ++q) g.b[q] = b[q];
    g.lumped = lumped != 0;
    g.tags.assign(element_tags, element_tags + count);
    g.conn.assign(connectivity, connectivity + 8 * static_cast<size_t>(count));
    m->groups.push_back(std::move(g));
  });
}
int fx_ssp_element_constants(const double* xl, double E, double nu, double* geo, double* con) {
  return guarded([&] {
    FX_REQUIRE(xl && geo && con && E > 0 && nu > -1.0 && nu < 0.5, "fx_ssp_element_constants: bad arguments");
    double x[3][8];
    for (int d = 0; d < 3; ++d)
      for (int a = 0; a < 8; ++a) x[d][a] = xl[8 * d + a];
    fx::ParamGP p{};
    p.E = E;
    p.nu = nu;
    double D[6][6];
    fx::elastic_D(p, D);
    fx::ssp::element_setup(x, D[0][0], D[0][1], D[3][3], fx::pimy::Slab<double>{geo, 1},
                           fx::pimy::Slab<double>{con, 1});
  });
}

int fx_model_add_fix(fx_model* m, int32_t n, const int32_t* node, const int32_t* dof) {
  return guarded([&] {
    FX_REQUIRE(m && n >= 0 && (n == 0 || (node && dof)), "fx_model_add_fix: bad arguments");
    m->fix_node.insert(m->fix_node.end(), node, node + n);
    m->fix_dof.insert(m->fix_dof.end(), dof, dof + n);
  });
}
int fx_model_add_equal_dof(fx_model* m, int32_t n, const int32_t* retained, const int32_t* constrained,
                           const int32_t* dof) {
  return guarded([&] {
    FX_REQUIRE(m && n >= 0 && (n == 0 || (retained && constrained && dof)), "fx_model_add_equal_dof: bad arguments");
    m->eqd_retained.insert(m->eqd_retained.end(), retained, retained + n);
    m->eqd_constrained.insert(m->eqd_constrained.end(), constrained, constrained + n);
    m->eqd_dof.insert(m->eqd_dof.end(), dof, dof + n);
  });
}
int fx_model_add_rayleigh(fx_model* m, double alphaM, double betaK, double betaKinit, double betaKcomm, int32_t n,
                          const int32_t* element_tags) {
  return guarded([&] {
    FX_REQUIRE(m && n >= 0 && (n == 0 || element_tags), "fx_model_add_rayleigh: bad arguments");
    fx::Region r{alphaM, betaK, betaKinit, betaKcomm, {}};
    r.elements.assign(element_tags, element_tags + n);
    m->regions.push_back(std::move(r));
  });
}
int fx_model_add_mass(fx_model* m, int32_t n, const int32_t* node, const int32_t* dof, const double* value) {
  return guarded([&] {
    FX_REQUIRE(m && n >= 0 && (n == 0 || (node && dof && value)), "fx_model_add_mass: bad arguments");
    m->mass_node.insert(m->mass_node.end(), node, node + n);
    m->mass_dof.insert(m->mass_dof.end(), dof, dof + n);
    m->mass_value.insert(m->mass_value.end(), value, value + n);
  });
}

// ------------------------------------------------------------------ compile
int fx_compile(const fx_model* m, int32_t renumbering, int32_t simd_width, int32_t coloring, fx_compiled** out) {
  return guarded([&] {
    FX_REQUIRE(m && out, "fx_compile: bad arguments");
    FX_REQUIRE(renumbering == FX_RENUMBER_OFF || renumbering == FX_RENUMBER_RCM, "fx_compile: unknown renumbering");
    auto* c = new fx_compiled;
    try {
      fx::compile_model(*m, renumbering, simd_width, coloring != 0, *c);
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
  });
}
void fx_compiled_destroy(fx_compiled* c) { delete c; }

int fx_compiled_sizes(const fx_compiled* c, int64_t* s) {
  return guarded([&] {
    FX_REQUIRE(c && s, "fx_compiled_sizes: bad arguments");
    s[0] = c->num_nodes;
    s[1] = c->num_equations;
    s[2] = c->num_equations;
    s[3] = c->count > 0 ? 1 : 0;
    s[4] = c->count;
    s[5] = c->padded;
    s[6] = static_cast<int64_t>(c->params.size());
    s[7] = c->color_start.empty() ? 0 : static_cast<int64_t>(c->color_start.size()) - 1;
  });
}

int64_t fx_compiled_array_i32(const fx_compiled* c, const char* name, int32_t* out) {
  if (!c || !name) return -1;
  const std::string n(name);
  const std::vector<int32_t>* v = nullptr;
  std::vector<int32_t> tmp;
  if (n == "node_tag") v = &c->node_tag;
  else if (n == "node_order") v = &c->node_order;
  else if (n == "element_order") v = &c->element_order;
  else if (n == "eq") v = &c->eq;
  else if (n == "dof_offset") v = &c->dof_offset;
  else if (n == "node_model_index") v = &c->node_model_index;
  else if (n == "b_node") v = &c->b_node;
  else if (n == "b_eq") v = &c->b_eq;
  else if (n == "b_param") v = &c->b_param;
  else if (n == "b_tag") v = &c->b_tag;
  else if (n == "color_start") v = &c->color_start;
  else if (n == "color_elements") v = &c->color_elements;
  else if (n == "eq_dof") v = &c->eq_dof;
  else return -1;
  if (out && !v->empty()) std::memcpy(out, v->data(), v->size() * sizeof(int32_t));
  return static_cast<int64_t>(v->size());
}

int64_t fx_compiled_array_f64(const fx_compiled* c, const char* name, double* out) {
  if (!c || !name) return -1;
  const std::string n(name);
  const std::vector<double>* v = nullptr;
  if (n == "coords") v = &c->coords;
  else if (n == "lumped_mass") v = &c->lumped_mass;
  else if (n == "lumped_alpha_mass") v = &c->lumped_alpha_mass;
  else if (n == "nodal_mass") v = &c->nodal_mass;
  else if (n == "nodal_alpha_mass") v = &c->nodal_alpha_mass;
  else return -1;
  if (out && !v->empty()) std::memcpy(out, v->data(), v->size() * sizeof(double));
  return static_cast<int64_t>(v->size());
}

int fx_compiled_mesh(const fx_compiled* c, fx_param_set* params, fx_mesh* mesh) {
  return guarded([&] {
    FX_REQUIRE(c && mesh && (c->params.empty() || params), "fx_compiled_mesh: bad arguments");
    std::copy(c->params.begin(), c->params.end(), params);
    fx_mesh m{};
    m.num_nodes = c->num_nodes;
    m.num_equations = c->num_equations;
    m.coords = c->coords.data();
    m.count = c->count;
    m.padded = c->padded;
    m.node = c->b_node.data();
    m.eq = c->b_eq.data();
    m.param = c->b_param.data();
    m.num_params = static_cast<int32_t>(c->params.size());
    m.params = params;
    m.lumped_mass = c->lumped_mass.data();
    m.nodal_mass = c->nodal_mass.data();
    m.nodal_alpha_mass = c->nodal_alpha_mass.data();
    m.eq_dof = nullptr;  // derived from the element maps by fx_force_create
    *mesh = m;
  });
}

// ------------------------------------------------------------------ force
int fx_force_create(const fx_mesh* mesh, int32_t device, fx_force** out) {
  return guarded([&] {
    FX_REQUIRE(mesh && out, "fx_force_create: bad arguments");
    const fx_mesh& m = *mesh;
    FX_REQUIRE(m.num_nodes >= 0 && m.num_equations >= 0 && m.count >= 0 && m.padded >= m.count,
               "fx_force_create: bad sizes");
    FX_REQUIRE(m.count == 0 || (m.coords && m.node && m.eq && m.param && m.params && m.num_params > 0),
               "fx_force_create: missing arrays");
    FX_CUDA(cudaSetDevice(device));
    auto* h = new fx_force;
    fx::ForceState& s = h->s;
    try {
      s.device = device;
      s.N = m.num_nodes;
      s.neq = m.num_equations;
      s.count = m.count;
      s.P = m.padded;
      s.nparams = m.num_params;
      const size_t P = static_cast<size_t>(m.padded);
      s.coords_h.assign(m.coords, m.coords + 3 * static_cast<size_t>(m.num_nodes));
      s.node_h.assign(m.node, m.node + 8 * P);
      s.eq_h.assign(m.eq, m.eq + 24 * P);
      s.param_h.assign(m.param, m.param + P);
      for (int32_t e = 0; e < m.count; ++e) {
        FX_REQUIRE(s.param_h[e] >= 0 && s.param_h[e] < m.num_params, "fx_force_create: parameter index out of range");
        for (int a = 0; a < 8; ++a) {
          const int32_t n = s.node_h[a * P + e];
          FX_REQUIRE(n >= 0 && n < m.num_nodes, "fx_force_create: node index out of range");
        }
        for (int k = 0; k < 24; ++k) FX_REQUIRE(s.eq_h[k * P + e] < m.num_equations, "fx_force_create: equation out of range");
      }
      s.params_h.resize(static_cast<size_t>(m.num_params));
      for (int32_t i = 0; i < m.num_params; ++i) {
        const fx_param_set& q = m.params[i];
        fx::ParamGP& p = s.params_h[i];
        p = fx::ParamGP{};
        p.E = q.E;
        p.nu = q.nu;
        p.rho = q.rho;
        for (int d = 0; d < 3; ++d) p.b[d] = q.b[d];
        p.alphaM = q.alphaM;
        p.betaK = q.betaK;
        p.betaKinit = q.betaKinit;
        p.betaKcomm = q.betaKcomm;
        p.mass_type = q.mass_type;
        p.kind = q.kind;
        p.sigma_y = q.sigma_y;
        p.H = q.H;
        p.hk = q.hk;
        p.element = q.element;
        FX_REQUIRE(p.element == FX_ELEM_STDBRICK || p.element == FX_ELEM_SSPBRICK, "fx_force_create: unknown element type");
        if (p.element == FX_ELEM_SSPBRICK) {
          if (p.kind != FX_MAT_ELASTIC)
            throw fx::Error(FX_E_UNSUPPORTED, "fx_force_create: SSPbrick sets take the elastic material");
          s.has_ssp = true;
        }
      }
      // per-equation slot lists in (element, DOF) order
      std::vector<int32_t> start(static_cast<size_t>(s.neq) + 1, 0);
      for (int32_t e = 0; e < m.count; ++e)
        for (int k = 0; k < 24; ++k) {
          const int32_t q = s.eq_h[k * P + e];
          if (q >= 0) ++start[q + 1];
        }
      for (int32_t q = 0; q < s.neq; ++q) start[q + 1] += start[q];
      std::vector<int32_t> list(static_cast<size_t>(start[s.neq])), fill(start.begin(), start.end() - 1);
      for (int32_t e = 0; e < m.count; ++e)
        for (int k = 0; k < 24; ++k) {
          const int32_t q = s.eq_h[k * P + e];
          if (q >= 0) list[fill[q]++] = static_cast<int32_t>(k * P + e);
        }
      s.coords.upload(s.coords_h);
      s.node.upload(s.node_h);
      s.eq.upload(s.eq_h);
      s.param.upload(s.param_h);
      s.params.upload(s.params_h);
      s.gstart.upload(start);
      s.glist.upload(list);
      std::vector<int32_t> heavy;
      for (int32_t q = 0; q < s.neq; ++q)
        if (start[q + 1] - start[q] > fx::kHeavySlots) heavy.push_back(q);
      s.nheavy = static_cast<int32_t>(heavy.size());
      if (!heavy.empty()) s.gheavy.upload(heavy);
      s.slots.alloc(24 * P);
      if (s.has_ssp) fx::ssp_setup(s);  // SSPbrick: each element's geometry and stabilization constants
      // J2 sets: state and tangent per Gauss point (virgin state, elastic tangent)
      for (const auto& q : s.params_h)
        if (q.kind == FX_MAT_J2) {
          s.has_j2 = true;
          if (q.betaK != 0.0 || q.betaKinit != 0.0 || q.betaKcomm != 0.0)
            throw fx::Error(FX_E_UNSUPPORTED, "stiffness-proportional Rayleigh damping on a J2 set");
          if (!(q.sigma_y > 0.0) || q.H < 0.0 || q.hk < 0.0 || q.hk > 1.0)
            throw fx::Error(FX_E_INVALID, "J2 set: sigma_y > 0, H >= 0 and 0 <= hk <= 1 required");
        }
      if (s.has_j2) {
        const size_t pts = static_cast<size_t>(8) * P;
        s.j2_committed.upload(std::vector<double>(pts * fx::kJ2State, 0.0));
        s.j2_trial.upload(std::vector<double>(pts * fx::kJ2State, 0.0));
        std::vector<double> tan(pts * fx::kJ2Tan, 0.0);
        std::fill(tan.begin(), tan.begin() + static_cast<std::ptrdiff_t>(pts), 1.0);  // theta = 1
        s.j2_tan.upload(tan);
        s.plastic_dev.alloc(1);
        FX_CUDA(cudaMemset(s.plastic_dev.ptr, 0, sizeof(int)));
      }
      auto nonzero = [&](const double* p) {
        if (!p) return false;
        for (int32_t q = 0; q < s.neq; ++q)
          if (p[q] != 0.0) return true;
        return false;
      };
      s.has_nodal_mass = nonzero(m.nodal_mass);
      s.has_nodal_alpha = nonzero(m.nodal_alpha_mass);
      if (s.has_nodal_mass) {
        s.nodal_mass_h.assign(m.nodal_mass, m.nodal_mass + s.neq);
        s.nodal_mass.upload(s.nodal_mass_h);
      }
      if (s.has_nodal_alpha) {
        s.nodal_alpha_h.assign(m.nodal_alpha_mass, m.nodal_alpha_mass + s.neq);
        s.nodal_alpha_mass.upload(s.nodal_alpha_h);
      }
      if (m.lumped_mass) {
        s.lumped_h.assign(m.lumped_mass, m.lumped_mass + s.neq);
        s.lumped_mass.upload(s.lumped_h);
      }
      // the DOF of every equation, from the element maps
      s.eq_dof_h.assign(static_cast<size_t>(s.neq), -1);
      for (int32_t e = 0; e < m.count; ++e)
        for (int k = 0; k < 24; ++k) {
          const int32_t q = s.eq_h[k * P + e];
          if (q >= 0) s.eq_dof_h[q] = static_cast<int8_t>(k % 3);
        }
      if (m.eq_dof)
        for (int32_t q = 0; q < s.neq; ++q) s.eq_dof_h[q] = m.eq_dof[q];
      s.eq_dof.upload(s.eq_dof_h);
      s.wx.alloc(static_cast<size_t>(std::max(s.neq, 1)));
      s.wy.alloc(static_cast<size_t>(std::max(s.neq, 1)));
      fx::box_build_plan(s);
      if (s.box.qualifies) {
        // FEMORAX_B200_BOX_LAUNCH="variant,kz" pins the launch shape instead of timing the
        // candidates, as the reference's FEMORAX_FORCE_SETTINGS overrides its autotuner
        // (src/exec/force_settings.cpp:186-190)
        int variant = 0, kz = 0;
        const char* o = std::getenv("FEMORAX_B200_BOX_LAUNCH");
        if (o && *o && std::sscanf(o, "%d,%d", &variant, &kz) == 2) fx::box_set_launch(s, variant, kz);
        else fx::box_autotune(s, nullptr);
      }
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

void fx_force_destroy(fx_force* f) { delete f; }

int fx_force_set_soil_corrector(fx_force* f, int32_t mode) {
  return guarded([&] {
    FX_REQUIRE(f && (mode == FX_SOIL_FUSED || mode == FX_SOIL_COMPACTED), "fx_force_set_soil_corrector: bad arguments");
    f->s.compact_soil = mode == FX_SOIL_COMPACTED;
  });
}

int fx_force_set_general_mode(fx_force* f, int32_t mode) {
  return guarded([&] {
    FX_REQUIRE(f && (mode == FX_GENERAL_EXACT || mode == FX_GENERAL_FAST), "fx_force_set_general_mode: bad arguments");
    f->s.fast_general = mode == FX_GENERAL_FAST;
  });
}

int fx_force_set_path(fx_force* f, int32_t path) {
  return guarded([&] {
    FX_REQUIRE(f, "fx_force_set_path: null handle");
    FX_REQUIRE(path == FX_PATH_AUTO || path == FX_PATH_GENERAL || path == FX_PATH_BOX, "fx_force_set_path: unknown path");
    if (path == FX_PATH_BOX && !f->s.box.qualifies)
      throw fx::Error(FX_E_UNSUPPORTED, "the box path needs a structured grid of equal boxes: " + f->s.box.why_not);
    f->s.path = path;
  });
}

int fx_force_info(const fx_force* f, int64_t* info) {
  return guarded([&] {
    FX_REQUIRE(f && info, "fx_force_info: bad arguments");
    const auto& s = f->s;
    info[0] = s.neq;
    info[1] = s.count;
    info[2] = s.use_box() ? FX_PATH_BOX : FX_PATH_GENERAL;
    info[3] = s.box.qualifies;
    info[4] = s.box.nx;
    info[5] = s.box.ny;
    info[6] = s.box.nz;
    info[7] = s.device_bytes();
    info[8] = s.use_box_force();
  });
}

int fx_force_set_launch(fx_force* f, int32_t variant, int32_t kz) {
  return guarded([&] {
    FX_REQUIRE(f, "fx_force_set_launch: null handle");
    if (!f->s.box.qualifies) throw fx::Error(FX_E_UNSUPPORTED, "no box plan: " + f->s.box.why_not);
    fx::box_set_launch(f->s, variant, kz);
  });
}

int fx_force_get_launch(const fx_force* f, int32_t* launch) {
  return guarded([&] {
    FX_REQUIRE(f && launch, "fx_force_get_launch: bad arguments");
    const auto& sh = f->s.box.shape[0][0];
    launch[0] = sh.variant;
    launch[1] = sh.persistent ? -sh.kz : sh.kz;
  });
}

int fx_force_get_launches(const fx_force* f, int32_t* launch) {
  return guarded([&] {
    FX_REQUIRE(f && launch, "fx_force_get_launches: bad arguments");
    for (int prec = 0; prec < 2; ++prec)
      for (int mode = 0; mode < 2; ++mode) {
        const auto& sh = f->s.box.shape[prec][mode];
        launch[(prec * 2 + mode) * 2] = sh.variant;
        launch[(prec * 2 + mode) * 2 + 1] = sh.persistent ? -sh.kz : sh.kz;
      }
  });
}

int fx_force_tune(fx_force* f, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f, "fx_force_tune: null handle");
    if (f->s.box.qualifies) fx::box_autotune(f->s, static_cast<cudaStream_t>(stream));
  });
}

int fx_apply_operator(fx_force* f, fx_coeffs k, const double* x, double* y, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f && (f->s.neq == 0 || (x && y)), "fx_apply_operator: bad arguments");
    FX_REQUIRE(x != y, "fx_apply_operator: x and y must not alias");
    const double kk[3] = {k.stiffness, k.damping, k.mass};
    auto st = static_cast<cudaStream_t>(stream);
    f->s.initial = k.initial != 0;
    if (f->s.use_box()) fx::box_apply(f->s, kk, x, y, st);
    else fx::general_apply(f->s, kk, x, y, st);
  });
}

int fx_apply_operator_f32(fx_force* f, fx_coeffs k, const float* x, float* y, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f && (f->s.neq == 0 || (x && y)), "fx_apply_operator_f32: bad arguments");
    FX_REQUIRE(x != y, "fx_apply_operator_f32: x and y must not alias");
    const double kk[3] = {k.stiffness, k.damping, k.mass};
    f->s.initial = k.initial != 0;
    if (f->s.use_box()) fx::box_apply_f32(f->s, kk, x, y, static_cast<cudaStream_t>(stream));
    else fx::general_apply_f32(f->s, kk, x, y, static_cast<cudaStream_t>(stream));
  });
}

int fx_apply_operator_host(fx_force* f, fx_coeffs k, const double* xh, double* yh, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f && (f->s.neq == 0 || (xh && yh)), "fx_apply_operator_host: bad arguments");
    auto st = static_cast<cudaStream_t>(stream);
    const size_t bytes = sizeof(double) * static_cast<size_t>(f->s.neq);
    const double kk[3] = {k.stiffness, k.damping, k.mass};
    f->s.initial = k.initial != 0;
    if (fx::box_apply_host(f->s, kk, xh, yh, st)) {  // page-locked buffers: copies and tiles overlapped
      FX_CUDA(cudaStreamSynchronize(st));
      return;
    }
    FX_CUDA(cudaMemcpyAsync(f->s.wx.ptr, xh, bytes, cudaMemcpyHostToDevice, st));
    if (f->s.use_box()) fx::box_apply(f->s, kk, f->s.wx.ptr, f->s.wy.ptr, st);
    else fx::general_apply(f->s, kk, f->s.wx.ptr, f->s.wy.ptr, st);
    FX_CUDA(cudaMemcpyAsync(yh, f->s.wy.ptr, bytes, cudaMemcpyDeviceToHost, st));
    FX_CUDA(cudaStreamSynchronize(st));
  });
}

int fx_operator_diagonal(fx_force* f, fx_coeffs k, double* d, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f && (f->s.neq == 0 || d), "fx_operator_diagonal: bad arguments");
    const double kk[3] = {k.stiffness, k.damping, k.mass};
    f->s.initial = k.initial != 0;
    fx::general_diagonal(f->s, kk, d, static_cast<cudaStream_t>(stream));
  });
}

int fx_operator_diagonal_host(fx_force* f, fx_coeffs k, double* dh, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f && (f->s.neq == 0 || dh), "fx_operator_diagonal_host: bad arguments");
    auto st = static_cast<cudaStream_t>(stream);
    const double kk[3] = {k.stiffness, k.damping, k.mass};
    f->s.initial = k.initial != 0;
    fx::general_diagonal(f->s, kk, f->s.wy.ptr, st);
    FX_CUDA(cudaMemcpyAsync(dh, f->s.wy.ptr, sizeof(double) * static_cast<size_t>(f->s.neq), cudaMemcpyDeviceToHost,
                            st));
    FX_CUDA(cudaStreamSynchronize(st));
  });
}

int fx_force_compute(fx_force* f, const double* u, const double* v, double* out, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f && (f->s.neq == 0 || (u && v && out)), "fx_force_compute: bad arguments");
    auto st = static_cast<cudaStream_t>(stream);
    if (f->s.use_box_force()) fx::box_force(f->s, u, v, out, st);
    else fx::general_force(f->s, u, v, out, st);
  });
}

int fx_force_compute_f32(fx_force* f, const float* u, const float* v, float* out, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f && (f->s.neq == 0 || (u && v && out)), "fx_force_compute_f32: bad arguments");
    if (!f->s.use_box_force())
      throw fx::Error(FX_E_UNSUPPORTED, "the FP32 force runs on the box path only: " + f->s.box.why_not);
    fx::box_force_f32(f->s, u, v, out, static_cast<cudaStream_t>(stream));
  });
}

int fx_mass_times_ground(fx_force* f, int32_t dir, double* y, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f && dir >= 0 && dir < 3 && (f->s.neq == 0 || y), "fx_mass_times_ground: bad arguments");
    fx::general_mass_times_ground(f->s, dir, y, static_cast<cudaStream_t>(stream));
  });
}

int fx_force_commit(fx_force* f, void* stream) {
  return guarded([&] {
    FX_REQUIRE(f, "fx_force_commit: null handle");
    fx::ForceState& s = f->s;
    if (s.has_j2)
      FX_CUDA(cudaMemcpyAsync(s.j2_committed.ptr, s.j2_trial.ptr, s.j2_committed.bytes(), cudaMemcpyDeviceToDevice,
                              static_cast<cudaStream_t>(stream)));
    fx::pimy_commit(s, static_cast<cudaStream_t>(stream));
  });
}

static fx::DeviceArray<double>& j2_array(fx::ForceState& s, int32_t which, int& comps) {
  if (!s.has_j2) throw fx::Error(FX_E_UNSUPPORTED, "the mesh has no J2 parameter set");
  if (which == 0 || which == 1) {
    comps = fx::kJ2State;
    return which == 0 ? s.j2_committed : s.j2_trial;
  }
  if (which == 2) {
    comps = fx::kJ2Tan;
    return s.j2_tan;
  }
  throw fx::Error(FX_E_INVALID, "J2 state: which must be 0 (committed), 1 (trial) or 2 (tangent)");
}

int fx_force_state(fx_force* f, int32_t which, double* host, int64_t count) {
  return guarded([&] {
    FX_REQUIRE(f && host, "fx_force_state: bad arguments");
    int comps = 0;
    fx::DeviceArray<double>& a = j2_array(f->s, which, comps);
    FX_REQUIRE(count >= static_cast<int64_t>(a.n), "fx_force_state: host buffer too small");
    FX_CUDA(cudaMemcpy(host, a.ptr, a.bytes(), cudaMemcpyDeviceToHost));
  });
}

int fx_force_set_state(fx_force* f, int32_t which, const double* host, int64_t count) {
  return guarded([&] {
    FX_REQUIRE(f && host, "fx_force_set_state: bad arguments");
    FX_REQUIRE(which == 0 || which == 1, "fx_force_set_state: which must be 0 (committed) or 1 (trial)");
    int comps = 0;
    fx::DeviceArray<double>& a = j2_array(f->s, which, comps);
    FX_REQUIRE(count == static_cast<int64_t>(a.n), "fx_force_set_state: count must be 13 * 8 * padded");
    FX_CUDA(cudaMemcpy(a.ptr, host, a.bytes(), cudaMemcpyHostToDevice));
  });
}

int fx_force_plastic_points(fx_force* f, int64_t* count) {
  return guarded([&] {
    FX_REQUIRE(f && count, "fx_force_plastic_points: bad arguments");
    int n = 0;
    if (f->s.has_j2 || f->s.has_pimy || f->s.has_pdmy)
      FX_CUDA(cudaMemcpy(&n, f->s.plastic_dev.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    f->s.plastic_points = n;
    *count = n;
  });
}

}  // extern "C"
