// Test infrastructure only: a C-ABI driver around the reference's own C++ code, compiled from
// the reference's sources (src/physics, src/compile, src/exec, src/solvers) together with the
// Kokkos-subset shim in this folder. It is the "reference run here" that pins the oracle and
// the CUDA path: the reference's compile step (index maps), its InternalForce operator and
// force evaluation (gather scatter, geometry cache), its CG/GMRES/Jacobi solvers and its
// per-element stdBrick physics, all on the host.
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg load the library built from this
// file (oracle/_ref/libfxref.so). The product library never links it.

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "compile/batches.hpp"
#include "exec/ground_motion.hpp"
#include "exec/internal_force.hpp"
#include "exec/matrix_free_operator.hpp"
#include "physics/elements/ssp_brick.hpp"
#include "physics/elements/std_brick.hpp"
#include "physics/materials/elastic_isotropic.hpp"
#include "physics/materials/pressure_depend_multi_yield.hpp"
#include "physics/materials/pressure_independ_multi_yield.hpp"
#include "physics/operators/element_operator.hpp"
#include "solvers/cg.hpp"
#include "solvers/gmres.hpp"
#include "solvers/jacobi.hpp"
#include "solvers/vector_ops.hpp"

using namespace femorax;

namespace {
thread_local std::string g_error;
int fail(const std::exception& e) {
  g_error = e.what();
  return -1;
}
using Brick = StdBrick<ElasticIsotropic>;
}  // namespace

extern "C" {

const char* fxref_last_error() { return g_error.c_str(); }

// ------------------------------------------------------------------------------ model
// A model is described by flat arrays (the fields of io::Model the hot path reads):
//   nodes: tags[N], coords[3N] row-major, ndf 3 for every node;
//   element groups g: material (E, nu, rho), body force b[3], lumped flag, element tags and
//   connectivity (8 node tags per element), group_start[G+1] offsets into the element arrays;
//   fix rows (node tag, dof 1..3); equalDOF rows (retained, constrained, dof);
//   Rayleigh regions r: alphaM, betaK, betaKinit, betaKcomm and element tags
//   (region_start[R+1] offsets); nodal masses (node tag, dof, value).
struct fxref_model {
  io::Model m;
};

fxref_model* fxref_model_create(int32_t N, const int32_t* tags, const double* coords) {
  auto* h = new fxref_model;
  h->m.ndm = 3;
  h->m.nodes.tags.assign(tags, tags + N);
  h->m.nodes.coords.assign(coords, coords + 3 * static_cast<std::size_t>(N));
  h->m.nodes.ndf.assign(static_cast<std::size_t>(N), 3);
  return h;
}

void fxref_model_destroy(fxref_model* h) { delete h; }

// Adds one material (tag = index + 1) and one stdBrick element group that uses it.
// element: 0 stdBrick, 1 SSPbrick.
int fxref_model_add_group(fxref_model* h, double E, double nu, double rho, const double* b, int lumped,
                          int32_t count, const int32_t* etags, const int32_t* conn, int element) {
  io::NDMaterial mat;
  mat.tag = static_cast<std::int32_t>(h->m.materials.size()) + 1;
  mat.data = io::ElasticIsotropicData{E, nu, rho};
  h->m.materials.push_back(mat);
  io::ElementGroup g;
  g.id = std::to_string(h->m.elements.size());
  g.type = element ? io::ElementType::SSPbrick : io::ElementType::StdBrick;
  g.material = mat.tag;
  g.body_force = {b[0], b[1], b[2]};
  g.lumped = lumped != 0;
  g.tags.assign(etags, etags + count);
  g.connectivity.assign(conn, conn + 8 * static_cast<std::size_t>(count));
  h->m.elements.push_back(std::move(g));
  return 0;
}

// The same with a PressureIndependMultiYield material (in9 as fxref_pimy_create; npairs > 0: a user
// backbone, noYieldSurf = -npairs as the model file gives it).
int fxref_model_add_group_pimy(fxref_model* h, const double* in9, const double* pairs, int32_t npairs, const double* b,
                               int lumped, int32_t count, const int32_t* etags, const int32_t* conn) {
  io::NDMaterial mat;
  mat.tag = static_cast<std::int32_t>(h->m.materials.size()) + 1;
  io::PressureIndependMultiYieldData d;
  d.nd = 3;
  d.rho = in9[0];
  d.refShearModul = in9[1];
  d.refBulkModul = in9[2];
  d.cohesi = in9[3];
  d.peakShearStra = in9[4];
  d.frictionAng = in9[5];
  d.refPress = in9[6];
  d.pressDependCoe = in9[7];
  d.noYieldSurf = npairs > 0 ? -npairs : static_cast<std::int32_t>(in9[8]);
  if (npairs > 0) d.pairs.assign(pairs, pairs + 2 * static_cast<std::size_t>(npairs));
  mat.data = d;
  h->m.materials.push_back(mat);
  io::ElementGroup g;
  g.id = std::to_string(h->m.elements.size());
  g.type = io::ElementType::StdBrick;
  g.material = mat.tag;
  g.body_force = {b[0], b[1], b[2]};
  g.lumped = lumped != 0;
  g.tags.assign(etags, etags + count);
  g.connectivity.assign(conn, conn + 8 * static_cast<std::size_t>(count));
  h->m.elements.push_back(std::move(g));
  return 0;
}

// The same with a PressureDependMultiYield material (in23 as fxref_pdmy_create but hv, pv unused:
// the model file has none; npairs > 0: a user backbone, noYieldSurf = -npairs).
int fxref_model_add_group_pdmy(fxref_model* h, const double* in, const double* pairs, int32_t npairs, const double* b,
                               int lumped, int32_t count, const int32_t* etags, const int32_t* conn) {
  io::NDMaterial mat;
  mat.tag = static_cast<std::int32_t>(h->m.materials.size()) + 1;
  io::PressureDependMultiYieldData d;
  d.nd = 3;
  d.rho = in[0];
  d.refShearModul = in[1];
  d.refBulkModul = in[2];
  d.frictionAng = in[3];
  d.peakShearStra = in[4];
  d.refPress = in[5];
  d.pressDependCoe = in[6];
  d.PTAng = in[7];
  d.contrac = in[8];
  d.dilat1 = in[9];
  d.dilat2 = in[10];
  d.liquefac1 = in[11];
  d.liquefac2 = in[12];
  d.liquefac3 = in[13];
  d.noYieldSurf = npairs > 0 ? -npairs : static_cast<std::int32_t>(in[14]);
  if (npairs > 0) d.pairs.assign(pairs, pairs + 2 * static_cast<std::size_t>(npairs));
  d.e = in[15];
  d.cs1 = in[16];
  d.cs2 = in[17];
  d.cs3 = in[18];
  d.pa = in[19];
  d.c = in[20];
  mat.data = d;
  h->m.materials.push_back(mat);
  io::ElementGroup g;
  g.id = std::to_string(h->m.elements.size());
  g.type = io::ElementType::StdBrick;
  g.material = mat.tag;
  g.body_force = {b[0], b[1], b[2]};
  g.lumped = lumped != 0;
  g.tags.assign(etags, etags + count);
  g.connectivity.assign(conn, conn + 8 * static_cast<std::size_t>(count));
  h->m.elements.push_back(std::move(g));
  return 0;
}

void fxref_model_add_fix(fxref_model* h, int32_t n, const int32_t* node, const int32_t* dof) {
  h->m.fix.node.insert(h->m.fix.node.end(), node, node + n);
  h->m.fix.dof.insert(h->m.fix.dof.end(), dof, dof + n);
}

void fxref_model_add_equal_dof(fxref_model* h, int32_t n, const int32_t* retained, const int32_t* constrained,
                               const int32_t* dof) {
  h->m.equal_dof.retained.insert(h->m.equal_dof.retained.end(), retained, retained + n);
  h->m.equal_dof.constrained.insert(h->m.equal_dof.constrained.end(), constrained, constrained + n);
  h->m.equal_dof.dof.insert(h->m.equal_dof.dof.end(), dof, dof + n);
}

void fxref_model_add_rayleigh(fxref_model* h, double alphaM, double betaK, double betaKinit, double betaKcomm,
                              int32_t n, const int32_t* etags) {
  io::RayleighRegion r;
  r.id = std::to_string(h->m.rayleigh.size());
  r.alphaM = alphaM;
  r.betaK = betaK;
  r.betaKinit = betaKinit;
  r.betaKcomm = betaKcomm;
  r.elements.assign(etags, etags + n);
  h->m.rayleigh.push_back(std::move(r));
}

void fxref_model_add_mass(fxref_model* h, int32_t n, const int32_t* node, const int32_t* dof, const double* value) {
  h->m.mass.node.insert(h->m.mass.node.end(), node, node + n);
  h->m.mass.dof.insert(h->m.mass.dof.end(), dof, dof + n);
  h->m.mass.value.insert(h->m.mass.value.end(), value, value + n);
}

// ------------------------------------------------------------------------------ compile
struct fxref_compiled {
  compile::Compiled c;
};

// renumbering: 0 off (file order), 1 RCM. simd_width: the batch padding.
fxref_compiled* fxref_compile(const fxref_model* h, int renumbering, int simd_width, int coloring) {
  try {
    compile::CompileOptions o;
    o.renumbering = renumbering ? compile::Renumbering::RCM : compile::Renumbering::Off;
    o.simd_width = simd_width;
    o.build_coloring = coloring != 0;
    auto* c = new fxref_compiled;
    c->c = compile::compile_model(h->m, o);
    return c;
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}
void fxref_compiled_destroy(fxref_compiled* c) { delete c; }

// Sizes: [num_nodes, num_equations, num_slots, num_batches, batch0 count, batch0 padded,
//         batch0 num params, batch0 num colors]
void fxref_compiled_sizes(const fxref_compiled* h, int64_t* out) {
  const auto& c = h->c;
  out[0] = c.dofs.num_nodes();
  out[1] = c.dofs.num_equations;
  out[2] = c.dofs.num_slots;
  out[3] = static_cast<int64_t>(c.batches.size());
  out[4] = c.batches.empty() ? 0 : c.batches[0].count;
  out[5] = c.batches.empty() ? 0 : c.batches[0].padded;
  out[6] = c.batches.empty() ? 0 : static_cast<int64_t>(c.batches[0].params.size());
  out[7] = c.batches.empty() ? 0 : c.batches[0].num_colors();
}

// Copies a named array of the compiled model (batch 0 for the per-element ones) into out; returns
// its length (call with out = NULL to ask). Names: coords, node_tag, node_order, eq (the DOF
// numbering's eq[ndof]), dof_offset, b_node, b_eq, b_param, b_tag, color_start, color_elements,
// lumped_mass, lumped_alpha_mass, nodal_mass, nodal_alpha_mass, eq_dof.
int64_t fxref_compiled_array_i32(const fxref_compiled* h, const char* name, int32_t* out) {
  const auto& c = h->c;
  const std::vector<std::int32_t>* v = nullptr;
  std::vector<std::int32_t> tmp;
  const std::string n(name);
  if (n == "node_tag") v = &c.dofs.node_tag;
  else if (n == "node_order") v = &c.ordering.node_order;
  else if (n == "element_order") v = &c.ordering.element_order;
  else if (n == "eq") v = &c.dofs.eq;
  else if (n == "dof_offset") v = &c.dofs.dof_offset;
  else if (n == "node_model_index") v = &c.dofs.node_model_index;
  else if (!c.batches.empty() && n == "b_node") v = &c.batches[0].node;
  else if (!c.batches.empty() && n == "b_eq") v = &c.batches[0].eq;
  else if (!c.batches.empty() && n == "b_param") v = &c.batches[0].param;
  else if (!c.batches.empty() && n == "b_tag") v = &c.batches[0].tag;
  else if (!c.batches.empty() && n == "color_start") v = &c.batches[0].color_start;
  else if (!c.batches.empty() && n == "color_elements") v = &c.batches[0].color_elements;
  else if (n == "eq_dof") {
    tmp.assign(c.eq_dof.begin(), c.eq_dof.end());
    v = &tmp;
  } else {
    return -1;
  }
  if (out) std::memcpy(out, v->data(), v->size() * sizeof(std::int32_t));
  return static_cast<int64_t>(v->size());
}

int64_t fxref_compiled_array_f64(const fxref_compiled* h, const char* name, double* out) {
  const auto& c = h->c;
  const std::vector<double>* v = nullptr;
  const std::string n(name);
  if (n == "coords") v = &c.coords;
  else if (n == "lumped_mass") v = &c.lumped_mass;
  else if (n == "lumped_alpha_mass") v = &c.lumped_alpha_mass;
  else if (n == "nodal_mass") v = &c.nodal_mass;
  else if (n == "nodal_alpha_mass") v = &c.nodal_alpha_mass;
  else return -1;
  if (out) std::memcpy(out, v->data(), v->size() * sizeof(double));
  return static_cast<int64_t>(v->size());
}

// Parameter set p of batch 0: [E, nu, rho, b0, b1, b2, massType, alphaM, betaK, betaKinit, betaKcomm,
// group, material, region].
int fxref_compiled_param(const fxref_compiled* h, int32_t p, double* out) {
  const auto& b = h->c.batches.at(0);
  const auto& ps = b.params.at(static_cast<std::size_t>(p));
  const auto bp = ps.params<Brick>();
  const double v[14] = {bp.mat.E,           bp.mat.v,          bp.mat.rho,
                        bp.b[0],            bp.b[1],           bp.b[2],
                        double(bp.massType), ps.damping.alphaM, ps.damping.betaK,
                        ps.damping.betaKinit, ps.damping.betaKcomm, double(ps.group),
                        double(ps.material), double(ps.region)};
  std::memcpy(out, v, sizeof(v));
  return 0;
}

// ------------------------------------------------------------------------------ exec
struct fxref_force {
  std::unique_ptr<exec::InternalForce> f;
  int32_t neq = 0;
  bool stored = false;  // enable_stored_tangents done
};

// cache: 0 Off, 1 On (the geometry cache).
fxref_force* fxref_force_create(const fxref_compiled* c, int cache) {
  try {
    auto* h = new fxref_force;
    h->f = std::make_unique<exec::InternalForce>(c->c, cache ? exec::GeometryCache::On : exec::GeometryCache::Off);
    h->neq = h->f->num_equations();
    return h;
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}
void fxref_force_destroy(fxref_force* h) { delete h; }

namespace {
exec::OperatorSettings op_settings(int scatter, int geometry) {
  exec::OperatorSettings s;
  s.scatter = scatter == 0 ? exec::Scatter::Gather : scatter == 1 ? exec::Scatter::Atomic : exec::Scatter::Colored;
  s.geometry = geometry ? exec::Geometry::Cached : exec::Geometry::Recompute;
  s.tangent = exec::TangentSource::Auto;
  return s;
}
exec::Vec wrap(const double* p, int64_t n) { return exec::Vec(const_cast<double*>(p), static_cast<std::size_t>(n)); }
}  // namespace

// y = (cK K + cC C + cM M) x through InternalForce::apply_operator (u = 0: elastic tangents).
int fxref_apply_operator(fxref_force* h, double cK, double cC, double cM, int scatter, int geometry, const double* x,
                         double* y) {
  try {
    exec::Vec u("u0", static_cast<std::size_t>(h->neq));
    h->f->apply_operator(OperatorCoefficients{cK, cC, cM, false}, op_settings(scatter, geometry), u, wrap(x, h->neq),
                         wrap(y, h->neq));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int fxref_operator_diagonal(fxref_force* h, double cK, double cC, double cM, int geometry, double* d) {
  try {
    exec::Vec u("u0", static_cast<std::size_t>(h->neq));
    h->f->operator_diagonal(OperatorCoefficients{cK, cC, cM, false}, op_settings(0, geometry), u, wrap(d, h->neq));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// y = M r_dir (UniformExcitation load shape), through InternalForce::mass_times_ground.
int fxref_mass_times_ground(fxref_force* h, int dir, double* y) {
  try {
    exec::Vec u("u0", static_cast<std::size_t>(h->neq));
    h->f->mass_times_ground(dir, op_settings(0, 1), u, wrap(y, h->neq));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// f = f_int(u) + Rayleigh damping forces at v (flat layout, gather scatter).
int fxref_force_compute(fxref_force* h, const double* u, const double* v, int geometry, double* f) {
  try {
    auto& F = *h->f;
    for (int32_t q = 0; q < h->neq; ++q) {
      F.u(q) = u[q];
      F.v(q) = v[q];
    }
    exec::ForceSettings s;
    s.layout = exec::Layout::Flat;
    s.scatter = exec::Scatter::Gather;
    s.geometry = geometry ? exec::Geometry::Cached : exec::Geometry::Recompute;
    F.compute(s);
    for (int32_t q = 0; q < h->neq; ++q) f[q] = F.f(q);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// updateMaterialStage of model material `material` (0-based), commitState.
int fxref_force_set_stage(fxref_force* h, int32_t material, int32_t stage) {
  try {
    return h->f->set_material_stage(material, stage) ? 0 : 1;
  } catch (const std::exception& e) {
    return fail(e);
  }
}
int fxref_force_commit(fxref_force* h) {
  try {
    h->f->commit_state();
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// y = K_eff x with each point's tangent determined at displacement u from the committed state and
// stored (store_tangents, TangentSource::Stored: the reference's operator for materials with
// history), and the diagonal likewise.
namespace {
exec::OperatorSettings stored_at(fxref_force* h, const double* u, exec::Vec& uu) {
  if (!h->stored) {
    h->f->enable_stored_tangents();
    h->stored = true;
  }
  for (int32_t q = 0; q < h->neq; ++q) uu(q) = u[q];
  exec::OperatorSettings s = op_settings(0, 1);
  s.tangent = exec::TangentSource::Stored;
  h->f->store_tangents(uu, s);
  return s;
}
}  // namespace
int fxref_apply_operator_at(fxref_force* h, double cK, double cC, double cM, int initial, const double* u,
                            const double* x, double* y) {
  try {
    exec::Vec uu("u", static_cast<std::size_t>(h->neq));
    const exec::OperatorSettings s = stored_at(h, u, uu);
    h->f->apply_operator(OperatorCoefficients{cK, cC, cM, initial != 0}, s, uu, wrap(x, h->neq), wrap(y, h->neq));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}
int fxref_operator_diagonal_at(fxref_force* h, double cK, double cC, double cM, int initial, const double* u,
                               double* d) {
  try {
    exec::Vec uu("u", static_cast<std::size_t>(h->neq));
    const exec::OperatorSettings s = stored_at(h, u, uu);
    h->f->operator_diagonal(OperatorCoefficients{cK, cC, cM, initial != 0}, s, uu, wrap(d, h->neq));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// scheme: 0 CentralDifference, 1 ExplicitDifference.
double fxref_min_critical_dt(fxref_force* h, int scheme) {
  return h->f->min_critical_dt(scheme ? ExplicitScheme::ExplicitDifference : ExplicitScheme::CentralDifference);
}

// Every element's stable step, the batches' in order (dt[] holds the model's element count).
int fxref_element_critical_dts(fxref_force* h, int scheme, double* dt) {
  try {
    const auto all = h->f->element_critical_dts(scheme ? ExplicitScheme::ExplicitDifference
                                                        : ExplicitScheme::CentralDifference);
    std::size_t k = 0;
    for (const auto& b : all)
      for (double v : b) dt[k++] = v;
    return static_cast<int>(k);
  } catch (const std::exception& e) {
    return fail(e);
  }
}
int fxref_stability_may_change(fxref_force* h) { return h->f->stability_may_change() ? 1 : 0; }
int fxref_prepare_stability_bounds(fxref_force* h) {
  try {
    h->f->prepare_stability_bounds();
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}
double fxref_min_critical_dt_bound(fxref_force* h, int scheme) {
  return h->f->min_critical_dt_bound(scheme ? ExplicitScheme::ExplicitDifference : ExplicitScheme::CentralDifference);
}

// ------------------------------------------------------------------------------ solvers
// result: [converged, iterations, rhs_norm, initial_residual, final_residual, indefinite]
int fxref_solve(fxref_force* h, int method, double cK, double cC, double cM, double rtol, double atol, int max_it,
                int lanes, int restart, const double* b, double* x, double* result) {
  try {
    exec::Vec u("u0", static_cast<std::size_t>(h->neq));
    exec::MatrixFreeOperator op(*h->f, u, OperatorCoefficients{cK, cC, cM, false});
    solvers::Jacobi jac;
    jac.setup(op);
    solvers::SolveOptions so;
    so.relative_tolerance = rtol;
    so.absolute_tolerance = atol;
    so.max_iterations = max_it;
    solvers::SolveResult r;
    exec::Vec xv = wrap(x, h->neq);
    if (method == 0) {
      solvers::ConjugateGradient cg(so, lanes);
      cg.setup(op, &jac);
      r = cg.solve(wrap(b, h->neq), xv);
    } else {
      solvers::Gmres gm(so, lanes, restart);
      gm.setup(op, &jac);
      r = gm.solve(wrap(b, h->neq), xv);
    }
    result[0] = r.converged;
    result[1] = r.iterations;
    result[2] = r.rhs_norm;
    result[3] = r.initial_residual;
    result[4] = r.final_residual;
    result[5] = r.indefinite;
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

double fxref_host_dot(const double* x, const double* y, int64_t n, int lanes) {
  std::vector<double> a(x, x + n), b(y, y + n);
  return solvers::VectorOps::host_dot(a, b, lanes);
}

// ------------------------------------------------------------------------------ element level
// One SSPbrick's geometry record (33) and element constants (110) with an elastic material:
// xl[3][8] corner coordinates (x of the 8 corners, then y, then z).
int fxref_ssp_constants(const double* xl, double E, double nu, double* geo, double* con) {
  using Ssp = SSPbrick<ElasticIsotropic>;
  double x[3][8];
  for (int d = 0; d < 3; ++d)
    for (int a = 0; a < 8; ++a) x[d][a] = xl[8 * d + a];
  Ssp::Params p{};
  p.mat = ElasticIsotropic::Params{E, nu, 0.0};
  Ssp::point_store_geometry(x, 0, Strided<double>{geo, 1});
  Ssp::element_constants(p, x, Strided<double>{con, 1});
  return 0;
}

// p = [E, nu, rho, b0, b1, b2, massType]; damp = [alphaM, betaK, betaKinit, betaKcomm];
// xe[8][3]. Outputs fe[24] and, if Ke != NULL, Ke[24][24] row-major.
int fxref_brick_compute(const double* p, const double* damp, const double* xe, const double* u, const double* v,
                        double* fe, double* Ke) {
  Brick::Params bp{{p[0], p[1], p[2]}, {p[3], p[4], p[5]}, static_cast<int>(p[6])};
  Rayleigh d{damp[0], damp[1], damp[2], damp[3], {}};
  const auto* x = reinterpret_cast<const double(*)[3]>(xe);
  if (Ke) {
    Brick::compute<true>(bp, d, x, u, v, {}, {}, fe, reinterpret_cast<double(*)[24]>(Ke));
  } else {
    Brick::compute<false>(bp, d, x, u, v, {}, {}, fe, nullptr);
  }
  return 0;
}

int fxref_brick_mass(const double* p, const double* xe, double* Me, double* lumped) {
  Brick::Params bp{{p[0], p[1], p[2]}, {p[3], p[4], p[5]}, static_cast<int>(p[6])};
  const auto* x = reinterpret_cast<const double(*)[3]>(xe);
  if (Me) Brick::mass(bp, x, Me);
  if (lumped) Brick::lumped_mass(bp, x, lumped);
  return 0;
}

// y_e = K_eff,e v_e by element_operator_apply with recomputed geometry and the constant tangent.
int fxref_brick_operator(const double* p, const double* damp, const double* k, const double* xe, const double* ve,
                         double* ye, int diagonal, const int32_t* eq) {
  Brick::Params bp{{p[0], p[1], p[2]}, {p[3], p[4], p[5]}, static_cast<int>(p[6])};
  Rayleigh d{damp[0], damp[1], damp[2], damp[3], {}};
  OperatorCoefficients kc{k[0], k[1], k[2], false};
  double xl[3][8];
  Brick::local_coords(reinterpret_cast<const double(*)[3]>(xe), xl);
  const auto geo = Brick::recomputed_geometry(xl, bp);
  auto tangent_at = [&](int, const Brick::PointShape&, double (*D)[6]) { ElasticIsotropic::initial_tangent(bp.mat, D); };
  auto committed_at = [&](int, double (*D)[6]) { ElasticIsotropic::initial_tangent(bp.mat, D); };
  if (diagonal) element_operator_diagonal<Brick>(bp, d, kc, geo, tangent_at, committed_at, eq, ye);
  else element_operator_apply<Brick>(bp, d, kc, geo, tangent_at, committed_at, ve, ye);
  return 0;
}

double fxref_brick_critical_dt(const double* p, const double* damp, int scheme, const double* xe) {
  Brick::Params bp{{p[0], p[1], p[2]}, {p[3], p[4], p[5]}, static_cast<int>(p[6])};
  Rayleigh d{damp[0], damp[1], damp[2], damp[3], {}};
  return Brick::critical_dt(bp, d, scheme ? ExplicitScheme::ExplicitDifference : ExplicitScheme::CentralDifference,
                            reinterpret_cast<const double(*)[3]>(xe), {});
}

// ------------------------------------------------------------------------------ ground motions
// exec::GroundMotions (src/exec/ground_motion.cpp) over time series and UniformExcitation
// patterns added one by one (pattern i uses series i); the motions object is built and every
// pattern activated at the first evaluation.
struct fxref_motions {
  io::Model m;
  std::unique_ptr<exec::GroundMotions> g;
};

fxref_motions* fxref_motions_create() { return new fxref_motions; }
void fxref_motions_destroy(fxref_motions* h) { delete h; }

// dof 0-based; times NULL: uniform spacing dt (PathSeries), else PathTimeSeries
int fxref_motions_add(fxref_motions* h, int32_t dof, double fact, const double* values, const double* times,
                      int32_t n, double dt, double factor, int32_t use_last, int32_t prepend_zero) {
  try {
    io::PathSeries s;
    s.tag = static_cast<int32_t>(h->m.time_series.size()) + 1;
    s.factor = factor;
    if (!times) s.dt = dt;
    else s.time.assign(times, times + n);
    s.values.assign(values, values + n);
    s.use_last = use_last != 0;
    s.prepend_zero = prepend_zero != 0;
    h->m.time_series.push_back(s);
    io::UniformExcitation p;
    p.tag = s.tag;
    p.dof = dof + 1;
    p.accel = s.tag;
    p.factor = fact;
    h->m.patterns.push_back(p);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// accel[p] = the active patterns' ground accelerations at time t (GroundMotions::evaluate)
int fxref_motions_evaluate(fxref_motions* h, double t, double* accel) {
  try {
    if (!h->g) {
      h->g = std::make_unique<exec::GroundMotions>(h->m);
      for (const auto& p : h->m.patterns) h->g->activate(p.tag);
    }
    h->g->evaluate(t);
    const auto a = h->g->accel();
    for (int p = 0; p < h->g->num_active(); ++p) accel[p] = a(p);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// ---- PressureIndependMultiYield (the reference's material, 40-surface bucket), one point at a
// time: in9 = rho, refShearModul, refBulkModul, cohesi, peakShearStra, frictionAng, refPress,
// pressDependCoe, noYieldSurf; pairs (gamma, G/Gmax) or NULL.
using Pimy40 = femorax::PressureIndependMultiYield<40>;
struct fxref_pimy {
  Pimy40::Params p{};
  std::vector<double> pairs;
};

int fxref_pimy_create(const double* in9, const double* pairs, int32_t npairs, fxref_pimy** out) {
  auto h = std::make_unique<fxref_pimy>();
  if (pairs && npairs > 0) h->pairs.assign(pairs, pairs + 2 * npairs);
  Pimy40::Input in{};
  in.rho = in9[0];
  in.refShearModul = in9[1];
  in.refBulkModul = in9[2];
  in.cohesi = in9[3];
  in.peakShearStra = in9[4];
  in.frictionAng = in9[5];
  in.refPress = in9[6];
  in.pressDependCoe = in9[7];
  in.numberOfYieldSurf = static_cast<int>(in9[8]);
  in.gredu = h->pairs.empty() ? nullptr : h->pairs.data();
  const int rc = Pimy40::setup(in, h->p);
  if (rc != Pimy40::Ok) return rc;
  *out = h.release();
  return 0;
}
void fxref_pimy_destroy(fxref_pimy* h) { delete h; }
int32_t fxref_pimy_nstate() { return Pimy40::NSTATE; }
// the setup's results: residualPress, frictionAngle, cohesion, then size[1..40], modulus[1..40]
void fxref_pimy_setup_values(const fxref_pimy* h, double* out) {
  out[0] = h->p.residualPress;
  out[1] = h->p.frictionAngle;
  out[2] = h->p.cohesion;
  for (int i = 1; i <= 40; ++i) {
    out[2 + i] = h->p.size[i];
    out[42 + i] = h->p.modulus[i];
  }
}
void fxref_pimy_initial_state(const fxref_pimy* h, double* s) { Pimy40::initial_state(h->p, {s, 1}); }
// update at total strain eps (engineering shear) from `committed`: trial state, stress, tangent
void fxref_pimy_update(fxref_pimy* h, int32_t stage, const double* committed, double* trial, const double* eps,
                       double* sig, double* D) {
  h->p.loadStage = stage;
  Pimy40::update(h->p, {committed, 1}, {trial, 1}, eps, sig, reinterpret_cast<double(*)[6]>(D));
}

// ---- PressureDependMultiYield (the reference's material, 40-surface bucket), one point at a time:
// in23 = rho, refShearModul, refBulkModul, frictionAng, peakShearStra, refPress, pressDependCoe,
// PTAng, contrac, dilat1, dilat2, liquefac1, liquefac2, liquefac3, noYieldSurf, e, cs1, cs2, cs3, pa,
// c, hv, pv; pairs (gamma, G/Gmax) or NULL.
using Pdmy40 = femorax::PressureDependMultiYield<40>;
struct fxref_pdmy {
  Pdmy40::Params p{};
  std::vector<double> pairs;
};

int fxref_pdmy_create(const double* in, const double* pairs, int32_t npairs, fxref_pdmy** out) {
  auto h = std::make_unique<fxref_pdmy>();
  if (pairs && npairs > 0) h->pairs.assign(pairs, pairs + 2 * npairs);
  Pdmy40::Input d{};
  d.rho = in[0];
  d.refShearModul = in[1];
  d.refBulkModul = in[2];
  d.frictionAng = in[3];
  d.peakShearStra = in[4];
  d.refPress = in[5];
  d.pressDependCoe = in[6];
  d.phaseTransformAng = in[7];
  d.contractionParam1 = in[8];
  d.dilationParam1 = in[9];
  d.dilationParam2 = in[10];
  d.liquefactionParam1 = in[11];
  d.liquefactionParam2 = in[12];
  d.liquefactionParam4 = in[13];
  d.numberOfYieldSurf = static_cast<int>(in[14]);
  d.gredu = h->pairs.empty() ? nullptr : h->pairs.data();
  d.e = in[15];
  d.volLimit1 = in[16];
  d.volLimit2 = in[17];
  d.volLimit3 = in[18];
  d.atm = in[19];
  d.cohesi = in[20];
  d.hv = in[21];
  d.pv = in[22];
  const int rc = Pdmy40::setup(d, h->p);
  if (rc != Pdmy40::Ok) return rc;
  *out = h.release();
  return 0;
}
void fxref_pdmy_destroy(fxref_pdmy* h) { delete h; }
int32_t fxref_pdmy_nstate() { return Pdmy40::NSTATE; }
// residualPress, frictionAngle, phaseTransfAngle, stressRatioPT, strainPTOcta, size[1..40], modulus[1..40]
void fxref_pdmy_setup_values(const fxref_pdmy* h, double* out) {
  out[0] = h->p.residualPress;
  out[1] = h->p.frictionAngle;
  out[2] = h->p.phaseTransfAngle;
  out[3] = h->p.stressRatioPT;
  out[4] = h->p.strainPTOcta;
  for (int i = 1; i <= 40; ++i) {
    out[4 + i] = h->p.size[i];
    out[44 + i] = h->p.modulus[i];
  }
}
void fxref_pdmy_initial_state(const fxref_pdmy* h, double* s) { Pdmy40::initial_state(h->p, {s, 1}); }
void fxref_pdmy_update(fxref_pdmy* h, int32_t stage, const double* committed, double* trial, const double* eps,
                       double* sig, double* D) {
  h->p.loadStage = stage;
  Pdmy40::update(h->p, {committed, 1}, {trial, 1}, eps, sig, reinterpret_cast<double(*)[6]>(D));
}

}  // extern "C"
