// Host-side structures of the library: the in-memory model, the compiled arrays, errors.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/femorax_b200.h"

namespace fx {

// Errors inside the library carry a status code; the C ABI turns them into return values.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
void set_error(const std::string& msg);

struct Group {
  fx_material mat;
  double b[3];
  bool lumped;
  std::vector<int32_t> tags, conn;  // conn: 8 node tags per element
};
struct Region {
  double alphaM, betaK, betaKinit, betaKcomm;
  std::vector<int32_t> elements;
};

}  // namespace fx

struct fx_model {
  std::vector<int32_t> tags;
  std::vector<double> coords;  // row-major, 3 per node
  std::vector<fx::Group> groups;
  std::vector<int32_t> fix_node, fix_dof;
  std::vector<int32_t> eqd_retained, eqd_constrained, eqd_dof;
  std::vector<fx::Region> regions;
  std::vector<int32_t> mass_node, mass_dof;
  std::vector<double> mass_value;
};

struct fx_compiled {
  int32_t num_nodes = 0, num_equations = 0, count = 0, padded = 0;
  std::vector<int32_t> node_tag, node_order, node_rank, element_order, node_model_index, dof_offset, eq;
  std::vector<double> coords;  // [3N] structure of arrays
  std::vector<int32_t> b_node, b_eq, b_param, b_tag, color_start, color_elements, eq_dof;
  std::vector<fx_param_set> params;
  std::vector<double> lumped_mass, lumped_alpha_mass, nodal_mass, nodal_alpha_mass;
};

namespace fx {
void compile_model(const fx_model& m, int renumbering, int simd_width, bool coloring, fx_compiled& c);
}
