// Test infrastructure only: the few io:: helpers the reference's compile and launch layers call.
// The reference defines them in src/io/model_reader.cpp next to its HDF5 reader, which cannot be
// built here (no HDF5); these are small definitions of the same functions written for the
// oracle, with the meaning their declarations in src/io/model.hpp give.
#include "io/model.hpp"

namespace femorax::io {

const char* to_string(ElementType t) {
  switch (t) {
    case ElementType::StdBrick: return "stdBrick";
    case ElementType::SSPbrick: return "SSPbrick";
    case ElementType::DispBeamColumn: return "dispBeamColumn";
    case ElementType::ForceBeamColumn: return "forceBeamColumn";
  }
  return "?";
}

int node_count(ElementType t) { return t == ElementType::DispBeamColumn || t == ElementType::ForceBeamColumn ? 2 : 8; }

bool is_section(const NDMaterial& m) { return std::holds_alternative<ElasticSection3dData>(m.data); }

const char* material_type_name(const NDMaterial& m) {
  if (std::holds_alternative<ElasticIsotropicData>(m.data)) return "ElasticIsotropic";
  if (std::holds_alternative<PressureDependMultiYieldData>(m.data)) return "PressureDependMultiYield";
  if (std::holds_alternative<PressureIndependMultiYieldData>(m.data)) return "PressureIndependMultiYield";
  return "Elastic";
}

bool has_material_stage(const NDMaterial& m) {
  return std::holds_alternative<PressureDependMultiYieldData>(m.data) ||
         std::holds_alternative<PressureIndependMultiYieldData>(m.data);
}

std::size_t Model::element_count() const {
  std::size_t n = 0;
  for (const auto& g : elements) n += g.size();
  return n;
}

}  // namespace femorax::io

// GroundMotions (src/exec/ground_motion.cpp) forwards to its H5DRM patterns; none is ever
// activated here (the DRM reader needs HDF5), so these are never reached.
#include "exec/drm_load.hpp"

namespace femorax::exec {
void DrmLoad::apply(double, const Vec&) {}
void DrmLoad::commit() {}
}  // namespace femorax::exec
