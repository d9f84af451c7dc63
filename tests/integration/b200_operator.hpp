// The reference-side binding a maintainer adds to amnp95/FemoraX to run its solvers on the
// femorax_b200 operator: a solvers::LinearOperator (src/solvers/linear_solver.hpp:57-67) over
// fx_apply_operator / fx_operator_diagonal, in the role of exec::MatrixFreeOperator
// (src/exec/matrix_free_operator.hpp:16-36). It compiles against the reference's own headers;
// tests/integration/reference_cg_driver.cpp builds it into the oracle and drives the reference's
// ConjugateGradient and Jacobi through it.
#pragma once

#include <cstdint>
#include <stdexcept>

#include "femorax_b200.h"
#include "physics/operators/element_operator.hpp"
#include "solvers/linear_solver.hpp"

namespace femorax::b200 {

// Where the solver's vectors (Kokkos views) live: device memory in the reference's CUDA build,
// host memory in a host build (Serial / OpenMP), for which the library's host-buffer calls copy.
enum class ViewMemory { Device, Host };

class B200Operator final : public solvers::LinearOperator {
 public:
  // force: a handle from fx_force_create on the compiled model; it must outlive this operator.
  B200Operator(fx_force* force, const OperatorCoefficients& k, void* stream = nullptr,
               ViewMemory memory = ViewMemory::Device)
      : force_(force), stream_(stream), memory_(memory) {
    int64_t i[9];
    check(fx_force_info(force_, i));
    info_.rows = i[0];
    info_.fields = {solvers::Field{"displacement", 0, i[0]}};
    set_coefficients(k);
  }

  // MatrixFreeOperator::set_coefficients; the symmetry follows operator_symmetry
  // (src/exec/matrix_free_operator.cpp:5-16) for the path's symmetric tangents.
  void set_coefficients(const OperatorCoefficients& k) {
    k_ = fx_coeffs{k.stiffness, k.damping, k.mass, k.initial ? 1 : 0, 0};
    const bool positive = k.stiffness >= 0.0 && k.damping >= 0.0 && k.mass >= 0.0 &&
                          (k.stiffness > 0.0 || k.mass > 0.0);
    info_.symmetry = positive ? solvers::Symmetry::SymmetricPositiveDefinite : solvers::Symmetry::Symmetric;
  }

  const solvers::OperatorInfo& info() const override { return info_; }

  // y = K_eff x; x and y never alias.
  void apply(const solvers::ConstVector& x, const solvers::Vector& y) const override {
    if (memory_ == ViewMemory::Device)
      check(fx_apply_operator(force_, k_, x.data(), y.data(), stream_));
    else
      check(fx_apply_operator_host(force_, k_, x.data(), y.data(), stream_));
  }

  // d = diag(K_eff).
  void diagonal(const solvers::Vector& d) const override {
    if (memory_ == ViewMemory::Device)
      check(fx_operator_diagonal(force_, k_, d.data(), stream_));
    else
      check(fx_operator_diagonal_host(force_, k_, d.data(), stream_));
  }

 private:
  static void check(int rc) {
    if (rc != FX_OK) throw std::runtime_error(fx_last_error());
  }
  fx_force* force_;
  fx_coeffs k_{};
  void* stream_;
  ViewMemory memory_;
  solvers::OperatorInfo info_;
};

}  // namespace femorax::b200
