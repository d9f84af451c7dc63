// Test infrastructure: the reference's own ConjugateGradient and Jacobi (its sources, built into
// oracle/_ref/libfxref.so with the Kokkos-subset shim, host views) solving through the
// B200Operator binding on a femorax_b200 force handle. Built by oracle/Makefile (target
// `adapter`) into oracle/_ref/libfxadapter.so; called by tests/test_gpu_adapter.py.
#include <cstdint>
#include <exception>
#include <string>

#include "b200_operator.hpp"
#include "solvers/cg.hpp"
#include "solvers/jacobi.hpp"

namespace {
thread_local std::string g_error;
}

extern "C" {

const char* fxadapt_last_error() { return g_error.c_str(); }

// Jacobi-PCG on K_eff = k[0] K + k[1] C + k[2] M of `force` (an fx_force*): b and x host
// vectors of n entries, x the initial guess on entry. out[6] = converged, iterations, rhs_norm,
// initial_residual, final_residual, indefinite (solvers::SolveResult). Returns 0, or -1 with the
// message in fxadapt_last_error().
int fxadapt_cg_solve(void* force, int64_t n, const double* k, const double* b, double* x, double rtol,
                     int max_iterations, double* out) {
  using namespace femorax;
  try {
    b200::B200Operator op(static_cast<fx_force*>(force), OperatorCoefficients{k[0], k[1], k[2], false}, nullptr,
                          b200::ViewMemory::Host);
    if (op.info().rows != n) throw std::runtime_error("fxadapt_cg_solve: vector length is not the operator's");
    solvers::Jacobi jacobi;
    jacobi.setup(op);
    solvers::SolveOptions options;
    options.relative_tolerance = rtol;
    options.max_iterations = max_iterations;
    solvers::ConjugateGradient cg(options, 1);
    cg.setup(op, &jacobi);
    solvers::Vector xv(x, static_cast<std::size_t>(n));
    solvers::ConstVector bv(b, static_cast<std::size_t>(n));
    const solvers::SolveResult r = cg.solve(bv, xv);
    out[0] = r.converged;
    out[1] = r.iterations;
    out[2] = r.rhs_norm;
    out[3] = r.initial_residual;
    out[4] = r.final_residual;
    out[5] = r.indefinite;
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

}  // extern "C"
