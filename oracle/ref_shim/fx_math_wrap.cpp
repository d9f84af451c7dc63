// Test infrastructure only: the definitions the linker's --wrap=pow,exp,log,cos sends the reference's
// calls of those C library functions to, when oracle/Makefile links _ref/libfxref_fxmath.so (the
// reference's own sources, unchanged, with the elementary functions of this library's device
// PressureDependMultiYield update, femorax_b200/csrc/fx_math.h). _ref/libfxref.so keeps the C library.
#include "fx_math.h"

extern "C" {
double __wrap_pow(double x, double y) { return fxm_pow(x, y); }
double __wrap_exp(double x) { return fxm_exp(x); }
double __wrap_log(double x) { return fxm_log(x); }
double __wrap_cos(double x) { return fxm_cos(x); }
}
