// Box kernels, F64 operator apply y = K_eff x: every launch shape of launch<double, 0>.
#include "box_kernels.cuh"

namespace fx {
namespace boxk {
template void launch<double, 0>(const BoxPlan&, const BoxArgs<double>&, cudaStream_t);
}  // namespace boxk
}  // namespace fx
