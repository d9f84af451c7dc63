// Box kernels, F32 operator apply y = K_eff x: every launch shape of launch<float, 0>.
#include "box_kernels.cuh"

namespace fx {
namespace boxk {
template void launch<float, 0>(const BoxPlan&, const BoxArgs<float>&, cudaStream_t);
}  // namespace boxk
}  // namespace fx
