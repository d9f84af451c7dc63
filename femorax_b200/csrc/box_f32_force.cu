// Box kernels, F32 internal force f = K (u + beta v) - body + la v: every launch shape of launch<float, 1>.
#include "box_kernels.cuh"

namespace fx {
namespace boxk {
template void launch<float, 1>(const BoxPlan&, const BoxArgs<float>&, cudaStream_t);
}  // namespace boxk
}  // namespace fx
