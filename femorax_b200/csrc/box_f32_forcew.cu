// Box kernels, F32 internal force from w = u + beta v formed beforehand: every launch shape of
// launch<float, 2>.
#include "box_kernels.cuh"

namespace fx {
namespace boxk {
template void launch<float, 2>(const BoxPlan&, const BoxArgs<float>&, cudaStream_t);
}  // namespace boxk
}  // namespace fx
