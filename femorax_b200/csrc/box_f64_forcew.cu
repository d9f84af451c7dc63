// Box kernels, F64 internal force from w = u + beta v formed beforehand: every launch shape of
// launch<double, 2>.
#include "box_kernels.cuh"

namespace fx {
namespace boxk {
template void launch<double, 2>(const BoxPlan&, const BoxArgs<double>&, cudaStream_t);
}  // namespace boxk
}  // namespace fx
