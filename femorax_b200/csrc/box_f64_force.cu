// Box kernels, F64 internal force f = K (u + beta v) - body + la v: every launch shape of launch<double, 1>.
#include "box_kernels.cuh"

namespace fx {
namespace boxk {
template void launch<double, 1>(const BoxPlan&, const BoxArgs<double>&, cudaStream_t);
}  // namespace boxk
}  // namespace fx
