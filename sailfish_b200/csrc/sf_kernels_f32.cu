// FP32 instantiation of the time-step kernels (stencils in FP32; fast-time accumulators,
// coupling column sums and set_depth in FP64).  Built with FMA contraction enabled.
#include "sf_kernels.cuh"

namespace sf {
template struct Ops<float>;
}
