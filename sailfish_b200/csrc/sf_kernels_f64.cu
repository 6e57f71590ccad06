// FP64 instantiation of the time-step kernels.  Built with -fmad=false: every expression is
// evaluated as written (no fused multiply-add), which is how the reference's expressions are
// evaluated by the oracle, so the FP64 path reproduces the oracle bit for bit.
#include "sf_kernels.cuh"

namespace sf {
template struct Ops<double>;
}
