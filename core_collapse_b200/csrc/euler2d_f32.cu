// FP32 instantiation of the 2D Euler/HLLC kernels (FMA, approximate division/sqrt;
// reductions stay in FP64).
#include "euler2d_impl.cuh"

namespace ccb {
template struct EHLaunch<float>;
}
