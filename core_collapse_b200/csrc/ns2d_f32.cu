// FP32 instantiation of the 2D Navier-Stokes kernels (FMA, approximate
// division/sqrt; reductions and dt stay in FP64).
#include "ns2d_impl.cuh"

namespace ccb {
template struct NSLaunch<float>;
}
