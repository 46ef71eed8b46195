// FP64 instantiation of the 2D Euler/HLLC kernels (the parity path; -fmad=false).
#include "euler2d_impl.cuh"

namespace ccb {
template struct EHLaunch<double>;
}
