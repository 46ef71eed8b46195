// FP64 instantiation of the 3D MHD kernels (the parity path; -fmad=false).
#include "mhd3d_impl.cuh"

namespace ccb {
template struct M3Launch<double>;
}
