// FP32 instantiation of the 3D MHD kernels (the bulk path; FMA contraction,
// approximate division and square root).  Reductions stay in FP64.
#include "mhd3d_impl.cuh"

namespace ccb {
template struct M3Launch<float>;
}
