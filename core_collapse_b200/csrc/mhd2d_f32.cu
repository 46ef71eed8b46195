// FP32 instantiation of the 2D MHD and Poisson kernels (the bulk path; FMA
// contraction allowed).  Reductions inside the kernels stay in FP64.
#include "mhd2d_impl.cuh"

namespace ccb {
template struct M2Launch<float>;
}
