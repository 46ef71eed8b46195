// FP64 instantiation of the 2D MHD and Poisson kernels (the parity path).
// Built with -fmad=false: no FMA contraction, so every operation rounds like
// the reference's x86-64 build.
#include "mhd2d_impl.cuh"

namespace ccb {
template struct M2Launch<double>;
}
