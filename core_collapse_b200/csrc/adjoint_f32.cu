// FP32 instantiation of the discrete adjoint (adjoint_impl.cuh), built with the
// flags of the FP32 forward kernels (FMA contraction, approximate division and
// square root, flush-to-zero), so that its recomputation of the forward's
// intermediates rounds like the FP32 forward it reverses.
#include "adjoint_impl.cuh"

namespace ccb {
template struct Adjoint<float>;
}
