// FP64 instantiation of the batched-ensemble kernels (built with -fmad=false,
// so an instance rounds exactly like the single-grid parity path).
#include "batch_impl.cuh"

namespace ccb {
template struct BatchLaunch<double>;
}
