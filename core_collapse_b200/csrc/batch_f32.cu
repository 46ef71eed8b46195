// FP32 instantiation of the batched-ensemble kernels (the bulk path).
#include "batch_impl.cuh"

namespace ccb {
template struct BatchLaunch<float>;
}
