// 2D step schedule, FP32 form (FP32 fields, transforms and product; FP64 state and epilogue).
#include "steps2d.cuh"

namespace bastr_impl {
template cudaError_t rhs2d<float>(bastr_handle*, int, bool, bool);
}  // namespace bastr_impl
