// 3D step schedule, FP32 form (FP32 fields, transforms and product; FP64 state and epilogue).
#include "steps3d.cuh"

namespace bastr_impl {
template cudaError_t rhs3d<float>(bastr_handle*, int, bool, bool);
}  // namespace bastr_impl
