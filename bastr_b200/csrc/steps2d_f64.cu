// 2D step schedule, FP64 form, and the FP64 transforms of the state between the host's physical
// field and the truncated spectral state (set_state / get_state).
#include "steps2d.cuh"

namespace bastr_impl {

template cudaError_t rhs2d<double>(bastr_handle*, int, bool, bool);

cudaError_t state2d_to_spectral(bastr_handle* h) {
    cudaError_t e = l2_xpass<double, XM_FROM_PHYS>(h, nullptr, 0, h->mb, h->phys, nullptr, nullptr);
    if (e != cudaSuccess) return e;
    StageIO<double> io{h->u0, nullptr, nullptr, nullptr, h->g.chk, h->g.err};
    return l2_yfwd<double, EPI_STORE>(h, h->mb, io, 0);
}

cudaError_t state2d_to_physical(bastr_handle* h) {
    cudaError_t e = l2_yinv<double, double, YI_STATE>(h, h->u0, h->ma, 2);
    if (e != cudaSuccess) return e;
    return l2_xpass<double, XM_TO_PHYS>(h, h->ma, 2, nullptr, nullptr, h->phys, nullptr);
}

}  // namespace bastr_impl
