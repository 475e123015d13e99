// 3D step schedule, FP64 form, and the FP64 transforms of the state between the host's physical
// field and the truncated spectral state (set_state / get_state).
#include "steps3d.cuh"

namespace bastr_impl {

template cudaError_t rhs3d<double>(bastr_handle*, int, bool, bool);

cudaError_t state3d_to_spectral(bastr_handle* h) {
    cudaError_t e = l3_xpass<double, X3_FROM_PHYS>(h, nullptr, h->mc, h->phys, nullptr, nullptr);
    if (e != cudaSuccess) return e;
    e = l3_yfwd<double>(h, h->mc, h->ma);
    if (e != cudaSuccess) return e;
    StageIO<double> io{h->u0, nullptr, nullptr, nullptr, h->g.chk, h->g.err};
    return l3_zfwd<double, EPI_STORE>(h, h->ma, io, 0);
}

cudaError_t state3d_to_physical(bastr_handle* h) {
    cudaError_t e = l3_zinv<double, double, ZI_STATE>(h, h->u0, h->ma, 3);
    if (e != cudaSuccess) return e;
    e = l3_yinv<double, YB_STATE>(h, h->ma, h->mb);
    if (e != cudaSuccess) return e;
    return l3_xpass<double, X3_TO_PHYS>(h, h->mb, nullptr, nullptr, h->phys, nullptr);
}

}  // namespace bastr_impl
