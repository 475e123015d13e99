// 2D step schedule: launchers of the three fused passes (pass2d.cu) and one right-hand-side
// evaluation with its stage combination.  Included by steps2d_f32.cu and steps2d_f64.cu, which
// instantiate it for one compute precision each.
#pragma once
#include "handle.cuh"
#include "pass2d.cu"

namespace bastr_impl {

// ---------------------------------------------------------------------------------------
// 2D launches
// ---------------------------------------------------------------------------------------
template <typename T, typename TIN, int SET>
cudaError_t l2_yinv(bastr_handle* h, const void* S, void* MA, int ftot) {
    SIZE_CASES(h->g.ny, {
        using P = YInv2D<T, TIN, NN, SET>;
        auto k = k2d_yinv<T, TIN, NN, SET>;
        const size_t smem = P::smem(h->g.KY);
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, smem, P::NT, cdiv(h->g.K, P::G), &grid);
        if (e != cudaSuccess) return e;
        const double K_ = h->g.K;
        ProfScope ps(h, SET == YI_VG ? "k2d_yinv_vg" : SET == YI_RHS_VG ? "k2d_yinv_rhs_vg" : "k2d_yinv",
                     K_ * h->g.KY * 2 * sizeof(cplx<TIN>) + (double)h->g.ny * K_ * P::F * sizeof(cplx<T>));
        LAUNCH(launch_k(h, k, grid, P::NT, smem, (const cplx<TIN>*)S, (cplx<T>*)MA, ftot, h->g, twp<T>(h->tw[1])));
    });
    return cudaGetLastError();
}

template <typename T, int MODE>
cudaError_t l2_xpass(bastr_handle* h, const void* MA, int ftot, void* MB, const double* pin, double* pout,
                     double* vg) {
    SIZE_CASES(h->g.nx, {
        using P = XPass2D<T, NN, MODE>;
        auto k = k2d_xpass<T, NN, MODE>;
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, P::SMEM, P::NT, cdiv(h->g.ny, P::G), &grid);
        if (e != cudaSuccess) return e;
        if (MODE == XM_RHS_VG) h->n_vg_blocks = grid;
        const double cs = sizeof(cplx<T>), mix = (double)h->g.ny * h->g.K, phys = 2.0 * h->g.nx * h->g.ny * 8;
        const double b = MODE == XM_RHS ? mix * 6 * cs : MODE == XM_RHS_VG ? mix * 8 * cs
                       : MODE == XM_TO_PHYS ? mix * 2 * cs + phys : phys + mix * 2 * cs;
        ProfScope ps(h, MODE == XM_RHS_VG ? "k2d_xpass_vg" : MODE == XM_RHS ? "k2d_xpass" : "k2d_xpass_state", b);
        // the x maps describe the compute precision's records: only that precision's product
        // modes are TMA-staged
        if (P::TMA && sizeof(T) != (h->fp32 ? 4u : 8u)) return cudaErrorInvalidValue;
        // tensor maps of the TMA-staged modes: the MA records of ftot fields (and the q pieces)
        const CUtensorMap& ta = h->tm[ftot == 8 ? TM_XA8 : TM_XA4];
        const CUtensorMap& tb = h->tm[TM_XB8];
        LAUNCH(launch_k(h, k, grid, P::NT, P::SMEM, (const cplx<T>*)MA, ftot, (cplx<T>*)MB, pin, pout, vg, h->g,
                        twp<T>(h->tw[0]), ta, tb));
    });
    return cudaGetLastError();
}

template <typename T, int EPI>
cudaError_t l2_yfwd(bastr_handle* h, const void* MB, StageIO<T> io, int from_u0) {
    SIZE_CASES(h->g.ny, {
        using P = YFwd2D<T, NN>;
        auto k = k2d_yfwd<T, NN, EPI>;
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, P::SMEM, P::NT, cdiv(h->g.K, P::G), &grid);
        if (e != cudaSuccess) return e;
        if (io.energy_part) h->n_en_blocks = grid;
        const double cs = sizeof(cplx<T>);
        ProfScope ps(h, "k2d_yfwd", (double)h->g.K * h->g.ny * 2 * cs +
                                    epi_bytes(EPI, from_u0, (double)h->g.K * h->g.KY * 2, cs));
        LAUNCH(launch_k(h, k, grid, P::NT, P::SMEM, (const cplx<T>*)MB, io, from_u0, h->g, twp<T>(h->tw[1]),
                        h->tm[sizeof(T) == 8 ? TM_YMB64 : TM_YMB32]));
    });
    return cudaGetLastError();
}

template <typename T, int EPI>
cudaError_t l2_yfwd_inv(bastr_handle* h, const void* MB, StageIO<T> io, int from_u0, void* MA) {
    SIZE_CASES(h->g.ny, {
        using P = YFwdInv2D<T, NN>;
        auto k = k2d_yfwd_inv<T, NN, EPI>;
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, P::SMEM, P::NT, cdiv(h->g.K, P::G), &grid);
        if (e != cudaSuccess) return e;
        const double cs = sizeof(cplx<T>);
        ProfScope ps(h, "k2d_yfwd_inv", (double)h->g.K * h->g.ny * 2 * cs +
                                        epi_bytes(EPI, from_u0, (double)h->g.K * h->g.KY * 2, cs) +
                                        (double)h->g.ny * h->g.K * 4 * cs);
        LAUNCH(launch_k(h, k, grid, P::NT, P::SMEM, (const cplx<T>*)MB, io, from_u0, h->g, twp<T>(h->tw[1]),
                        (cplx<T>*)MA, h->tm[sizeof(T) == 8 ? TM_YMB64 : TM_YMB32]));
    });
    return cudaGetLastError();
}


// One right-hand-side evaluation F(u_s) and its combination, 2D.  Stages after the first find
// their pass A already done when the previous stage's forward pass handed its stage input on
// (k2d_yfwd_inv, h->ma_ready).
template <typename T>
cudaError_t rhs2d(bastr_handle* h, int epi, bool from_u0, bool vg) {
    cudaError_t e = cudaSuccess;
    const int ftot = vg ? 8 : 4;
    if (from_u0 && vg) e = l2_yinv<T, double, YI_RHS_VG>(h, h->u0, h->ma, ftot);
    else if (from_u0) e = l2_yinv<T, double, YI_RHS>(h, h->u0, h->ma, ftot);
    else if (!h->ma_ready || vg) e = l2_yinv<T, T, YI_RHS>(h, h->us, h->ma, ftot);
    h->ma_ready = false;
    if (e != cudaSuccess) return e;
    if (vg) {
        if (!from_u0) {   // the statistics are of the state u0
            e = l2_yinv<T, double, YI_VG>(h, h->u0, h->ma, ftot);
            if (e != cudaSuccess) return e;
        }
        e = l2_xpass<T, XM_RHS_VG>(h, h->ma, ftot, h->mb, nullptr, nullptr, h->vg_part);
    } else {
        e = l2_xpass<T, XM_RHS>(h, h->ma, ftot, h->mb, nullptr, nullptr, nullptr);
    }
    if (e != cudaSuccess) return e;
    StageIO<T> io{h->u0, (cplx<T>*)h->us, (cplx<T>*)h->acc, nullptr, h->g.chk, h->g.err};
    const bool need_en = (epi == EPI_RK3 || epi == EPI_CN_LAST) &&
                         (h->p.forcemethod == 1 || h->p.forcemethod >= 3);
    if (need_en) io.energy_part = h->en_part;
    if (BASTR_FUSE_Y && (epi == EPI_RK1 || epi == EPI_RK2 || epi == EPI_CN_MID)) {
        h->ma_ready = true;
        switch (epi) {
            case EPI_RK1: return l2_yfwd_inv<T, EPI_RK1>(h, h->mb, io, from_u0, h->ma);
            case EPI_RK2: return l2_yfwd_inv<T, EPI_RK2>(h, h->mb, io, from_u0, h->ma);
            case EPI_CN_MID: return l2_yfwd_inv<T, EPI_CN_MID>(h, h->mb, io, from_u0, h->ma);
        }
    }
    switch (epi) {
        case EPI_RK1: return l2_yfwd<T, EPI_RK1>(h, h->mb, io, from_u0);
        case EPI_RK2: return l2_yfwd<T, EPI_RK2>(h, h->mb, io, from_u0);
        case EPI_RK3: return l2_yfwd<T, EPI_RK3>(h, h->mb, io, from_u0);
        case EPI_CN_MID: return l2_yfwd<T, EPI_CN_MID>(h, h->mb, io, from_u0);
        case EPI_CN_LAST: return l2_yfwd<T, EPI_CN_LAST>(h, h->mb, io, from_u0);
    }
    return cudaErrorInvalidValue;
}

}  // namespace bastr_impl
