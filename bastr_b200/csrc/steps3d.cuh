// 3D step schedule: launchers of the five fused passes (pass3d.cu) and one right-hand-side
// evaluation with its stage combination.  Included by steps3d_f32.cu and steps3d_f64.cu, which
// instantiate it for one compute precision each.
#pragma once
#include "handle.cuh"
#include "pass2d.cu"   // shared pass helpers (ept_fit, groups_per_block, pack_at, ...)
#include "pass3d.cu"

namespace bastr_impl {

// ---------------------------------------------------------------------------------------
// 3D launches
// ---------------------------------------------------------------------------------------

template <typename T, typename TIN, int SET>
cudaError_t l3_zinv(bastr_handle* h, const void* S, void* MA, int ftot) {
    SIZE_CASES3(h->g.nz, {
        using P = ZInv3D<T, TIN, NN, SET>;
        auto k = k3d_zinv<T, TIN, NN, SET>;
        const size_t smem = P::smem(h->g.KZ);
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, smem, P::NT, cdiv(h->g.K * h->g.KY, P::G), &grid);
        if (e != cudaSuccess) return e;
        const double lines = (double)h->g.K * h->g.KY;
        ProfScope ps(h, SET == ZI_VG ? "k3d_zinv_vg" : "k3d_zinv",
                     lines * h->g.KZ * 3 * sizeof(cplx<TIN>) + lines * h->g.nz * P::F * sizeof(cplx<T>));
        LAUNCH(launch_k(h, k, grid, P::NT, smem, (const cplx<TIN>*)S, (cplx<T>*)MA, ftot, h->g, twp<T>(h->tw[2])));
    });
    return cudaGetLastError();
}

template <typename T, int SET>
cudaError_t l3_yinv(bastr_handle* h, const void* MA, void* MB) {
    SIZE_CASES3(h->g.ny, {
        using P = YInv3D<T, NN, SET>;
        auto k = k3d_yinv<T, NN, SET>;
        const size_t smem = P::smem(h->g.KY);
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, smem, P::NT, cdiv(h->g.K * h->g.nz, P::G), &grid);
        if (e != cudaSuccess) return e;
        const double cs = sizeof(cplx<T>);
        ProfScope ps(h, SET == YB_RHS_VG ? "k3d_yinv_vg" : "k3d_yinv",
                     (double)h->g.K * h->g.nz * (h->g.KY * P::FIN + h->g.ny * P::F) * cs);
        LAUNCH(launch_k(h, k, grid, P::NT, smem, (const cplx<T>*)MA, (cplx<T>*)MB, h->g, twp<T>(h->tw[1]),
                        h->tm3[SET == YB_RHS_VG ? TM_Y3MA10 : TM_Y3MA6]));
    });
    return cudaGetLastError();
}

template <typename T, int MODE>
cudaError_t l3_xpass(bastr_handle* h, const void* MB, void* MC, const double* pin, double* pout, double* vg) {
    SIZE_CASES3(h->g.nx, {
        using P = XPass3D<T, NN, MODE>;
        auto k = k3d_xpass<T, NN, MODE>;
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, P::SMEM, P::NT, cdiv(h->g.ny * h->g.nz, P::G), &grid);
        if (e != cudaSuccess) return e;
        if (MODE == X3_RHS_VG) h->n_vg_blocks = grid;
        const double cs = sizeof(cplx<T>), mix = (double)h->g.ny * h->g.nz * h->g.K;
        const double phys = 3.0 * h->g.nx * h->g.ny * h->g.nz * 8;
        const double b = MODE == X3_RHS ? mix * 12 * cs : MODE == X3_RHS_VG ? mix * 16 * cs
                       : MODE == X3_TO_PHYS ? mix * 3 * cs + phys : phys + mix * 3 * cs;
        ProfScope ps(h, MODE == X3_RHS_VG ? "k3d_xpass_vg" : MODE == X3_RHS ? "k3d_xpass" : "k3d_xpass_state", b);
        LAUNCH(launch_k(h, k, grid, P::NT, P::SMEM, (const cplx<T>*)MB, (cplx<T>*)MC, pin, pout, vg, h->g,
                        twp<T>(h->tw[0]), h->tm3[MODE == X3_RHS_VG ? TM_X3MB13 : TM_X3MB9]));
    });
    return cudaGetLastError();
}

template <typename T>
cudaError_t l3_yfwd(bastr_handle* h, const void* MC, void* MD) {
    SIZE_CASES3(h->g.ny, {
        using P = YFwd3D<T, NN>;
        auto k = k3d_yfwd<T, NN>;
        const size_t smem = P::smem(h->g.KY);
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, smem, P::NT, cdiv(h->g.K * h->g.nz, P::G), &grid);
        if (e != cudaSuccess) return e;
        ProfScope ps(h, "k3d_yfwd", (double)h->g.K * h->g.nz * (h->g.ny + h->g.KY) * 3 * sizeof(cplx<T>));
        LAUNCH(launch_k(h, k, grid, P::NT, smem, (const cplx<T>*)MC, (cplx<T>*)MD, h->g, twp<T>(h->tw[1])));
    });
    return cudaGetLastError();
}

template <typename T, int EPI>
cudaError_t l3_zfwd(bastr_handle* h, const void* MD, StageIO<T> io, int from_u0) {
    SIZE_CASES3(h->g.nz, {
        using P = ZFwd3D<T, NN>;
        auto k = k3d_zfwd<T, NN, EPI>;
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, P::SMEM, P::NT, cdiv(h->g.K * h->g.KY, P::G), &grid);
        if (e != cudaSuccess) return e;
        if (io.energy_part) h->n_en_blocks = grid;
        const double cs = sizeof(cplx<T>), lines = (double)h->g.K * h->g.KY;
        ProfScope ps(h, "k3d_zfwd", lines * h->g.nz * 3 * cs + epi_bytes(EPI, from_u0, lines * h->g.KZ * 3, cs));
        LAUNCH(launch_k(h, k, grid, P::NT, P::SMEM, (const cplx<T>*)MD, io, from_u0, h->g, twp<T>(h->tw[2])));
    });
    return cudaGetLastError();
}

template <typename T>
cudaError_t rhs3d(bastr_handle* h, int epi, bool from_u0, bool vg) {
    cudaError_t e;
    const int ftot = vg ? 10 : 6;
    if (from_u0) e = l3_zinv<T, double, ZI_RHS>(h, h->u0, h->ma, ftot);
    else e = l3_zinv<T, T, ZI_RHS>(h, h->us, h->ma, ftot);
    if (e != cudaSuccess) return e;
    if (vg) {
        e = l3_zinv<T, double, ZI_VG>(h, h->u0, h->ma, ftot);
        if (e != cudaSuccess) return e;
        e = l3_yinv<T, YB_RHS_VG>(h, h->ma, h->mb);
        if (e != cudaSuccess) return e;
        e = l3_xpass<T, X3_RHS_VG>(h, h->mb, h->mc, nullptr, nullptr, h->vg_part);
    } else {
        e = l3_yinv<T, YB_RHS>(h, h->ma, h->mb);
        if (e != cudaSuccess) return e;
        e = l3_xpass<T, X3_RHS>(h, h->mb, h->mc, nullptr, nullptr, nullptr);
    }
    if (e != cudaSuccess) return e;
    e = l3_yfwd<T>(h, h->mc, h->ma);
    if (e != cudaSuccess) return e;
    StageIO<T> io{h->u0, (cplx<T>*)h->us, (cplx<T>*)h->acc, nullptr, h->g.chk, h->g.err};
    const bool need_en = (epi == EPI_RK3 || epi == EPI_CN_LAST) &&
                         (h->p.forcemethod == 1 || h->p.forcemethod >= 3);
    if (need_en) io.energy_part = h->en_part;
    switch (epi) {
        case EPI_RK1: return l3_zfwd<T, EPI_RK1>(h, h->ma, io, from_u0);
        case EPI_RK2: return l3_zfwd<T, EPI_RK2>(h, h->ma, io, from_u0);
        case EPI_RK3: return l3_zfwd<T, EPI_RK3>(h, h->ma, io, from_u0);
        case EPI_CN_MID: return l3_zfwd<T, EPI_CN_MID>(h, h->ma, io, from_u0);
        case EPI_CN_LAST: return l3_zfwd<T, EPI_CN_LAST>(h, h->ma, io, from_u0);
    }
    return cudaErrorInvalidValue;
}

}  // namespace bastr_impl
