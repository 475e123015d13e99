// C ABI of the B200 Burgers time step: handle creation, the step loop with its diagnostics and
// forcing, state transfer, records, profiling, and the post-processing entry points.  The pass
// schedules of the right-hand side live in steps2d_*.cu / steps3d_*.cu.
#include "handle.cuh"
#include "diag.cu"
#include "fullfft.cu"
#include "closure.cu"
#include "transfer.cu"
#include "hitgen.cu"
#include "subgrid.cu"

using namespace bastr_impl;

namespace {

// One axis of the full-grid transform on the device array A (complex, [nz][ny][nx]).
// One axis of the full-grid transform of a complex grid A of extents ns[3] ([nz][ny][nx]) with
// the twiddle table tw of that axis's length.
template <bool INV>
cudaError_t full_axis_n(bastr_handle* h, double2* A, const int ns[3], int axis, double scale, const double2* tw) {
    const long long total = (long long)ns[0] * ns[1] * ns[2];
    const int N = ns[axis];
    const int nlines = (int)(total / N);
    const long long S = axis == 0 ? 1 : axis == 1 ? ns[0] : (long long)ns[0] * ns[1];
    const long long R = axis == 1 ? (long long)ns[0] * ns[1] : ns[0];
    SIZE_CASES(N, {
        using P = FullLine<NN>;
        auto k = k_full_axis<NN, INV>;
        int grid = 1;
        cudaError_t e = persistent_grid(h, k, P::SMEM, P::NT, cdiv(nlines, P::G), &grid);
        if (e != cudaSuccess) return e;
        ProfScope ps(h, "k_full_axis", (double)total * 32);
        LAUNCH(launch_k(h, k, grid, P::NT, P::SMEM, A, ns[0], S, R, nlines, scale, tw));
    });
    return cudaGetLastError();
}

// One axis of the full-grid transform on the handle's own grid.
template <bool INV> cudaError_t full_axis(bastr_handle* h, double2* A, int axis, double scale) {
    const int ns[3] = {h->g.nx, h->g.ny, h->g.nz};
    return full_axis_n<INV>(h, A, ns, axis, scale, (const double2*)h->tw[axis].d64);
}

// bastr_fft: host array -> the handle's physical-field buffer (2 or 3 doubles per point, so a
// complex grid fits) -> one pass per axis -> host.  dir -1: forward, scaled 1/N on its last axis.
int full_fft(bastr_handle* h, double* array, int dir) {
    const Geo& g = h->g;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    double2* A = reinterpret_cast<double2*>(h->phys);
    CK(cudaMemcpyAsync(A, array, n * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
    for (int a = 0; a < g.d; ++a) {
        const double scale = (dir < 0 && a == g.d - 1) ? g.inv_n : 1.0;
        if (dir < 0) CK(full_axis<false>(h, A, a, scale));
        else CK(full_axis<true>(h, A, a, scale));
    }
    CK(cudaMemcpyAsync(array, A, n * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return BASTR_OK;
}

// ---------------------------------------------------------------------------------------
// dimension-generic step pieces
// ---------------------------------------------------------------------------------------
cudaError_t launch_rhs(bastr_handle* h, int epi, bool from_u0, bool vg) {
    if (h->g.d == 2) return h->fp32 ? rhs2d<float>(h, epi, from_u0, vg) : rhs2d<double>(h, epi, from_u0, vg);
    return h->fp32 ? rhs3d<float>(h, epi, from_u0, vg) : rhs3d<double>(h, epi, from_u0, vg);
}

// halt_code: the value the spectra kernel stores in the handle's stop word when Es+Ed is NaN
// (the step's record slot + 1), 0 outside a batch of steps.
cudaError_t launch_spectra(bastr_handle* h, double* rec, double* shells_out, unsigned int halt_code) {
    if (h->n_items > 0) {
        ProfScope ps(h, "k_spectra", (double)h->n_disk * (h->g.d * 16 + 4));
        if (h->g.d == 2)
            LAUNCH(launch_k(h, k_spectra_fused<2, 256>, h->n_items, 256, 0, h->u0, h->g, h->pend, h->sp_modes,
                            h->sp_item_lo, h->sp_item_part, h->done + T_SPECTRA, h->sp_shell_item, h->nshell,
                            h->allkmax, rec, shells_out, halt_code));
        else
            LAUNCH(launch_k(h, k_spectra_fused<3, 256>, h->n_items, 256, 0, h->u0, h->g, h->pend, h->sp_modes,
                            h->sp_item_lo, h->sp_item_part, h->done + T_SPECTRA, h->sp_shell_item, h->nshell,
                            h->allkmax, rec, shells_out, halt_code));
    } else {
        ProfScope ps(h, "k_spectra_final", 0);
        LAUNCH(launch_k(h, k_spectra_items_final<256>, 1, 256, 0, h->sp_item_part, h->sp_shell_item, h->nshell,
                                                              h->allkmax, rec, shells_out, h->pend, h->g,
                                                              halt_code));
    }
    h->scale_pending = false;
    return cudaGetLastError();
}

// The forcing of a step, and the velocity-gradient statistics of the step (when vg) in the same
// kernel (one block each, side by side); without forcing they get their own launch.
cudaError_t launch_forcing(bastr_handle* h, double* rec, bool vg) {
    const int m = h->p.forcemethod;
    const double* vgp = vg ? h->vg_part : nullptr;
    const int vgn = vg ? h->n_vg_blocks : 0;
    if (m == 0) {
        if (vg) {
            ProfScope ps(h, "k_velgrad_final", (double)h->n_vg_blocks * 64);
            LAUNCH(launch_k(h, k_velgrad_final<256>, 1, 256, 0, h->vg_part, h->n_vg_blocks, h->g, rec));
        }
        return cudaGetLastError();
    }
    if (m == 1) {
        ProfScope ps(h, "k_force_linear", (double)h->n_en_blocks * 8);
        LAUNCH(launch_k(h, k_force_linear<256>, vgn > 0 ? 2 : 1, 256, 0, h->en_part, h->n_en_blocks, rec, h->p.target_energy, h->pend,
                        vgp, vgn, h->g));
        h->scale_pending = true;
        return cudaGetLastError();
    }
    if (m >= 3) {
        ProfScope ps(h, "k_sum_partials", (double)h->n_en_blocks * 8);
        LAUNCH(launch_k(h, k_sum_partials<256>, 1, 256, 0, h->en_part, h->n_en_blocks, 1.0, rec, R_ENERGY, h->g));
    }
    {
        const int proj = (m == 5 && h->g.d == 2 && h->p.lprojectd) ? 1 : 0;
        ProfScope ps(h, "k_force_band", 0);
        if (h->g.d == 2)
            LAUNCH(launch_k(h, k_force_band<2, 256>, vgn > 0 ? 2 : 1, 256, 0, h->u0, h->g, m, h->p.forcek, h->p.target_energy, proj, rec,
                            h->rng, vgp, vgn, (const int*)h->sp_modes, h->band_lo, h->band_hi));
        else
            LAUNCH(launch_k(h, k_force_band<3, 256>, vgn > 0 ? 2 : 1, 256, 0, h->u0, h->g, m, h->p.forcek, h->p.target_energy, proj, rec,
                            h->rng, vgp, vgn, (const int*)h->sp_modes, h->band_lo, h->band_hi));
    }
    return cudaGetLastError();
}

// One iteration of the main loop body for record slot `slot`.
cudaError_t launch_step(bastr_handle* h, int slot, bool vg) {
    double* rec = h->rec + (size_t)slot * R_COUNT;
    double* sh = h->shells_dev + (size_t)slot * 2 * (h->allkmax + 1);
    cudaError_t e = launch_spectra(h, rec, sh, (unsigned int)slot + 1u);
    if (e != cudaSuccess) return e;
    if (h->p.timemethod == 1) {
        // the statistics' partials (first stage) stay untouched until the forcing kernel sums them
        e = launch_rhs(h, EPI_RK1, true, vg);
        if (e != cudaSuccess) return e;
        e = launch_rhs(h, EPI_RK2, false, false);
        if (e != cudaSuccess) return e;
        e = launch_rhs(h, EPI_RK3, false, false);
        if (e != cudaSuccess) return e;
    } else {
        for (int s = 1; s <= 6; ++s) {
            e = launch_rhs(h, s == 6 ? EPI_CN_LAST : EPI_CN_MID, s == 1, vg && s == 1);
            if (e != cudaSuccess) return e;
        }
    }
    return launch_forcing(h, rec, vg);
}

int count_launches(bastr_handle* h, bool vg) {
    int n = 1;                                      // spectra (finished by its last block)
    const int per_rhs = h->g.d == 2 ? 3 : 5;
    const int nrhs = h->p.timemethod == 1 ? 3 : 6;
    n += per_rhs * nrhs;
    if (h->g.d == 2 && BASTR_FUSE_Y) n -= nrhs - 1;  // pass A of every stage but the first is fused
    if (h->g.d == 2 && vg) n -= 1;                   // 2D: one pass A makes the product and statistics fields
    const int m = h->p.forcemethod;
    if (vg) n += m == 0 ? 2 : 1;                    // extra inverse pass; the final reduction runs in
                                                    // the forcing kernel, or alone without forcing
    if (m == 1) n += 1;
    else if (m == 2) n += 1;
    else if (m == 3 || m == 4) n += 2;
    else if (m == 5) n += 2;
    return n;
}

void host_twiddles(int n, std::vector<double2>& t64, std::vector<float2>& t32) {
    t64.resize(n);
    t32.resize(n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < n; ++m) {
        const long double a = -2.0L * pi * (long double)m / (long double)n;
        const double c = (double)cosl(a), s = (double)sinl(a);
        t64[m] = make_double2(c, s);
        t32[m] = make_float2((float)cosl(a), (float)sinl(a));
    }
}

// Shell geometry over the full grid: Ecount and kn (solution.F90:974-995).
void host_shells(bastr_handle* h) {
    const int am = h->allkmax;
    std::vector<double> ksum(am + 1, 0.0);
    std::vector<int64_t> cnt(am + 1, 0);
    auto wav = [](int i, int n) { return i <= n / 2 ? i : i - n; };
    const int nx = h->g.nx, ny = h->g.ny, nz = h->g.d == 3 ? h->g.nz : 1;
    const double lim = (am + 0.5) * (am + 0.5);
    for (int k = 0; k < nz; ++k) {
        const int kz = h->g.d == 3 ? wav(k, nz) : 0;
        for (int j = 0; j < ny; ++j) {
            const int ky = wav(j, ny);
            const double r2 = (double)ky * ky + (double)kz * kz;
            if (r2 > lim) continue;
            for (int i = 0; i < nx; ++i) {
                const int kx = wav(i, nx);
                const double m = r2 + (double)kx * kx;
                if (m > lim) continue;
                const double kk = std::sqrt(m);
                const int s = (int)std::floor(kk / 1.0 + 0.5);
                if (s <= am) {
                    cnt[s] += 1;
                    ksum[s] += kk;
                }
            }
        }
    }
    h->kn.assign(am + 1, 0.0);
    h->ecount = cnt;
    h->kn[0] = ksum[0];
    for (int s = 1; s <= am; ++s) h->kn[s] = ksum[s] / (double)cnt[s];
}

template <typename P> void dev_alloc(bastr_handle* h, P** ptr, size_t bytes, cudaError_t& st) {
    if (st != cudaSuccess) return;
    void* q = nullptr;
    st = cudaMalloc(&q, bytes ? bytes : 16);
    if (st == cudaSuccess) {
        st = cudaMemset(q, 0, bytes ? bytes : 16);
        h->dev_bytes += (int64_t)bytes;
    }
    if (st == cudaSuccess) st = track_alloc(h, q, bytes ? bytes : 16);
    *ptr = (P*)q;
}

void free_all(bastr_handle* h) {
    void* ptrs[] = {h->u0, h->us, h->acc, h->ma, h->mb, h->mc, h->phys, h->vg_part, h->en_part, h->done, h->pend, h->rng, h->closure_buf, h->tr_buf, h->tr_modes, h->hg_part,
                    h->sg_buf, h->sg_tw,
                    h->rec, h->shells_dev, h->sp_modes, h->sp_item_lo, h->sp_shell_item,
                    h->sp_item_part, h->chk_table};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    for (auto& t : h->tw) {
        if (t.d64) cudaFree(t.d64);
        if (t.d32) cudaFree(t.d32);
    }
    if (h->stage_dev) cudaFree(h->stage_dev);
    if (h->stage_host) cudaFreeHost(h->stage_host);
    for (cudaEvent_t ev : h->ev_pool) cudaEventDestroy(ev);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
}

// Applies a linear-forcing scale that the next step's spectra would otherwise apply, so that the
// state the host reads is the one the reference holds after its forcing.
cudaError_t flush_pending_scale(bastr_handle* h) {
    if (!h->scale_pending) return cudaSuccess;
    k_apply_pending<<<148 * 4, 256, 0, h->stream>>>(h->u0, h->n_state, h->pend);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(h->pend, 0, sizeof(double2), h->stream);
    h->scale_pending = false;
    return e;
}

// Physical <-> truncated spectral state, always in FP64.
cudaError_t to_spectral(bastr_handle* h) {
    return h->g.d == 2 ? state2d_to_spectral(h) : state3d_to_spectral(h);
}

cudaError_t to_physical(bastr_handle* h) {
    return h->g.d == 2 ? state2d_to_physical(h) : state3d_to_physical(h);
}

}  // namespace

// =========================================================================================
// exported C ABI
// =========================================================================================
extern "C" {

int bastr_create(const bastr_params* p, bastr_handle** out) {
    if (!p || !out) return BASTR_E_INVALID;
    *out = nullptr;
    bastr_handle* h = new bastr_handle();
    h->p = *p;
    const int d = p->ka == 0 ? 2 : 3;
    *out = h;   // also on failure, so that the caller can read the message; destroy it either way
    if (p->ja == 0) return fail(h, BASTR_E_INVALID, "1D case is not implemented yet!");
    if (p->timemethod != 1 && p->timemethod != 2) { int r = fail(h, BASTR_E_INVALID, "Undefined time method"); return r; }
    if (p->forcemethod < 0 || p->forcemethod > 5) { int r = fail(h, BASTR_E_INVALID, "forcemethod %d", p->forcemethod); return r; }
    if (p->precision != BASTR_FP64 && p->precision != BASTR_FP32) { int r = fail(h, BASTR_E_INVALID, "precision"); return r; }
    const int nz = d == 3 ? p->ka : 1;
    if (!is_pow2(p->ia) || !is_pow2(p->ja) || (d == 3 && !is_pow2(p->ka))) {
        int r = fail(h, BASTR_E_UNSUPPORTED, "grid %dx%dx%d: each extent must be a power of two in [16, 2048]",
                     p->ia, p->ja, p->ka);
        return r;
    }
    const int K = p->ia / 3;
    if (p->ja < 2 * K || (d == 3 && p->ka < 2 * K)) {
        int r = fail(h, BASTR_E_UNSUPPORTED, "ja and ka must be at least 2*floor(ia/3) (Nyquist modes dealiased)");
        return r;
    }
    if (d == 3 && (p->ia > 512 || p->ja > 512 || p->ka > 512)) {
        int r = fail(h, BASTR_E_UNSUPPORTED, "3D extents above 512 are not built");
        return r;
    }
    h->fp32 = p->precision == BASTR_FP32;
    Geo& g = h->g;
    g.nx = p->ia; g.ny = p->ja; g.nz = nz; g.d = d; g.K = K;
    g.KY = 2 * K - 1; g.KZ = d == 3 ? 2 * K - 1 : 1;
    g.lproject = p->lprojectd ? 1 : 0;
    g.ps = 1;
    g.nu = p->reynolds == 0.0 ? 0.0 : [&] {
        const double tc = 110.4 / p->ref_tem, tc1 = 1.0 + tc;   // miucal(1.d0), solution.F90:1315-1329
        return 1.0 * std::sqrt(1.0) * tc1 / (1.0 + tc);
    }() / p->reynolds;
    g.dt = p->deltat;
    g.inv_n = 1.0 / ((double)p->ia * (double)p->ja * (double)nz);
    h->allkmax = std::min(p->ia / 3, p->kmax);
    if (h->allkmax < 0) h->allkmax = 0;
    h->nshell = K + 1;
    h->device = p->device;

    if (cudaSetDevice(h->device) != cudaSuccess) return fail(h, BASTR_E_CUDA, "cudaSetDevice(%d) failed", h->device);
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;

    const size_t cs = h->fp32 ? sizeof(float2) : sizeof(double2);
    const size_t npts = (size_t)g.nx * g.ny * g.nz;
    cudaError_t st = cudaSuccess;
    if (d == 2) {
        h->n_state = (size_t)K * g.KY * 2;
        const size_t ma = std::max((size_t)g.ny * K * 8 * cs, (size_t)g.ny * K * 2 * sizeof(double2));
        const size_t mb = (size_t)K * g.ny * 2 * std::max(cs, sizeof(double2));
        dev_alloc(h, &h->ma, ma, st);
        dev_alloc(h, &h->mb, mb, st);
        h->n_vg_blocks = 1;   // set by the launches (persistent grids)
        h->n_en_blocks = 1;
    } else {
        g.ps = (((long long)K * g.KY * g.KZ + 31) / 32) * 32;   // component planes, 256-byte aligned
        h->n_state = (size_t)g.ps * 3;
        size_t ma, mb, mc;
        sizes3d(h, cs, ma, mb, mc);
        dev_alloc(h, &h->ma, ma, st);
        dev_alloc(h, &h->mb, mb, st);
        dev_alloc(h, &h->mc, mc, st);
        h->n_vg_blocks = 1;   // set by the launches (persistent grids)
        h->n_en_blocks = 1;
    }
    dev_alloc(h, &h->u0, h->n_state * sizeof(double2), st);
    dev_alloc(h, &h->us, h->n_state * cs, st);
    dev_alloc(h, &h->acc, h->n_state * cs, st);
    dev_alloc(h, &h->phys, (size_t)d * npts * sizeof(double), st);
    // partial sums: at most one per line group of the passes that produce them
    dev_alloc(h, &h->done, kTickets * sizeof(unsigned int), st);
    dev_alloc(h, &h->pend, sizeof(double2), st);
    dev_alloc(h, &h->rng, sizeof(unsigned long long), st);
    dev_alloc(h, &h->vg_part, (size_t)std::max(g.ny * g.nz, 1) * 8 * sizeof(double), st);
    dev_alloc(h, &h->en_part, (size_t)std::max(K * g.KY, 1) * sizeof(double), st);
    dev_alloc(h, &h->rec, (size_t)kChunk * R_COUNT * sizeof(double), st);
    dev_alloc(h, &h->shells_dev, (size_t)kChunk * 2 * (h->allkmax + 1) * sizeof(double), st);
    if (st != cudaSuccess) return fail(h, BASTR_E_CUDA, "device allocation failed: %s", cudaGetErrorString(st));
    g.err = h->done + T_ERR;
    if (d == 2) {
        // TMA tensor maps of the 2D mixed-field buffers (compute precision; see TensorMapSlot)
        const uint64_t el = cs / 2, RB = 4 * cs, NY = g.ny, KK = K;
        const uint32_t BK = (uint32_t)std::min(K, 256), BY = (uint32_t)std::min(g.ny / 2, 256);
        const int swa = (int)RB;                       // 32 (FP32) / 64 (FP64)
        const int swb = 2 * cs == 32 ? 32 : 0;
        const uint64_t d4[4] = {8, NY, 1, KK}, s4[3] = {RB, NY * RB, NY * RB};
        const uint64_t d8[4] = {8, NY, 2, KK}, s8[3] = {RB, NY * RB, 2 * NY * RB};
        const uint32_t ba[4] = {8, 1, 1, BK}, bb[4] = {4, 1, 1, BK};
        // MB records of FP32 (32 bytes) and FP64 (64 bytes) values; MB holds the FP64 layout always
        const uint64_t dy[3] = {8, KK, NY / 2}, sy32[2] = {32, KK * 32}, sy64[2] = {64, KK * 64};
        const uint32_t by[3] = {8, 1, BY};
        const bool ok = encode_map(h, &h->tm[TM_XA4], h->ma, (int)el, 4, d4, s4, ba, swa) &&
                        encode_map(h, &h->tm[TM_XA8], h->ma, (int)el, 4, d8, s8, ba, swa) &&
                        encode_map(h, &h->tm[TM_XB8], h->ma, (int)el, 4, d8, s8, bb, swb) &&
                        encode_map(h, &h->tm[TM_YMB32], h->mb, 4, 3, dy, sy32, by, 0) &&
                        encode_map(h, &h->tm[TM_YMB64], h->mb, 8, 3, dy, sy64, by, 64);
        if (!ok) return fail(h, BASTR_E_CUDA, "cuTensorMapEncodeTiled rejected a mixed-field tensor map, or it reaches past its buffer");
    } else if (cs == sizeof(float2) && K <= 256 && g.KY <= 256) {
        // TMA tensor maps of the FP32 3D passes (see TensorMapSlot3): MB [z][kx][f][y] for the x
        // pass (4 consecutive y x every field x every kx x 1 z plane, 32-byte swizzle) and
        // MA [kx][kyi][f][z] for the y-inverse pass (4 consecutive z x every field and one more x
        // every kyi x 1 kx, 32-byte swizzle)
        const uint64_t NY = g.ny, KK = K, NZ = g.nz, KY = g.KY;
        bool ok = true;
        const int fins[2] = {9, 13};
        for (int m = 0; m < 2; ++m) {
            const uint64_t F = fins[m];
            const uint64_t dm[4] = {2 * NY, F, KK, NZ}, sm[3] = {NY * 8, F * NY * 8, KK * F * NY * 8};
            const uint32_t bx[4] = {8, (uint32_t)F, (uint32_t)KK, 1};
            ok = ok && encode_map(h, &h->tm3[m], h->mb, 4, 4, dm, sm, bx, 32);
        }
        const int finy[2] = {6, 10};
        for (int m = 0; m < 2; ++m) {
            const uint64_t F = finy[m];
            const uint64_t dm[4] = {2 * NZ, F, KY, KK}, sm[3] = {NZ * 8, F * NZ * 8, KY * F * NZ * 8};
            const uint32_t bx[4] = {8, (uint32_t)F + 1, (uint32_t)KY, 1};   // one field past MA's: zeros
            ok = ok && encode_map(h, &h->tm3[TM_Y3MA6 + m], h->ma, 4, 4, dm, sm, bx, 32);
        }
        if (!ok) return fail(h, BASTR_E_CUDA, "cuTensorMapEncodeTiled rejected a 3D mixed-field tensor map, or it reaches past its buffer");
    }

    const int ns[3] = {g.nx, g.ny, d == 3 ? g.nz : 0};
    for (int a = 0; a < 3; ++a) {
        if (!ns[a]) continue;
        std::vector<double2> t64;
        std::vector<float2> t32;
        host_twiddles(ns[a], t64, t32);
        h->tw[a].n = ns[a];
        CK(cudaMalloc(&h->tw[a].d64, ns[a] * sizeof(double2)));
        CK(cudaMalloc(&h->tw[a].d32, ns[a] * sizeof(float2)));
        CK(track_alloc(h, h->tw[a].d64, ns[a] * sizeof(double2)));
        CK(track_alloc(h, h->tw[a].d32, ns[a] * sizeof(float2)));
        CK(cudaMemcpy(h->tw[a].d64, t64.data(), ns[a] * sizeof(double2), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->tw[a].d32, t32.data(), ns[a] * sizeof(float2), cudaMemcpyHostToDevice));
    }
    host_shells(h);
    {
        // kept modes grouped by shell nint(|k|) (counting sort, increasing offset within a shell)
        const long long K2 = (long long)K * K;
        const int KZ = g.KZ, KYv = g.KY;
        std::vector<int> cnt(h->nshell + 1, 0);
        auto shell_of = [](long long m) { return (int)std::floor(std::sqrt((double)m) + 0.5); };
        auto each_mode = [&](auto&& fn) {
            for (int kx = 0; kx < K; ++kx)
                for (int kyi = 0; kyi < KYv; ++kyi) {
                    const long long ky = kyi < K ? kyi : kyi - KYv;
                    const long long r = (long long)kx * kx + ky * ky;
                    if (r >= K2) continue;
                    for (int kzi = 0; kzi < KZ; ++kzi) {
                        const long long kz = d == 3 ? (kzi < K ? kzi : kzi - KZ) : 0;
                        const long long m = r + kz * kz;
                        if (m == 0 || m >= K2) continue;
                        fn((int)(((long long)kx * KYv + kyi) * KZ + kzi), shell_of(m));
                    }
                }
        };
        each_mode([&](int, int sh) { cnt[sh + 1]++; });
        for (int i = 1; i <= h->nshell; ++i) cnt[i] += cnt[i - 1];
        std::vector<int> modes(cnt[h->nshell]);
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        each_mode([&](int idx, int sh) { modes[fill[sh]++] = idx; });
        h->n_disk = modes.size() + 1;   // plus the k = 0 mode
        constexpr int kItem = BASTR_SPECTRA_ITEM;   // list entries per work item
        std::vector<int> item_lo, shell_item(h->nshell + 1, 0);
        for (int sh = 0; sh < h->nshell; ++sh) {
            shell_item[sh] = (int)item_lo.size();
            for (int a = cnt[sh]; a < cnt[sh + 1]; a += kItem) item_lo.push_back(a);
        }
        shell_item[h->nshell] = (int)item_lo.size();
        h->n_items = (int)item_lo.size();
        item_lo.push_back(cnt[h->nshell]);
        // the band of the band-forcing methods: shell forcek of the list (empty past the last shell)
        const int fk = p->forcek;
        h->band_lo = fk >= 1 && fk < h->nshell ? cnt[fk] : cnt[h->nshell];
        h->band_hi = fk >= 1 && fk < h->nshell ? cnt[fk + 1] : cnt[h->nshell];
        dev_alloc(h, &h->sp_modes, std::max<size_t>(modes.size(), 1) * sizeof(int), st);
        dev_alloc(h, &h->sp_item_lo, item_lo.size() * sizeof(int), st);
        dev_alloc(h, &h->sp_shell_item, shell_item.size() * sizeof(int), st);
        dev_alloc(h, &h->sp_item_part, (size_t)std::max(h->n_items, 1) * 4 * sizeof(double), st);
        if (st != cudaSuccess) return fail(h, BASTR_E_CUDA, "device allocation failed: %s", cudaGetErrorString(st));
        if (!modes.empty())
            CK(cudaMemcpy(h->sp_modes, modes.data(), modes.size() * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->sp_item_lo, item_lo.data(), item_lo.size() * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->sp_shell_item, shell_item.data(), shell_item.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    h->launches_per_step = count_launches(h, p->velgrad_every > 0);
    CK(cudaDeviceSynchronize());
    return BASTR_OK;
}

int bastr_destroy(bastr_handle* h) {
    if (!h) return BASTR_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return BASTR_OK;
}

int bastr_set_state(bastr_handle* h, const double* u1, const double* u2, const double* u3) {
    NvtxRange range("bastr_set_state");
    if (!h || !u1 || !u2 || (h->g.d == 3 && !u3)) return fail(h, BASTR_E_INVALID, "null field pointer");
    CK(cudaSetDevice(h->device));
    const size_t npts = (size_t)h->g.nx * h->g.ny * h->g.nz;
    const double* src[3] = {u1, u2, u3};
    for (int c = 0; c < h->g.d; ++c)
        CK(cudaMemcpyAsync(h->phys + c * npts, src[c], npts * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(to_spectral(h));
    if (h->scale_pending) {   // a new state replaces the one the scale was meant for
        CK(cudaMemsetAsync(h->pend, 0, sizeof(double2), h->stream));
        h->scale_pending = false;
    }
    CK(cudaStreamSynchronize(h->stream));
    h->have_state = true;
    return BASTR_OK;
}

int bastr_get_state(bastr_handle* h, double* u1, double* u2, double* u3) {
    NvtxRange range("bastr_get_state");
    if (!h || !u1 || !u2 || (h->g.d == 3 && !u3)) return fail(h, BASTR_E_INVALID, "null field pointer");
    if (!h->have_state) return fail(h, BASTR_E_STATE, "no state set");
    CK(cudaSetDevice(h->device));
    CK(flush_pending_scale(h));
    CK(to_physical(h));
    const size_t npts = (size_t)h->g.nx * h->g.ny * h->g.nz;
    double* dst[3] = {u1, u2, u3};
    for (int c = 0; c < h->g.d; ++c)
        CK(cudaMemcpyAsync(dst[c], h->phys + c * npts, npts * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return BASTR_OK;
}

int bastr_set_counters(bastr_handle* h, int64_t nstep, double time) {
    if (!h) return BASTR_E_INVALID;
    h->nstep = nstep;
    h->time = time;
    // the random-phase forcing stream continues from the step counter after a restart
    const unsigned long long ctr = (unsigned long long)nstep;
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->rng, &ctr, sizeof(ctr), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return BASTR_OK;
}

int bastr_get_counters(bastr_handle* h, int64_t* nstep, double* time) {
    if (!h) return BASTR_E_INVALID;
    if (nstep) *nstep = h->nstep;
    if (time) *time = h->time;
    return BASTR_OK;
}

}  // extern "C"

namespace {

// Per-step records of the last batch (device slots 0..nsteps-1, R_COUNT doubles each) -> the
// caller's bastr_step_out array, with nstep/time as the reference counts them.
void decode_records(const bastr_handle* h, const double* rec, int nsteps, bastr_step_out* out) {
    const int64_t n0 = h->batch_n0;
    double t = h->batch_t0;   // times accumulate exactly as the reference's time = time + deltat
    for (int i = 0; i < nsteps; ++i) {
        if (out) {
            const double* r = &rec[(size_t)i * R_COUNT];
            bastr_step_out& o = out[i];
            o.nstep = n0 + i;
            o.time = t;
            o.Esspe = r[R_ES]; o.Edspe = r[R_ED]; o.k2Edspe = r[R_K2ED]; o.kMEdspe = r[R_KMED];
            const bool vg = h->p.velgrad_every > 0 && ((n0 + i) % h->p.velgrad_every) == 0;
            for (int k = 0; k < 8; ++k) o.velgrad[k] = vg ? r[R_VG0 + k] : NAN;
            o.factor = h->p.forcemethod ? r[R_FACTOR] : NAN;
            o.E = h->p.forcemethod >= 2 ? r[R_E] : NAN;
            const bool rnd = h->p.forcemethod == 3 || h->p.forcemethod == 4;
            o.energy = rnd ? r[R_ENERGY] : NAN;
            o.Fen = rnd ? r[R_FEN] : NAN;
        }
        t = t + h->p.deltat;
    }
}

// Launches nsteps steps on the handle's stream into record slots 0..nsteps-1 and advances the
// host counters.  The batch's stop word is cleared first; the kernels of the batch see it through
// h->g.halt, which is set only while they are launched (calls outside a batch, such as the state
// read-back after a NaN stop, must not skip).
cudaError_t launch_batch(bastr_handle* h, int nsteps) {
    h->batch_n0 = h->nstep;
    h->batch_t0 = h->time;
    unsigned int* halt = h->done + T_HALT;
    cudaError_t e = cudaMemsetAsync(halt, 0, sizeof(unsigned int), h->stream);
    if (e != cudaSuccess) return e;
    h->g.halt = halt;
    for (int i = 0; i < nsteps && e == cudaSuccess; ++i) {
        const int64_t n = h->nstep;
        const bool vg = h->p.velgrad_every > 0 && (n % h->p.velgrad_every) == 0;
        e = launch_step(h, i, vg);
        if (e != cudaSuccess) break;
        h->nstep += 1;
        h->time = h->time + h->p.deltat;
    }
    h->g.halt = nullptr;
    if (e != cudaSuccess) return e;
    h->chunk_used = nsteps;
    return cudaSuccess;
}

// After a batch whose stop word read `halt` (0: ran to the end; else the slot + 1 of the step
// whose Es+Ed was NaN): winds the host counters back to that step, as the reference stops before
// its nstep = nstep + 1 (solution.F90:81-84), and keeps only the records up to it.  Returns the
// number of valid records.
int apply_halt(bastr_handle* h, unsigned int halt, int nsteps) {
    if (halt == 0 || (int)halt > nsteps) return nsteps;
    const int k = (int)halt - 1;
    h->nstep = h->batch_n0;
    h->time = h->batch_t0;
    for (int i = 0; i < k; ++i) {
        h->nstep += 1;
        h->time = h->time + h->p.deltat;
    }
    h->chunk_used = k + 1;
    return k + 1;
}

// Records from slot `valid` on belong to steps that did not run after a NaN stop: NaN values.
void blank_records(bastr_step_out* out, int valid, int nsteps) {
    if (!out) return;
    for (int i = valid; i < nsteps; ++i) {
        bastr_step_out& o = out[i];
        const int64_t n = out[valid - 1].nstep;
        const double t = out[valid - 1].time;
        o.nstep = n;
        o.time = t;
        o.Esspe = o.Edspe = o.k2Edspe = o.kMEdspe = NAN;
        for (double& v : o.velgrad) v = NAN;
        o.factor = o.E = o.energy = o.Fen = NAN;
    }
}

}  // namespace

extern "C" {

int bastr_set_plan(bastr_handle* h, int32_t share_log2) {
    if (!h) return BASTR_E_INVALID;
    if (share_log2 < 0 || share_log2 > 7) return fail(h, BASTR_E_INVALID, "share_log2 must be in [0, 7]");
    h->share_log2 = share_log2;
    return BASTR_OK;
}

int bastr_step_async(bastr_handle* h, int32_t nsteps) {
    NvtxRange range("bastr_step");
    if (!h || nsteps < 0) return fail(h, BASTR_E_INVALID, "nsteps");
    if (!h->have_state) return fail(h, BASTR_E_STATE, "no state set");
    if (nsteps > kChunk) return fail(h, BASTR_E_INVALID, "bastr_step_async: at most %d steps per call", kChunk);
    CK(cudaSetDevice(h->device));
    CK(launch_batch(h, nsteps));
    return BASTR_OK;
}

// Gathers a batch's read-back into one contiguous buffer: [stop word, error word] as doubles,
// then nrec record values, then nsh shell values, so that the host fetches it with one copy.
__global__ void k_pack_records(const double* __restrict__ rec, const double* __restrict__ shells,
                               const unsigned int* __restrict__ words, size_t nrec, size_t nsh,
                               double* __restrict__ out) {
    const size_t n = 2 + nrec + nsh;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = i < 2 ? (double)words[i] : i < 2 + nrec ? rec[i - 2] : shells[i - 2 - nrec];
}

int bastr_step_records(bastr_handle* h, int32_t nsteps, bastr_step_out* out, double* shells) {
    if (!h) return BASTR_E_INVALID;
    if (nsteps < 0 || nsteps > h->chunk_used) return fail(h, BASTR_E_INVALID, "only %d records available", h->chunk_used);
    CK(cudaSetDevice(h->device));
    // the records, the shells asked for and the batch's two words in one copy into pinned memory
    const size_t nrec = (size_t)nsteps * R_COUNT;
    const size_t nsh = shells ? (size_t)nsteps * 2 * (h->allkmax + 1) : 0;
    const size_t cap = 2 + (size_t)kChunk * (R_COUNT + 2 * (h->allkmax + 1));
    if (!h->stage_host) {
        CK(cudaMalloc(&h->stage_dev, cap * sizeof(double)));
        CK(track_alloc(h, h->stage_dev, cap * sizeof(double)));
        CK(cudaMallocHost(&h->stage_host, cap * sizeof(double)));
    }
    const int grid = (int)std::min<size_t>((2 + nrec + nsh + 255) / 256, 148);
    k_pack_records<<<grid, 256, 0, h->stream>>>(h->rec, h->shells_dev, h->done + T_HALT, nrec, nsh, h->stage_dev);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->stage_host, h->stage_dev, (2 + nrec + nsh) * sizeof(double), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const double* staged = h->stage_host;
    const unsigned int words[2] = {(unsigned int)staged[0], (unsigned int)staged[1]};   // stop, error
    const double* rec = staged + 2;
    if (shells && nsh) std::memcpy(shells, staged + 2 + nrec, nsh * sizeof(double));
    const unsigned int halt = words[0];
    if (words[1] != 0) {
        CK(cudaMemsetAsync(h->done + T_ERR, 0, sizeof(unsigned int), h->stream));
        return fail(h, BASTR_E_CUDA,
                    "a kernel of the last batch reported an error (error word %u: 1 = a TMA staging wait gave up, "
                    "2 = an index check of the checked build failed)",
                    words[1]);
    }
    // the stop word belongs to the last batch (chunk_used steps); a NaN step within the records asked for
    const int valid = apply_halt(h, halt, h->chunk_used);
    const int nv = std::min(valid, (int)nsteps);
    decode_records(h, rec, nv, out);
    if (nv < nsteps) {
        blank_records(out, nv, nsteps);
        if (shells)
            std::fill(shells + (size_t)nv * 2 * (h->allkmax + 1), shells + (size_t)nsteps * 2 * (h->allkmax + 1),
                      (double)NAN);
    }
    if (halt != 0 && (int)halt <= nsteps)
        return fail(h, BASTR_E_NAN, "\"E\" is a NaN at nstep %lld", (long long)(h->batch_n0 + (int)halt - 1));
    return BASTR_OK;
}

int bastr_step(bastr_handle* h, int32_t nsteps, bastr_step_out* out, double* shells) {
    if (!h || nsteps < 0) return fail(h, BASTR_E_INVALID, "nsteps");
    if (!h->have_state) return fail(h, BASTR_E_STATE, "no state set");
    int done = 0;
    while (done < nsteps) {
        const int n = std::min(kChunk, nsteps - done);
        int r = bastr_step_async(h, n);
        if (r) return r;
        r = bastr_step_records(h, n, out ? out + done : nullptr,
                               shells ? shells + (size_t)done * 2 * (h->allkmax + 1) : nullptr);
        if (r == BASTR_E_NAN) {
            // the records after the NaN step, in this chunk and the ones not run, are NaN
            const int valid = h->chunk_used;
            blank_records(out ? out + done : nullptr, valid, nsteps - done);
            if (shells)
                std::fill(shells + (size_t)(done + valid) * 2 * (h->allkmax + 1),
                          shells + (size_t)nsteps * 2 * (h->allkmax + 1), (double)NAN);
            return r;
        }
        if (r) return r;
        done += n;
    }
    return BASTR_OK;
}

int bastr_spectra(bastr_handle* h, double* kn, double* Es, double* Ed, int64_t* Ecount) {
    if (!h) return BASTR_E_INVALID;
    if (!h->have_state) return fail(h, BASTR_E_STATE, "no state set");
    CK(cudaSetDevice(h->device));
    const int am = h->allkmax;
    // use the last chunk slot as scratch
    double* rec = h->rec + (size_t)(kChunk - 1) * R_COUNT;
    double* sh = h->shells_dev + (size_t)(kChunk - 1) * 2 * (am + 1);
    CK(launch_spectra(h, rec, sh, 0u));
    std::vector<double> buf(2 * (am + 1));
    CK(cudaMemcpyAsync(buf.data(), sh, buf.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int s = 0; s <= am; ++s) {
        if (kn) kn[s] = h->kn[s];
        if (Es) Es[s] = buf[s];
        if (Ed) Ed[s] = buf[am + 1 + s];
        if (Ecount) Ecount[s] = h->ecount[s];
    }
    return BASTR_OK;
}

int bastr_fft(bastr_handle* h, double* array, int32_t dir) {
    if (!h || !array || (dir != 1 && dir != -1)) return fail(h, BASTR_E_INVALID, "bastr_fft arguments");
    CK(cudaSetDevice(h->device));
    return full_fft(h, array, dir);
}

int bastr_profile(bastr_handle* h, int32_t nsteps, bastr_kernel_stat* stats, int32_t max_stats, int32_t* n_stats) {
    if (!h || nsteps < 1 || nsteps > kChunk) return fail(h, BASTR_E_INVALID, "bastr_profile: 1..%d steps", kChunk);
    if (!h->have_state) return fail(h, BASTR_E_STATE, "no state set");
    CK(cudaSetDevice(h->device));
    const size_t need = (size_t)2 * nsteps * (h->launches_per_step + 4);
    while (h->ev_pool.size() < need) {
        cudaEvent_t ev;
        CK(cudaEventCreate(&ev));
        h->ev_pool.push_back(ev);
    }
    h->ev_used = 0;
    h->prof.clear();
    h->prof_on = true;
    const int r = bastr_step_async(h, nsteps);
    h->prof_on = false;
    if (r) return r;
    CK(cudaStreamSynchronize(h->stream));
    std::vector<std::string> names;
    std::vector<double> tot, bytes;
    std::vector<int> cnt;
    for (const auto& pr : h->prof) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, h->ev_pool[pr.ev], h->ev_pool[pr.ev + 1]));
        size_t i = 0;
        while (i < names.size() && names[i] != pr.name) ++i;
        if (i == names.size()) { names.push_back(pr.name); tot.push_back(0); bytes.push_back(0); cnt.push_back(0); }
        tot[i] += ms;
        bytes[i] += pr.bytes;
        cnt[i] += 1;
    }
    const int n = (int)std::min<size_t>(names.size(), (size_t)std::max(max_stats, 0));
    for (int i = 0; i < n && stats; ++i) {
        memset(stats[i].name, 0, sizeof stats[i].name);
        strncpy(stats[i].name, names[i].c_str(), sizeof stats[i].name - 1);
        stats[i].launches = cnt[i];
        stats[i].total_ms = tot[i];
        stats[i].bytes_per_launch = bytes[i] / cnt[i];
    }
    if (n_stats) *n_stats = (int32_t)names.size();
    return BASTR_OK;
}

int bastr_set_stream(bastr_handle* h, void* s) {
    if (!h) return BASTR_E_INVALID;
    CK(cudaSetDevice(h->device));
    if (h->stream) CK(cudaStreamSynchronize(h->stream));
    if (h->own_stream && h->stream) CK(cudaStreamDestroy(h->stream));
    h->own_stream = false;
    h->stream = (cudaStream_t)s;
    return BASTR_OK;
}

int bastr_sync(bastr_handle* h) {
    if (!h) return BASTR_E_INVALID;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    return BASTR_OK;
}

int bastr_info(bastr_handle* h, int32_t* allkmax, int32_t* launches, int64_t* bytes) {
    if (!h) return BASTR_E_INVALID;
    if (allkmax) *allkmax = h->allkmax;
    if (launches) *launches = h->launches_per_step;
    if (bytes) *bytes = h->dev_bytes;
    return BASTR_OK;
}

int bastr_last_error(bastr_handle* h, char* buf, int32_t n) {
    if (!h) return 0;
    const int len = (int)h->err.size();
    if (buf && n > 0) {
        const int m = std::min(len, n - 1);
        memcpy(buf, h->err.data(), m);
        buf[m] = 0;
    }
    return len;
}

}  // extern "C"

extern "C" {

int bastr_net_nparams(void) { return kNetNP; }

int bastr_net_grad_blocks(void) { return 2 * 148; }

int bastr_net_forward(int32_t nx, int32_t ny, int32_t nz, const float* d_u, const uint16_t* d_w, float* d_out,
                      float scale, void* stream) {
    if (nx < 3 || ny < 3 || nz < 3 || !d_u || !d_w || !d_out) return BASTR_E_INVALID;
    const size_t n = (size_t)nx * ny * nz;
    if (3 * n >= ((size_t)1 << 31)) return BASTR_E_UNSUPPORTED;   // the kernel's 32-bit tap offsets
    const int grid = (int)std::min<size_t>((n + kFwdNT - 1) / kFwdNT, 148 * 4);
    k_net_forward_tc<float><<<grid, kFwdNT, kFwdSmem, (cudaStream_t)stream>>>(d_u, (const __nv_bfloat16*)d_w, d_out,
                                                                            nx, ny, nz, scale, nullptr);
    return cudaGetLastError() == cudaSuccess ? BASTR_OK : BASTR_E_CUDA;
}

int bastr_net_grad(int32_t nx, int32_t ny, int32_t nz, const float* d_u, const float* d_tau, const uint16_t* d_w,
                   float* d_part, int32_t nblk, float* d_grad, double* d_loss, void* stream) {
    if (nx < 3 || ny < 3 || nz < 3 || !d_u || !d_tau || !d_w || !d_part || !d_grad || nblk < 1)
        return BASTR_E_INVALID;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_net_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem);
    });
    if (attr != cudaSuccess) return BASTR_E_CUDA;
    const size_t n = (size_t)nx * ny * nz;
    cudaStream_t st = (cudaStream_t)stream;
    k_net_grad<<<nblk, kGradNT, kGradSmem, st>>>(d_u, d_tau, (const __nv_bfloat16*)d_w, d_part, nx, ny, nz);
    k_net_reduce<<<(kNetNP + 1 + 255) / 256, 256, 0, st>>>(d_part, nblk, d_grad, d_loss, 1.0 / (3.0 * (double)n));
    return cudaGetLastError() == cudaSuccess ? BASTR_OK : BASTR_E_CUDA;
}

int bastr_net_adam(float* d_w, uint16_t* d_wb, float* d_m, float* d_v, const float* d_g, int32_t t, float lr,
                   float b1, float b2, float eps, void* stream) {
    if (!d_w || !d_wb || !d_m || !d_v || !d_g || t < 1) return BASTR_E_INVALID;
    k_net_adam<<<(kNetNP + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_w, (__nv_bfloat16*)d_wb, d_m, d_v, d_g, t,
                                                                       lr, b1, b2, eps);
    return cudaGetLastError() == cudaSuccess ? BASTR_OK : BASTR_E_CUDA;
}

// Transfer spectra of the current state (transfer2d/transfer3d, Bastrpp.F90:174-305, 418-599):
// T, T1, T2 for shells 0..allkmax (host arrays of allkmax+1 doubles).
int bastr_transfer(bastr_handle* h, double* T, double* T1, double* T2) {
    if (!h) return BASTR_E_INVALID;
    if (!h->have_state) return fail(h, BASTR_E_STATE, "no state set");
    CK(cudaSetDevice(h->device));
    const Geo& g = h->g;
    const int D = g.d;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    const size_t narr = (size_t)(D + D * D + D + D + D * D);
    const size_t nmodes = (size_t)g.K * g.KY * g.KZ;
    if (!h->tr_buf) {
        CK(cudaMalloc(&h->tr_buf, narr * n * sizeof(double2)));
        CK(track_alloc(h, h->tr_buf, narr * n * sizeof(double2)));
    }
    if (!h->tr_modes) {
        const size_t bytes = (nmodes * 3 + (size_t)std::max(h->n_items, 1) * 3 + 3 * (size_t)h->nshell) * sizeof(double);
        CK(cudaMalloc(&h->tr_modes, bytes));
        CK(track_alloc(h, h->tr_modes, bytes));
    }
    double2* U = h->tr_buf;
    double2* Dv = U + (size_t)D * n;
    double2* tA = Dv + (size_t)D * D * n;
    double2* tC = tA + (size_t)D * n;
    double2* P = tC + (size_t)D * n;
    double* tr = h->tr_modes;
    double* part = tr + nmodes * 3;
    double* out = part + (size_t)std::max(h->n_items, 1) * 3;
    CK(flush_pending_scale(h));
    CK(cudaMemsetAsync(U, 0, (size_t)D * n * sizeof(double2), h->stream));
    const int gs = 148 * 8;
    if (D == 2) k_tr_scatter<2><<<gs, 256, 0, h->stream>>>(h->u0, g, U, n);
    else k_tr_scatter<3><<<gs, 256, 0, h->stream>>>(h->u0, g, U, n);
    CK(cudaGetLastError());
    for (int c = 0; c < D; ++c)
        for (int j = 0; j < D; ++j) k_tr_deriv<<<gs, 256, 0, h->stream>>>(U + (size_t)c * n, Dv + (size_t)(c * D + j) * n, j, g);
    CK(cudaGetLastError());
    // to physical space: u_c and d_cj
    for (size_t a = 0; a < (size_t)(D + D * D); ++a)
        for (int ax = 0; ax < D; ++ax) CK(full_axis<true>(h, U + a * n, ax, 1.0));
    if (D == 2) k_tr_products<2><<<gs, 256, 0, h->stream>>>(U, Dv, tA, tC, P, n);
    else k_tr_products<3><<<gs, 256, 0, h->stream>>>(U, Dv, tA, tC, P, n);
    CK(cudaGetLastError());
    // forward transforms (scaled 1/N) of tA, tC, P
    for (size_t a = 0; a < (size_t)(D + D + D * D); ++a)
        for (int ax = 0; ax < D; ++ax) CK(full_axis<false>(h, tA + a * n, ax, ax == D - 1 ? g.inv_n : 1.0));
    if (D == 2) k_tr_modes<2><<<gs, 256, 0, h->stream>>>(h->u0, g, tA, tC, P, tr, n);
    else k_tr_modes<3><<<gs, 256, 0, h->stream>>>(h->u0, g, tA, tC, P, tr, n);
    CK(cudaGetLastError());
    if (h->n_items > 0) k_tr_items<256><<<h->n_items, 256, 0, h->stream>>>(tr, h->sp_modes, h->sp_item_lo, part);
    else CK(cudaMemsetAsync(part, 0, 3 * sizeof(double), h->stream));
    k_tr_shells<<<(h->nshell + 127) / 128, 128, 0, h->stream>>>(part, h->sp_shell_item, h->nshell, out);
    CK(cudaGetLastError());
    std::vector<double> buf(3 * (size_t)h->nshell);
    CK(cudaMemcpyAsync(buf.data(), out, buf.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double* dst[3] = {T, T1, T2};
    for (int k = 0; k < 3; ++k) {
        if (!dst[k]) continue;
        for (int s2 = 0; s2 <= h->allkmax; ++s2) dst[k][s2] = s2 < h->nshell ? buf[(size_t)k * h->nshell + s2] : 0.0;
    }
    return BASTR_OK;
}

// Bastrpp's initial-field generators (hitgen.cu).  Work arrays: full complex grids of the
// transfer buffer (R, field A, field B, angle) and the physical-field buffer for the result.
int bastr_hitgen(bastr_handle* h, int32_t variant, uint64_t seed, double* u1, double* u2, double* u3,
                 double* angle, double* stats) {
    if (!h) return BASTR_E_INVALID;
    if (variant != 0 && variant != 1) return fail(h, BASTR_E_INVALID, "hitgen variant must be 0 or 1");
    const Geo& g = h->g;
    const int D = g.d;
    if (variant == 1 && D != 2) return fail(h, BASTR_E_UNSUPPORTED, "hitgen2dbis is two-dimensional");
    if (!(h->p.forcek > 0)) return fail(h, BASTR_E_INVALID, "hitgen needs forcek > 0");
    CK(cudaSetDevice(h->device));
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    const size_t narr = (size_t)(D + D * D + D + D + D * D);   // the transfer buffer's size
    constexpr int NB = 148 * 4, NT = 256;
    if (!h->tr_buf) {
        CK(cudaMalloc(&h->tr_buf, narr * n * sizeof(double2)));
        CK(track_alloc(h, h->tr_buf, narr * n * sizeof(double2)));
    }
    if (!h->hg_part) {
        CK(cudaMalloc(&h->hg_part, (size_t)NB * 4 * sizeof(double)));
        CK(track_alloc(h, h->hg_part, (size_t)NB * 4 * sizeof(double)));
    }
    const bool bis = variant == 1;
    double2* R = h->tr_buf;
    double2* A = R + n;
    double2* B = A + 3 * n;
    double* ang = reinterpret_cast<double*>(bis ? B + 3 * n : A + 3 * n);
    const int gs = 148 * 8;
    std::vector<double> part((size_t)NB * 4);
    auto sums = [&](const double2* X, const double2* Y, double alpha, int mode, double out[4]) -> int {
        k_hg_sums<NT><<<NB, NT, 0, h->stream>>>(X, Y, alpha, D, n, mode, h->hg_part);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(part.data(), h->hg_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (int i = 0; i < 4; ++i) out[i] = 0.0;
        for (int b = 0; b < NB; ++b)
            for (int i = 0; i < 4; ++i) out[i] += part[(size_t)b * 4 + i];
        return BASTR_OK;
    };
    // one draw: uniform field -> R -> modes of F -> physical (real parts used)
    auto draw = [&](int d, double2* F) -> int {
        k_hg_uniform<<<gs, 256, 0, h->stream>>>(R, ang, n, d, (unsigned long long)seed);
        CK(cudaGetLastError());
        for (int a = 0; a < D; ++a) CK(full_axis<false>(h, R, a, a == D - 1 ? g.inv_n : 1.0));
        if (D == 2) k_hg_modes<2><<<gs, 256, 0, h->stream>>>(R, F, ang, g, (double)h->p.forcek, bis, bis);
        else k_hg_modes<3><<<gs, 256, 0, h->stream>>>(R, F, ang, g, (double)h->p.forcek, 0, 0);
        CK(cudaGetLastError());
        const int nf = bis ? D + 1 : D;
        for (int c = 0; c < nf; ++c)
            for (int a = 0; a < D; ++a) CK(full_axis<true>(h, F + (size_t)c * n, a, 1.0));
        return BASTR_OK;
    };
    int rc = draw(0, A);
    if (rc != BASTR_OK) return rc;
    double alpha = 0.0, check = std::nan(""), q[4] = {0, 0, 0, 0};
    const double2* Bc = nullptr;
    if (bis) {
        rc = draw(1, B);
        if (rc != BASTR_OK) return rc;
        rc = sums(A, B, 0.0, 1, q);
        if (rc != BASTR_OK) return rc;
        for (int i = 0; i < 4; ++i) q[i] *= g.inv_n;
        alpha = hitgen_cubic_root(q[0], q[1], q[2], q[3]);
        check = q[0] + alpha * q[1] + alpha * alpha * q[2] + alpha * alpha * alpha * q[3];
        Bc = B;
    }
    double e[4];
    rc = sums(A, Bc, alpha, 0, e);
    if (rc != BASTR_OK) return rc;
    const double energy = e[0] / ((double)g.nx * g.ny * g.nz);
    const double factor = std::sqrt(h->p.target_energy / energy);
    k_hg_finish<<<gs, 256, 0, h->stream>>>(A, Bc, alpha, factor, D, n, h->phys);
    CK(cudaGetLastError());
    double* dst[3] = {u1, u2, u3};
    for (int c = 0; c < D; ++c)
        if (dst[c]) CK(cudaMemcpyAsync(dst[c], h->phys + (size_t)c * n, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (angle) CK(cudaMemcpyAsync(angle, ang, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (stats) {
        const double v[8] = {energy, factor, bis ? alpha : std::nan(""), check, q[0], q[1], q[2], q[3]};
        for (int i = 0; i < 8; ++i) stats[i] = v[i];
    }
    return BASTR_OK;
}

// Filtered fields and the subgrid term of the current state (subgrid.cu), for closure training:
// d_ubar, d_tau: device arrays of d * (nx/r)(ny/r)(nz/r) floats, [component][coarse grid], x
// fastest (either may be NULL).  Work buffers are allocated on the first call (and when r changes).
int bastr_subgrid(bastr_handle* h, int32_t r, float* d_ubar, float* d_tau) {
    if (!h) return BASTR_E_INVALID;
    if (!h->have_state) return fail(h, BASTR_E_STATE, "no state set");
    const Geo& g = h->g;
    const int D = g.d;
    if (r < 2 || (r & (r - 1)) || g.nx % r || g.ny % r || (D == 3 && g.nz % r))
        return fail(h, BASTR_E_INVALID, "filter width %d must be a power of two dividing the grid", r);
    const int cns[3] = {g.nx / r, g.ny / r, D == 3 ? g.nz / r : 1};
    for (int a = 0; a < D; ++a)
        if (cns[a] < 16) return fail(h, BASTR_E_UNSUPPORTED, "coarse extents below 16 are not built");
    if (!d_ubar && !d_tau) return fail(h, BASTR_E_INVALID, "no output");
    CK(cudaSetDevice(h->device));
    const size_t N = (size_t)g.nx * g.ny * g.nz, nc = (size_t)cns[0] * cns[1] * cns[2];
    if (h->sg_r != r) {
        if (h->sg_buf) CK(cudaFree(h->sg_buf));
        if (h->sg_tw) CK(cudaFree(h->sg_tw));
        h->sg_buf = nullptr;
        h->sg_tw = nullptr;
        h->sg_r = 0;
        CK(cudaMalloc(&h->sg_buf, (3 * N + nc * (4 * (size_t)D + 3)) * sizeof(double)));
        CK(cudaMalloc(&h->sg_tw, (size_t)(cns[0] + cns[1] + cns[2]) * sizeof(double2)));
        CK(track_alloc(h, h->sg_buf, (3 * N + nc * (4 * (size_t)D + 3)) * sizeof(double)));
        CK(track_alloc(h, h->sg_tw, (size_t)(cns[0] + cns[1] + cns[2]) * sizeof(double2)));
        size_t o = 0;
        for (int a = 0; a < 3; ++a) {
            std::vector<double2> t64;
            std::vector<float2> t32;
            host_twiddles(cns[a], t64, t32);
            CK(cudaMemcpy(h->sg_tw + o, t64.data(), cns[a] * sizeof(double2), cudaMemcpyHostToDevice));
            o += cns[a];
        }
        h->sg_r = r;
    }
    const double2* ctw[3] = {h->sg_tw, h->sg_tw + cns[0], h->sg_tw + cns[0] + cns[1]};
    double2* W = reinterpret_cast<double2*>(h->sg_buf);          // fine complex scratch
    double* acc = h->sg_buf + 2 * N;                               // fine products
    double* ub = acc + N;                                          // [D][nc]
    double* fadv = ub + D * nc;                                    // [D][nc]
    double* cadv = fadv + D * nc;                                  // [nc]
    double2* uh = reinterpret_cast<double2*>(cadv + nc);           // [D][nc] spectra of ub
    double2* Wc = uh + D * nc;                                     // coarse complex scratch
    cudaStream_t st = h->stream;
    const int gs = 148 * 8;
    CK(flush_pending_scale(h));
    CK(to_physical(h));                                            // h->phys = u, [D][N]
    // filter(u_j d_j u_i) on the fine grid
    for (int i = 0; i < D; ++i) {
        for (int j = 0; j < D; ++j) {
            CK(cudaMemsetAsync(W, 0, N * sizeof(double2), st));
            if (D == 2) k_sg_scatter<2><<<gs, 256, 0, st>>>(h->u0, g, i, j, W);
            else k_sg_scatter<3><<<gs, 256, 0, st>>>(h->u0, g, i, j, W);
            CK(cudaGetLastError());
            for (int a = 0; a < D; ++a) CK(full_axis<true>(h, W, a, 1.0));
            k_sg_accum<<<gs, 256, 0, st>>>(acc, h->phys + (size_t)j * N, W, N, j == 0);
            CK(cudaGetLastError());
        }
        k_sg_filter<<<gs, 256, 0, st>>>(acc, g.nx, g.ny, g.nz, r, D, fadv + (size_t)i * nc);
        CK(cudaGetLastError());
    }
    // ub and its spectra on the coarse grid
    for (int c = 0; c < D; ++c) {
        k_sg_filter<<<gs, 256, 0, st>>>(h->phys + (size_t)c * N, g.nx, g.ny, g.nz, r, D, ub + (size_t)c * nc);
        k_sg_complex<<<gs, 256, 0, st>>>(ub + (size_t)c * nc, uh + (size_t)c * nc, nc);
        CK(cudaGetLastError());
        for (int a = 0; a < D; ++a)
            CK(full_axis_n<false>(h, uh + (size_t)c * nc, cns, a, a == D - 1 ? 1.0 / (double)nc : 1.0, ctw[a]));
    }
    // ub_j d_j ub_i on the coarse grid, and the outputs
    for (int i = 0; i < D; ++i) {
        for (int j = 0; j < D; ++j) {
            k_sg_deriv<<<gs, 256, 0, st>>>(uh + (size_t)i * nc, Wc, cns[0], cns[1], cns[2], j);
            CK(cudaGetLastError());
            for (int a = 0; a < D; ++a) CK(full_axis_n<true>(h, Wc, cns, a, 1.0, ctw[a]));
            k_sg_accum<<<gs, 256, 0, st>>>(cadv, ub + (size_t)j * nc, Wc, nc, j == 0);
            CK(cudaGetLastError());
        }
        k_sg_finish<<<gs, 256, 0, st>>>(fadv + (size_t)i * nc, cadv, ub + (size_t)i * nc,
                                         d_tau ? d_tau + (size_t)i * nc : nullptr,
                                         d_ubar ? d_ubar + (size_t)i * nc : nullptr, nc);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(st));
    return BASTR_OK;
}

// One closure sub-step on a 3D handle's state: u <- u - dt * scale * net(u) in physical space,
// then back to the (dealiased) spectral state.
int bastr_closure_apply(bastr_handle* h, const uint16_t* d_w, float scale, double dt) {
    NvtxRange range("bastr_closure_apply");
    if (!h || !d_w) return BASTR_E_INVALID;
    if (h->g.d != 3) return fail(h, BASTR_E_UNSUPPORTED, "the closure network is three-dimensional");
    if (!h->have_state) return fail(h, BASTR_E_STATE, "no state set");
    CK(cudaSetDevice(h->device));
    const size_t n = (size_t)h->g.nx * h->g.ny * h->g.nz;
    if (3 * n >= ((size_t)1 << 31)) return fail(h, BASTR_E_UNSUPPORTED, "closure network: grid too large");
    if (!h->closure_buf) {
        CK(cudaMalloc(&h->closure_buf, 3 * n * sizeof(float)));
        CK(track_alloc(h, h->closure_buf, 3 * n * sizeof(float)));
    }
    CK(flush_pending_scale(h));
    CK(to_physical(h));
    const int grid = (int)std::min<size_t>((n + kFwdNT - 1) / kFwdNT, 148 * 4);
    k_net_forward_tc<double><<<grid, kFwdNT, kFwdSmem, h->stream>>>(h->phys, (const __nv_bfloat16*)d_w,
                                                                      h->closure_buf, h->g.nx, h->g.ny, h->g.nz,
                                                                      scale, h->done + T_ERR);
    CK(cudaGetLastError());
    k_closure_update<<<148 * 4, 256, 0, h->stream>>>(h->phys, h->closure_buf, 3 * n, dt);
    CK(cudaGetLastError());
    CK(to_spectral(h));
    return BASTR_OK;
}

}  // extern "C"

#include "ensemble.cu"
#include "slab.cu"
