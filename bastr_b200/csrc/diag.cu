// Per-step diagnostics and forcing on the truncated FP64 state, with deterministic
// (fixed-order) FP64 reductions: two runs on the same input agree bitwise.
//
//  k_spectra_fused  spectra_compute2D/3D (solution.F90:930-1108): work items are runs of a
//                   per-shell list of the stored modes (shell nint(|k|), tool.F90:145; Hermitian
//                   partners counted by weight 2); the block that finishes last sums the items
//                   of each shell in fixed order -> Es, Ed shells, Esspe, Edspe, k2Edspe, kMEdspe.
//  k_velgrad_final  velgrad_calculate2D/3D reductions and derived lengths (solution.F90:1168-1180,
//                   1268-1280) from the x pass's per-block partials.
//  k_force_*        forcing2D/3D methods 1-5 (solution.F90:315-812).  The random phases of
//                   methods 3 and 4 come from Philox-4x32-10 (counter-based; the reference draws
//                   them from gfortran's random_number, so they agree in distribution only).
#pragma once
#include <cstdint>
#include "solver.cuh"

// List entries a thread of the spectra kernel loads together (their index and state loads in
// flight at once).
#ifndef BASTR_SPECTRA_U
#define BASTR_SPECTRA_U 4
#endif
// List entries of one work item (one block) of the spectra kernel.
#ifndef BASTR_SPECTRA_ITEM
#define BASTR_SPECTRA_ITEM 2048
#endif

namespace bastr {

// Record slots (doubles) written per step on the device.
enum RecSlot : int {
    R_ES = 0, R_ED, R_K2ED, R_KMED,
    R_VG0 = 4,            // 8 velocity-gradient statistics, slots 4..11
    R_FACTOR = 12, R_E = 13, R_ENERGY = 14, R_FEN = 15,
    R_COUNT = 16
};

__device__ __forceinline__ long long isqrt_floor(long long v) {
    if (v <= 0) return 0;
    long long r = (long long)sqrt((double)v);
    while (r * r > v) --r;
    while ((r + 1) * (r + 1) <= v) ++r;
    return r;
}
__device__ __forceinline__ long long isqrt_ceil(long long v) {
    if (v <= 0) return 0;
    long long r = isqrt_floor(v);
    return r * r == v ? r : r + 1;
}

// Adds the contributions of one stored mode (kx >= 0 half) to the shell accumulators.
template <int D>
__device__ __forceinline__ void spectra_mode(double2* __restrict__ U0, const Geo& g, int kx,
                                             int ky, int kz, double acc[4], bool scale = false,
                                             double f = 1.0) {
    const int K = g.K;
    const int kyi = ky >= 0 ? ky : ky + g.KY;
    const long long m = (long long)kx * kx + (long long)ky * ky + (long long)kz * kz;
    if (m == 0) return;   // kk <= dk/2: us = ud = 0
    const double kk = sqrt((double)m);
    const double ik = 1.0 / kk;
    const double w = kx == 0 ? 1.0 : 2.0;
    // unit wavevector, one reciprocal per mode
    const double h1 = kx * ik, h2 = ky * ik, h3 = kz * ik;
    double es, ed;
    if constexpr (D == 2) {
        const size_t o = ((size_t)kx * g.KY + kyi) * 2;
        double2 a = BASTR_AT(U0, o, g), b = BASTR_AT(U0, o + 1, g);
        if (scale) {   // the linear forcing of the previous step, applied here (forcing3D-style u *= f)
            a = make_double2(f * a.x, f * a.y);
            b = make_double2(f * b.x, f * b.y);
            BASTR_AT(U0, o, g) = a;
            BASTR_AT(U0, o + 1, g) = b;
        }
        // usspe = u1 k2/kk - u2 k1/kk ; udspe = u1 k1/kk + u2 k2/kk  (solution.F90:958-959)
        const double usx = a.x * h2 - b.x * h1, usy = a.y * h2 - b.y * h1;
        const double udx = a.x * h1 + b.x * h2, udy = a.y * h1 + b.y * h2;
        es = (usx * usx + usy * usy) / 2;
        ed = (udx * udx + udy * udy) / 2;
        (void)h3;
    } else {
        const int kzi = kz >= 0 ? kz : kz + g.KZ;
        const size_t o = ((size_t)kx * g.KY + kyi) * g.KZ + kzi;
        double2 a = BASTR_AT(U0, o, g), b = BASTR_AT(U0, o + g.ps, g), c = BASTR_AT(U0, o + 2 * g.ps, g);
        if (scale) {   // the linear forcing of the previous step, applied here (solution.F90:328-331)
            a = make_double2(f * a.x, f * a.y);
            b = make_double2(f * b.x, f * b.y);
            c = make_double2(f * c.x, f * c.y);
            BASTR_AT(U0, o, g) = a;
            BASTR_AT(U0, o + g.ps, g) = b;
            BASTR_AT(U0, o + 2 * g.ps, g) = c;
        }
        // solution.F90:1047-1053
        const double udx = a.x * h1 + b.x * h2 + c.x * h3;
        const double udy = a.y * h1 + b.y * h2 + c.y * h3;
        const double s1x = a.x - udx * h1, s1y = a.y - udy * h1;
        const double s2x = b.x - udx * h2, s2y = b.y - udy * h2;
        const double s3x = c.x - udx * h3, s3y = c.y - udy * h3;
        es = (s1x * s1x + s1y * s1y) / 2 + (s2x * s2x + s2y * s2y) / 2 + (s3x * s3x + s3y * s3y) / 2;
        ed = (udx * udx + udy * udy) / 2;
    }
    (void)K;
    acc[0] += w * es;
    acc[1] += w * ed;
    acc[2] += w * (ed * (double)m);
    acc[3] += w * (ed * ik);
}

// Shell sums from the item partials (items of shell s are shell_item[s] .. shell_item[s+1]-1),
// totals over all shells in fixed order, and the copy of shells 0..allkmax for the spect log.
// Run by one whole block; reads the partials through L2.
template <int NT>
__device__ __forceinline__ void spectra_finish(const double* item_part, const int* __restrict__ shell_item,
                                               int nshell, int allkmax, double* __restrict__ rec,
                                               double* __restrict__ shells_out, double* scratch,
                                               unsigned int* halt, unsigned int halt_code) {
    double acc[4] = {0, 0, 0, 0};
    for (int s = threadIdx.x; s < nshell; s += NT) {
        double sh[4] = {0, 0, 0, 0};
        for (int it = shell_item[s]; it < shell_item[s + 1]; ++it) {
#pragma unroll
            for (int i = 0; i < 4; ++i) sh[i] += __ldcg(item_part + (size_t)it * 4 + i);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i] += sh[i];
        if (shells_out && s <= allkmax) {
            shells_out[s] = sh[0];
            shells_out[allkmax + 1 + s] = sh[1];
        }
    }
    if (shells_out) {
        for (int s = nshell + threadIdx.x; s <= allkmax; s += NT) {
            shells_out[s] = 0.0;
            shells_out[allkmax + 1 + s] = 0.0;
        }
    }
    block_sum<4, NT>(acc, scratch);
    if (threadIdx.x == 0) {
        rec[R_ES] = acc[0];
        rec[R_ED] = acc[1];
        rec[R_K2ED] = acc[2];
        rec[R_KMED] = acc[3];
        // solution.F90:69-81: a NaN energy stops the run with this step's state and counters
        if (halt && halt_code && isnan(acc[0] + acc[1])) *halt = halt_code;
    }
}

// One work item per block: its run of list entries, U entries per thread with their index and
// state loads issued together; then the last block to finish forms the shell sums.
// pend = (pending, factor): the previous step's linear-forcing scale u *= factor, applied here
// to every mode that can be non-zero (|k| < K; the others are zero) before its spectra, then
// cleared by the last block.
template <int D, int NT>
__global__ void __launch_bounds__(NT) k_spectra_fused(double2* __restrict__ U0, Geo g, double2* pend,
                                                      const int* __restrict__ modes,
                                                      const int* __restrict__ item_lo,
                                                      double* item_part /* [items][4] */,
                                                      unsigned int* done, const int* __restrict__ shell_item,
                                                      int nshell, int allkmax, double* __restrict__ rec,
                                                      double* __restrict__ shells_out, unsigned int halt_code) {
    pdl_wait();
    if (halted(g)) return;
    __shared__ double scratch[4 * NT];
    __shared__ unsigned int flag;
    constexpr int U = BASTR_SPECTRA_U;
    const int lo = item_lo[blockIdx.x], hi = item_lo[blockIdx.x + 1];
    const double2 pd = pend[0];
    const bool scale = pd.x != 0.0;
    if (scale && blockIdx.x == 0 && threadIdx.x == 0) {
        // the k = 0 mode is in no shell list (it adds nothing to the spectra) but is scaled too
        const size_t cst = D == 2 ? 1 : (size_t)g.ps;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const double2 v = U0[c * cst];
            U0[c * cst] = make_double2(pd.y * v.x, pd.y * v.y);
        }
    }
    double acc[4] = {0, 0, 0, 0};
    for (int i0 = lo + threadIdx.x; i0 < hi; i0 += U * NT) {
        int m[U];
#pragma unroll
        for (int j = 0; j < U; ++j) m[j] = i0 + j * NT < hi ? modes[i0 + j * NT] : -1;
#pragma unroll
        for (int j = 0; j < U; ++j) {
            if (m[j] < 0) continue;
            if constexpr (D == 2) {
                const int kx = m[j] / g.KY, kyi = m[j] - kx * g.KY;
                spectra_mode<2>(U0, g, kx, trunc_k(kyi, g.K, g.KY), 0, acc, scale, pd.y);
            } else {
                const int kzi = m[j] % g.KZ, r = m[j] / g.KZ;
                const int kx = r / g.KY, kyi = r - kx * g.KY;
                spectra_mode<3>(U0, g, kx, trunc_k(kyi, g.K, g.KY), trunc_k(kzi, g.K, g.KZ), acc, scale, pd.y);
            }
        }
    }
    block_sum<4, NT>(acc, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) item_part[(size_t)blockIdx.x * 4 + i] = acc[i];
    }
    if (!last_block_arrives(done, &flag)) return;
    spectra_finish<NT>(item_part, shell_item, nshell, allkmax, rec, shells_out, scratch, g.halt, halt_code);
    if (threadIdx.x == 0) {
        *done = 0;
        pend[0].x = 0.0;   // every block has read it
    }
}

// Shell sums alone (used when no mode survives the truncation: every shell is empty, and a
// pending scale has nothing to act on).
template <int NT>
__global__ void __launch_bounds__(NT) k_spectra_items_final(const double* __restrict__ item_part,
                                                            const int* __restrict__ shell_item, int nshell,
                                                            int allkmax, double* __restrict__ rec,
                                                            double* __restrict__ shells_out, double2* pend,
                                                            Geo g, unsigned int halt_code) {
    pdl_wait();
    if (halted(g)) return;
    __shared__ double scratch[4 * NT];
    spectra_finish<NT>(item_part, shell_item, nshell, allkmax, rec, shells_out, scratch, g.halt, halt_code);
    if (threadIdx.x == 0) pend[0].x = 0.0;
}

// velgrad_calculate2D/3D, solution.F90:1168-1184 / 1268-1284: sums of the nblk per-block
// partials [7 sums, max|theta|] in fixed order and the derived statistics.  Run by one whole
// block (scratch: 7*NT doubles); reads the partials through L2.
template <int NT>
__device__ __forceinline__ void velgrad_finish(const double* part, int nblk, const Geo& g,
                                               double* __restrict__ rec, double* scratch) {
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double dm = 0.0;   // largest |theta| over the grid
    for (int b = threadIdx.x; b < nblk; b += NT) {
#pragma unroll
        for (int i = 0; i < 7; ++i) acc[i] += __ldcg(part + (size_t)b * 8 + i);
        dm = fmax(dm, __ldcg(part + (size_t)b * 8 + 7));
    }
    block_sum<7, NT>(acc, scratch);
    dm = -block_min<NT>(-dm, scratch);
    if (threadIdx.x == 0) {
        const double N = (double)g.nx * (double)g.ny * (double)g.nz;
        const double nu = g.nu;
        const double dd = (double)g.d;
        const double umumtheta2 = acc[0] / N;
        const double umumijji = acc[1] / N;
        const double u2theta = acc[2] / N;
        const double dissp = acc[3] / N;
        const double epsilon = acc[4] / N;
        // eta_min starts at the default-real product 2*3.14 (solution.F90:1145, 1236); the
        // minimum of sqrt(nu/|theta|) over the points is sqrt(nu/max|theta|)
        const double eta0 = (double)(2.0f * 3.14f);
        const double eta_min = fmin(eta0, sqrt(nu / dm));
        const double urms = sqrt(acc[5] / N);
        const double dudx2 = acc[6] / N;
        const double ufluc = urms / sqrt(dd);
        const double tay = ufluc / sqrt(dudx2 / dd);
        const double retay = ufluc * tay / nu;
        const double kol = sqrt(sqrt(nu * nu * nu / epsilon));
        rec[R_VG0 + 0] = umumtheta2;
        rec[R_VG0 + 1] = umumijji;
        rec[R_VG0 + 2] = u2theta;
        rec[R_VG0 + 3] = dissp;
        rec[R_VG0 + 4] = eta_min;
        rec[R_VG0 + 5] = tay;
        rec[R_VG0 + 6] = retay;
        rec[R_VG0 + 7] = kol;
    }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_velgrad_final(const double* __restrict__ part, int nblk,
                                                      Geo g, double* __restrict__ rec) {
    pdl_wait();
    if (halted(g)) return;
    __shared__ double scratch[7 * NT];
    velgrad_finish<NT>(part, nblk, g, rec, scratch);
}

// Sum of per-block partials in fixed order -> rec[slot] (scaled).
template <int NT>
__global__ void __launch_bounds__(NT) k_sum_partials(const double* __restrict__ part, int n, double scale,
                                                     double* __restrict__ rec, int slot, Geo g) {
    pdl_wait();
    if (halted(g)) return;
    __shared__ double scratch[NT];
    double acc[1] = {0};
    for (int b = threadIdx.x; b < n; b += NT) acc[0] += part[b];
    block_sum<1, NT>(acc, scratch);
    if (threadIdx.x == 0) rec[slot] = acc[0] * scale;
}

// Linear forcing, method 1 (solution.F90:315-378): the energy partials of the last stage sum in
// fixed order to sum_k w|u^|^2 = mean(|u|^2) (Parseval with the 1/N forward normalisation);
// factor = sqrt(target / mean(|u|^2/2)).  The scale u *= factor itself is left pending: the
// next step's spectra kernel (or k_apply_pending) applies it.
// With vg_nblk > 0 the kernel is launched with a second block that finishes the step's
// velocity-gradient statistics from the x pass's partials beside the forcing (they are read only
// from the record, so they need no launch of their own).
template <int NT>
__global__ void __launch_bounds__(NT) k_force_linear(const double* __restrict__ part, int n,
                                                     double* __restrict__ rec, double target, double2* pend,
                                                     const double* __restrict__ vg_part, int vg_nblk, Geo g) {
    pdl_wait();
    if (halted(g)) return;
    __shared__ double scratch[7 * NT];
    if (blockIdx.x == 1) {   // launched with vg_nblk > 0: the statistics in a block of their own
        velgrad_finish<NT>(vg_part, vg_nblk, g, rec, scratch);
        return;
    }
    double acc[1] = {0};
    for (int b = threadIdx.x; b < n; b += NT) acc[0] += part[b];
    block_sum<1, NT>(acc, scratch);
    if (threadIdx.x == 0) {
        rec[R_ENERGY] = acc[0];
        const double factor = sqrt(target / (acc[0] / 2.0));
        rec[R_FACTOR] = factor;
        rec[R_E] = 0.0 / 0.0;
        pend[0] = make_double2(1.0, factor);
    }
}

// Applies a pending linear-forcing scale to the whole state (before the host reads it).
__global__ void k_apply_pending(double2* __restrict__ U0, size_t n, const double2* __restrict__ pend) {
    const double2 pd = pend[0];
    if (pd.x == 0.0) return;
    const double f = pd.y;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double2 v = U0[i];
        U0[i] = make_double2(f * v.x, f * v.y);
    }
}

// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC 2011): 10 rounds of two 32x32 -> 64-bit multiplies on a 128-bit counter, key bumped by the
// Weyl constants between rounds.
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// Random phase in [-pi, pi) of band mode (kx >= 0, ky, kz) at forcing call `ctr`: the mode's
// canonical half (kx > 0, or kx = 0 with (ky, kz) > 0 lexicographically) draws it, its
// Hermitian partner on kx = 0 takes the negative, so the force stays real.
__device__ __forceinline__ double band_phase(int kx, int ky, int kz, unsigned long long ctr) {
    double sgn = 1.0;
    if (kx == 0 && (ky < 0 || (ky == 0 && kz < 0))) { ky = -ky; kz = -kz; sgn = -1.0; }
    uint32_t c[4] = {(uint32_t)kx | ((uint32_t)(ky + 1024) << 11), (uint32_t)(kz + 1024), (uint32_t)ctr,
                     (uint32_t)(ctr >> 32)};
    philox4x32_10(c, 0xB5A57F01u, 0x7E5D0C2Bu);
    const double u = ((double)c[0] + 0.5) * (1.0 / 4294967296.0);
    return sgn * (2.0 * 3.141592653589793 * u - 3.141592653589793);
}

// Band forcing, methods 2-5: the band |kk - forcek| < 1/2 is exactly the shell nint(kk) =
// forcek (no integer |k|^2 lies on a half-integer radius), whose kept modes are the entries
// band_lo .. band_hi-1 of the spectra's shell-sorted mode list; the threads of the one block
// take one entry each (forcek = 0: the k = 0 mode alone).  Methods 2 and 5: f = the band part of
// u, E = mean(f^2) in fixed order, then u += factor*f.  Methods 3 and 4 (solution.F90:379-482,
// 631-753): f has unit-amplitude dilatational modes k/|k| (sin phi + i cos phi) with random
// phases phi; E = mean(f.u), Fen = mean(f^2), energy = mean(|u|^2) (rec[R_ENERGY]); factor =
// (sqrt(max((target - energy) Fen + E^2, 0)) - E) / Fen (method 3) or target (method 4);
// u += factor*f.  *rng counts the forcing calls (the random stream's counter).
template <int D, int NT>
__global__ void __launch_bounds__(NT) k_force_band(double2* __restrict__ U0, Geo g, int method, int forcek,
                                                   double target, int project2d, double* __restrict__ rec,
                                                   unsigned long long* rng, const double* __restrict__ vg_part,
                                                   int vg_nblk, const int* __restrict__ modes, int band_lo,
                                                   int band_hi) {
    pdl_wait();
    if (halted(g)) return;
    __shared__ double scratch[7 * NT];
    __shared__ double s_factor;
    if (blockIdx.x == 1) {   // the step's velocity-gradient statistics, as k_force_linear does
        velgrad_finish<NT>(vg_part, vg_nblk, g, rec, scratch);
        return;
    }
    const bool rnd = method == 3 || method == 4;
    const unsigned long long ctr = rnd ? *rng : 0ull;
    const size_t cst = D == 2 ? 1 : (size_t)g.ps;
    // entries of the band: list entries, or the k = 0 mode (index -1) for forcek = 0
    const int nband = forcek == 0 ? 1 : band_hi - band_lo;
    // the force of list entry j at its state offset o, and the mode's Hermitian weight
    auto force_of = [&](int j, size_t& o, double& w, double2 (&f)[3]) {
        int kx = 0, kyv = 0, kzv = 0;
        if (forcek != 0) {
            const int idx = modes[band_lo + j];   // ((kx KY + kyi) KZ + kzi)
            const int kzi = D == 3 ? idx % g.KZ : 0;
            const int r = D == 3 ? idx / g.KZ : idx;
            kx = r / g.KY;
            const int kyi = r - kx * g.KY;
            kyv = trunc_k(kyi, g.K, g.KY);
            kzv = D == 3 ? trunc_k(kzi, g.K, g.KZ) : 0;
            o = D == 2 ? (size_t)idx * 2 : (size_t)idx;
        } else {
            o = 0;
        }
        w = kx == 0 ? 1.0 : 2.0;
        const long long m2 = (long long)kx * kx + (long long)kyv * kyv + (long long)kzv * kzv;
        if (rnd) {
            const double phi = band_phase(kx, kyv, kzv, ctr);
            const double kk = sqrt((double)m2);
            const double kv[3] = {(double)kx, (double)kyv, (double)kzv};
            const double2 e = make_double2(sin(phi), cos(phi));
            for (int c = 0; c < D; ++c) f[c] = make_double2(kv[c] / kk * e.x, kv[c] / kk * e.y);
        } else {
            for (int c = 0; c < D; ++c) f[c] = BASTR_AT(U0, o + c * cst, g);
        }
        if (!rnd && D == 2 && project2d) {
            // solution.F90:498-501
            const double kk = sqrt((double)m2);
            const double k1 = kx, k2 = kyv;
            double2 ud;
            ud.x = f[0].x * k1 / kk + f[1].x * k2 / kk;
            ud.y = f[0].y * k1 / kk + f[1].y * k2 / kk;
            f[0] = make_double2(ud.x * k1 / kk, ud.y * k1 / kk);
            f[1] = make_double2(ud.x * k2 / kk, ud.y * k2 / kk);
        }
    };
    // pass 1: E (and Fen), fixed order
    double acc[2] = {0, 0};
    for (int j = threadIdx.x; j < nband; j += NT) {
        size_t o;
        double w;
        double2 f[3];
        force_of(j, o, w, f);
        double e2 = 0, fu = 0;
        for (int c = 0; c < D; ++c) {
            e2 += f[c].x * f[c].x + f[c].y * f[c].y;
            if (rnd) {
                const double2 u = BASTR_AT(U0, o + c * cst, g);
                fu += f[c].x * u.x + f[c].y * u.y;   // Re(f conj(u))
            }
        }
        acc[0] += w * e2;
        acc[1] += w * fu;
    }
    block_sum<2, NT>(acc, scratch);
    if (threadIdx.x == 0) {
        double fac, E;
        if (method == 2) {
            E = acc[0];
            fac = sqrt(target / E) - 1.0;
        } else if (method == 5) {
            E = acc[0];
            const double energy = rec[R_ENERGY];
            fac = target > energy ? sqrt((target - energy) / E + 1.0) - 1.0 : 0.0;
        } else {
            const double fen = acc[0], energy = rec[R_ENERGY];
            E = acc[1];
            fac = method == 3 ? (sqrt(fmax((target - energy) * fen + E * E, 0.0)) - E) / fen : target;
            rec[R_FEN] = fen;
            *rng = ctr + 1;
        }
        rec[R_FACTOR] = fac;
        rec[R_E] = E;
        s_factor = fac;
    }
    __syncthreads();
    // pass 2: u += factor * f on the same entries (each thread the entries it summed)
    const double factor = s_factor;
    for (int j = threadIdx.x; j < nband; j += NT) {
        size_t o;
        double w;
        double2 f[3];
        force_of(j, o, w, f);
        for (int c = 0; c < D; ++c) {
            const double2 u = BASTR_AT(U0, o + c * cst, g);
            BASTR_AT(U0, o + c * cst, g) = make_double2(u.x + factor * f[c].x, u.y + factor * f[c].y);
        }
    }
}

}  // namespace bastr
