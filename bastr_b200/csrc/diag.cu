// Per-step diagnostics and forcing on the truncated FP64 state, with deterministic
// (fixed-order) FP64 reductions: two runs on the same input agree bitwise.
//
//  k_spectra        spectra_compute2D/3D (solution.F90:930-1108): one block per shell s,
//                   enumerating exactly the integer |k|^2 in [s^2-s+1, s^2+s] (the modes with
//                   nint(|k|) = s, tool.F90:145); Hermitian partners counted by weight 2.
//  k_spectra_final  shell sums -> Esspe, Edspe, k2Edspe, kMEdspe; copies Es/Ed shells.
//  k_velgrad_final  velgrad_calculate2D/3D reductions and derived lengths (solution.F90:1168-1180,
//                   1268-1280).
//  k_force_*        forcing2D/3D methods 1, 2, 5 (solution.F90:315-378, 483-538, 554-630, 754-812).
#include "solver.cuh"

namespace bastr {

// Record slots (doubles) written per step on the device.
enum RecSlot : int {
    R_ES = 0, R_ED, R_K2ED, R_KMED,
    R_VG0 = 4,            // 8 velocity-gradient statistics, slots 4..11
    R_FACTOR = 12, R_E = 13, R_ENERGY = 14,
    R_COUNT = 16
};

// Largest kx range a 2D shell block enumerates (K <= 682 for grids up to 2048).
constexpr int kSpectraMaxCols = 2048;

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
__device__ __forceinline__ void spectra_mode(const double2* __restrict__ U0, const Geo& g, int kx,
                                             int ky, int kz, double acc[4]) {
    const int K = g.K;
    const int kyi = ky >= 0 ? ky : ky + g.KY;
    const long long m = (long long)kx * kx + (long long)ky * ky + (long long)kz * kz;
    if (m == 0) return;   // kk <= dk/2: us = ud = 0
    const double kk = sqrt((double)m);
    const double w = kx == 0 ? 1.0 : 2.0;
    const double k1 = kx, k2 = ky, k3 = kz;
    double es, ed;
    if constexpr (D == 2) {
        const size_t o = ((size_t)kx * g.KY + kyi) * 2;
        const double2 a = U0[o], b = U0[o + 1];
        // usspe = u1 k2/kk - u2 k1/kk ; udspe = u1 k1/kk + u2 k2/kk  (solution.F90:958-959)
        const double usx = a.x * k2 / kk - b.x * k1 / kk, usy = a.y * k2 / kk - b.y * k1 / kk;
        const double udx = a.x * k1 / kk + b.x * k2 / kk, udy = a.y * k1 / kk + b.y * k2 / kk;
        es = (usx * usx + usy * usy) / 2;
        ed = (udx * udx + udy * udy) / 2;
    } else {
        const int kzi = kz >= 0 ? kz : kz + g.KZ;
        const size_t o = ((size_t)kx * g.KY + kyi) * g.KZ + kzi;
        const double2 a = U0[o], b = U0[o + g.ps], c = U0[o + 2 * g.ps];
        // solution.F90:1047-1053
        const double udx = a.x * k1 / kk + b.x * k2 / kk + c.x * k3 / kk;
        const double udy = a.y * k1 / kk + b.y * k2 / kk + c.y * k3 / kk;
        const double s1x = a.x - udx * k1 / kk, s1y = a.y - udy * k1 / kk;
        const double s2x = b.x - udx * k2 / kk, s2y = b.y - udy * k2 / kk;
        const double s3x = c.x - udx * k3 / kk, s3y = c.y - udy * k3 / kk;
        es = (s1x * s1x + s1y * s1y) / 2 + (s2x * s2x + s2y * s2y) / 2 + (s3x * s3x + s3y * s3y) / 2;
        ed = (udx * udx + udy * udy) / 2;
    }
    (void)K;
    acc[0] += w * es;
    acc[1] += w * ed;
    acc[2] += w * (ed * (kk * kk));
    acc[3] += w * (ed / kk);
}

template <int D, int NT>
__global__ void __launch_bounds__(NT) k_spectra(const double2* __restrict__ U0, Geo g,
                                                double* __restrict__ shell /* [SH][4] */) {
    __shared__ double scratch[4 * NT];
    const int s = blockIdx.x;
    const int K = g.K;
    const long long lo = s == 0 ? 0 : (long long)s * s - s + 1;
    long long hi = s == 0 ? 0 : (long long)s * s + s;
    const long long K2m1 = (long long)K * K - 1;   // kept modes have |k|^2 < K^2
    if (hi > K2m1) hi = K2m1;
    double acc[4] = {0, 0, 0, 0};
    if (lo <= hi) {
        const int kmax = s < K - 1 ? s : K - 1;
        if constexpr (D == 2) {
            // Flatten the shell: per kx the modes are ky in [a,b] and [-b,-a] (a > 0) so that
            // consecutive threads read consecutive ky of one column.
            __shared__ int off[kSpectraMaxCols + 1];
            __shared__ int ka[kSpectraMaxCols], kb[kSpectraMaxCols];
            for (int kx = threadIdx.x; kx <= kmax; kx += NT) {
                const long long rlo = lo - (long long)kx * kx, rhi = hi - (long long)kx * kx;
                int a = 0, b = -1;
                if (rhi >= 0) {
                    a = (int)isqrt_ceil(rlo);
                    b = (int)isqrt_floor(rhi);
                }
                ka[kx] = a;
                kb[kx] = b;
                off[kx + 1] = b >= a ? 2 * (b - a + 1) - (a == 0 ? 1 : 0) : 0;
            }
            if (threadIdx.x == 0) off[0] = 0;
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int kx = 1; kx <= kmax + 1; ++kx) off[kx] += off[kx - 1];
            }
            __syncthreads();
            const int total = off[kmax + 1];
            for (int idx = threadIdx.x; idx < total; idx += NT) {
                int l = 0, r = kmax;   // last kx with off[kx] <= idx
                while (l < r) {
                    const int m = (l + r + 1) >> 1;
                    if (off[m] <= idx) l = m; else r = m - 1;
                }
                const int kx = l;
                const int rr = idx - off[kx];
                const int a = ka[kx], b = kb[kx];
                const int npos = b - a + 1;
                const int ky = rr < npos ? a + rr : -((a == 0 ? 1 : a) + (rr - npos));
                spectra_mode<2>(U0, g, kx, ky, 0, acc);
            }
        } else {
            const int ny2 = 2 * kmax + 1;
            const int npair = (kmax + 1) * ny2;
            for (int e = threadIdx.x; e < npair; e += NT) {
                const int kx = e / ny2, ky = e - kx * ny2 - kmax;
                const long long rr = (long long)kx * kx + (long long)ky * ky;
                const long long rlo = lo - rr, rhi = hi - rr;
                if (rhi < 0) continue;
                const int a = (int)isqrt_ceil(rlo), b = (int)isqrt_floor(rhi);
                for (int kz = a; kz <= b; ++kz) {
                    spectra_mode<3>(U0, g, kx, ky, kz, acc);
                    if (kz != 0) spectra_mode<3>(U0, g, kx, ky, -kz, acc);
                }
            }
        }
    }
    block_sum<4, NT>(acc, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) shell[(size_t)s * 4 + i] = acc[i];
    }
}

// Shell sums from a precomputed mode list: `modes` holds the state offset (in modes) of every
// kept mode with 0 < |k|^2 < K^2, grouped by shell nint(|k|) and in increasing offset within a
// shell; work item i covers modes [item_lo[i], item_lo[i+1]) of one shell.  One block per item
// writes its four partial sums; consecutive threads read consecutive list entries.
template <int D, int NT>
__global__ void __launch_bounds__(NT) k_spectra_items(const double2* __restrict__ U0, Geo g,
                                                      const int* __restrict__ modes,
                                                      const int* __restrict__ item_lo,
                                                      double* __restrict__ item_part /* [items][4] */) {
    __shared__ double scratch[4 * NT];
    const int lo = item_lo[blockIdx.x], hi = item_lo[blockIdx.x + 1];
    double acc[4] = {0, 0, 0, 0};
    for (int i = lo + threadIdx.x; i < hi; i += NT) {
        const int m = modes[i];
        if constexpr (D == 2) {
            const int kx = m / g.KY, kyi = m - kx * g.KY;
            spectra_mode<2>(U0, g, kx, trunc_k(kyi, g.K, g.KY), 0, acc);
        } else {
            const int kzi = m % g.KZ, r = m / g.KZ;
            const int kx = r / g.KY, kyi = r - kx * g.KY;
            spectra_mode<3>(U0, g, kx, trunc_k(kyi, g.K, g.KY), trunc_k(kzi, g.K, g.KZ), acc);
        }
    }
    block_sum<4, NT>(acc, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) item_part[(size_t)blockIdx.x * 4 + i] = acc[i];
    }
}

// Per-shell sums of the work items (items of shell s are shell_item[s] .. shell_item[s+1]-1),
// totals over all shells in fixed order, and the copy of shells 0..allkmax for the spect log.
template <int NT>
__global__ void __launch_bounds__(NT) k_spectra_items_final(const double* __restrict__ item_part,
                                                            const int* __restrict__ shell_item, int nshell,
                                                            int allkmax, double* __restrict__ rec,
                                                            double* __restrict__ shells_out) {
    __shared__ double scratch[4 * NT];
    double acc[4] = {0, 0, 0, 0};
    for (int s = threadIdx.x; s < nshell; s += NT) {
        double sh[4] = {0, 0, 0, 0};
        for (int it = shell_item[s]; it < shell_item[s + 1]; ++it) {
#pragma unroll
            for (int i = 0; i < 4; ++i) sh[i] += item_part[(size_t)it * 4 + i];
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
    }
}

// Totals over all shells (fixed order) and a copy of shells 0..allkmax for the spect log.
template <int NT>
__global__ void __launch_bounds__(NT) k_spectra_final(const double* __restrict__ shell, int nshell,
                                                      int allkmax, double* __restrict__ rec,
                                                      double* __restrict__ shells_out /* [2][allkmax+1] */) {
    __shared__ double scratch[4 * NT];
    double acc[4] = {0, 0, 0, 0};
    for (int s = threadIdx.x; s < nshell; s += NT) {
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i] += shell[(size_t)s * 4 + i];
    }
    block_sum<4, NT>(acc, scratch);
    if (threadIdx.x == 0) {
        rec[R_ES] = acc[0];
        rec[R_ED] = acc[1];
        rec[R_K2ED] = acc[2];
        rec[R_KMED] = acc[3];
    }
    if (shells_out) {
        for (int s = threadIdx.x; s <= allkmax; s += NT) {
            shells_out[s] = s < nshell ? shell[(size_t)s * 4 + 0] : 0.0;
            shells_out[allkmax + 1 + s] = s < nshell ? shell[(size_t)s * 4 + 1] : 0.0;
        }
    }
}

// velgrad_calculate2D/3D, solution.F90:1168-1184 / 1268-1284.
template <int NT>
__global__ void __launch_bounds__(NT) k_velgrad_final(const double* __restrict__ part, int nblk,
                                                      Geo g, double* __restrict__ rec) {
    __shared__ double scratch[7 * NT];
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double dm = 0.0;   // largest |theta| over the grid
    for (int b = threadIdx.x; b < nblk; b += NT) {
#pragma unroll
        for (int i = 0; i < 7; ++i) acc[i] += part[(size_t)b * 8 + i];
        dm = fmax(dm, part[(size_t)b * 8 + 7]);
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

// Sum of per-block partials in fixed order -> rec[slot] (scaled).
template <int NT>
__global__ void __launch_bounds__(NT) k_sum_partials(const double* __restrict__ part, int n, double scale,
                                                     double* __restrict__ rec, int slot) {
    __shared__ double scratch[NT];
    double acc[1] = {0};
    for (int b = threadIdx.x; b < n; b += NT) acc[0] += part[b];
    block_sum<1, NT>(acc, scratch);
    if (threadIdx.x == 0) rec[slot] = acc[0] * scale;
}

// Linear forcing, method 1: factor = sqrt(target / mean(|u|^2/2)).  rec[R_ENERGY] holds
// sum_k w|u^|^2 = mean(|u|^2) (Parseval with the 1/N forward normalisation).
__global__ void k_force_linear_factor(double* __restrict__ rec, double target) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const double energy = rec[R_ENERGY] / 2.0;
        rec[R_FACTOR] = sqrt(target / energy);
        rec[R_E] = 0.0 / 0.0;
    }
}

__global__ void k_scale_state(double2* __restrict__ U0, size_t n, const double* __restrict__ rec) {
    const double f = rec[R_FACTOR];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double2 v = U0[i];
        U0[i] = make_double2(f * v.x, f * v.y);
    }
}

// Band forcing, methods 2 and 5: the band |kk - forcek| < 1/2 is exactly the shell nint(kk) =
// forcek.  One block enumerates it, reduces E = mean(f^2) in fixed order, then adds factor*f.
template <int D, int NT>
__global__ void __launch_bounds__(NT) k_force_band(double2* __restrict__ U0, Geo g, int method, int forcek,
                                                   double target, int project2d, double* __restrict__ rec) {
    __shared__ double scratch[NT];
    const int s = forcek;
    const int K = g.K;
    const long long lo = s == 0 ? 0 : (long long)s * s - s + 1;
    long long hi = s == 0 ? 0 : (long long)s * s + s;
    const long long K2m1 = (long long)K * K - 1;
    if (hi > K2m1) hi = K2m1;
    const int kmax = s < K - 1 ? s : K - 1;
    const int ny2 = 2 * kmax + 1;
    const int npair = D == 2 ? (kmax + 1) : (kmax + 1) * ny2;

    // pass 1 (sum) and pass 2 (apply) walk the same modes in the same order
    for (int phase = 0; phase < 2; ++phase) {
        double acc[1] = {0};
        double factor = 0;
        if (phase == 1) factor = rec[R_FACTOR];
        if (lo <= hi) {
            for (int e = threadIdx.x; e < npair; e += NT) {
                int kx, ky = 0;
                long long rr;
                if (D == 2) { kx = e; rr = (long long)kx * kx; }
                else { kx = e / ny2; ky = e - kx * ny2 - kmax; rr = (long long)kx * kx + (long long)ky * ky; }
                const long long rlo = lo - rr, rhi = hi - rr;
                if (rhi < 0) continue;
                const int a = (int)isqrt_ceil(rlo), b = (int)isqrt_floor(rhi);
                for (int t = a; t <= b; ++t) {
                    for (int sg = 0; sg < (t == 0 ? 1 : 2); ++sg) {
                        const int tt = sg ? -t : t;
                        const double w = kx == 0 ? 1.0 : 2.0;
                        size_t o;
                        int kyv, kzv;
                        if (D == 2) {
                            kyv = tt; kzv = 0;
                            const int kyi = kyv >= 0 ? kyv : kyv + g.KY;
                            o = ((size_t)kx * g.KY + kyi) * 2;
                        } else {
                            kyv = ky; kzv = tt;
                            const int kyi = kyv >= 0 ? kyv : kyv + g.KY;
                            const int kzi = kzv >= 0 ? kzv : kzv + g.KZ;
                            o = ((size_t)kx * g.KY + kyi) * g.KZ + kzi;
                        }
                        double2 f[3];
                        const size_t cst = D == 2 ? 1 : (size_t)g.ps;
                        for (int c = 0; c < D; ++c) f[c] = U0[o + c * cst];
                        if (D == 2 && project2d) {
                            // solution.F90:498-501
                            const double kk = sqrt((double)(rr + (long long)tt * tt));
                            const double k1 = kx, k2 = kyv;
                            double2 ud;
                            ud.x = f[0].x * k1 / kk + f[1].x * k2 / kk;
                            ud.y = f[0].y * k1 / kk + f[1].y * k2 / kk;
                            f[0] = make_double2(ud.x * k1 / kk, ud.y * k1 / kk);
                            f[1] = make_double2(ud.x * k2 / kk, ud.y * k2 / kk);
                        }
                        if (phase == 0) {
                            double e2 = 0;
                            for (int c = 0; c < D; ++c) e2 += f[c].x * f[c].x + f[c].y * f[c].y;
                            acc[0] += w * e2;
                        } else {
                            for (int c = 0; c < D; ++c) {
                                double2 u = U0[o + c * cst];
                                U0[o + c * cst] = make_double2(u.x + factor * f[c].x, u.y + factor * f[c].y);
                            }
                        }
                    }
                }
            }
        }
        if (phase == 0) {
            block_sum<1, NT>(acc, scratch);
            if (threadIdx.x == 0) {
                const double E = acc[0];
                double fac;
                if (method == 2) {
                    fac = sqrt(target / E) - 1.0;
                } else {
                    const double energy = rec[R_ENERGY];
                    fac = target > energy ? sqrt((target - energy) / E + 1.0) - 1.0 : 0.0;
                }
                rec[R_FACTOR] = fac;
                rec[R_E] = E;
            }
            __syncthreads();
        }
    }
}

}  // namespace bastr
