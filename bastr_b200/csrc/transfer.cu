// Energy transfer spectra of the current state: Bastrpp's transfer2d / transfer3d
// (Bastrpp.F90:174-305, 418-599), FP64, on full complex grids with the full-grid transforms of
// fullfft.cu.
//
//   u^ = the state;  d_cj = IFFT(i k_j u^_c);  u_c = IFFT(u^_c)            (physical, real)
//   tA_c = -u_j d_cj,  tC_c = u_c d_jj,  P_cj = u_c u_j                     (physical)
//   per mode: trans  = sum_c Re(conj(u^_c) FFT(tA_c))
//             trans1 = sum_c sum_j Im(k_j FFT(P_cj) conj(u^_c))
//             trans2 = sum_c Re(conj(u^_c) FFT(tC_c))
//   T(s), T1(s), T2(s) = sums over the modes of shell nint(|k|) = s.
//
// Only modes with u^ != 0 contribute, i.e. the stored half spectrum |k| < K; a mode and its
// Hermitian partner contribute equal values, so the stored modes are summed with weight 2
// (1 on kx = 0) through the shell lists of the spectra (fixed order: deterministic).
#pragma once
#include "diag.cu"
#include "solver.cuh"

namespace bastr {

__device__ __forceinline__ int full_k(int i, int n) { return i <= n / 2 ? i : i - n; }

// Full complex grids [nz][ny][nx] of the state's components (zeros elsewhere): every stored mode
// and, for kx > 0, its conjugate partner.  Grid i = kx (x) etc.; truncated index kyi, kzi.
template <int D>
__global__ void k_tr_scatter(const double2* __restrict__ U0, Geo g, double2* __restrict__ F, size_t nfull) {
    const size_t nmodes = (size_t)g.K * g.KY * g.KZ;
    const size_t cst = D == 2 ? 1 : (size_t)g.ps;
    for (size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x; m < nmodes; m += (size_t)gridDim.x * blockDim.x) {
        const int kzi = (int)(m % g.KZ), kyi = (int)((m / g.KZ) % g.KY), kx = (int)(m / ((size_t)g.KZ * g.KY));
        const int ky = trunc_k(kyi, g.K, g.KY), kz = D == 3 ? trunc_k(kzi, g.K, g.KZ) : 0;
        const size_t o = D == 2 ? ((size_t)kx * g.KY + kyi) * 2 : m;
        const int iy = (ky + g.ny) % g.ny, iz = (kz + g.nz) % g.nz;
        const int jy = (g.ny - ky) % g.ny, jz = (g.nz - kz) % g.nz, jx = (g.nx - kx) % g.nx;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const double2 v = U0[o + c * cst];
            double2* Fc = F + (size_t)c * nfull;
            Fc[((size_t)iz * g.ny + iy) * g.nx + kx] = v;
            if (kx > 0) Fc[((size_t)jz * g.ny + jy) * g.nx + jx] = make_double2(v.x, -v.y);
        }
    }
}

// dst = i k_axis src over a full grid.
__global__ void k_tr_deriv(const double2* __restrict__ src, double2* __restrict__ dst, int axis, Geo g) {
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(p % g.nx), iy = (int)((p / g.nx) % g.ny), iz = (int)(p / ((size_t)g.nx * g.ny));
        const double k = axis == 0 ? full_k(ix, g.nx) : axis == 1 ? full_k(iy, g.ny) : full_k(iz, g.nz);
        const double2 v = src[p];
        dst[p] = make_double2(-k * v.y, k * v.x);
    }
}

// Point products from physical u_c (U, D arrays) and d_cj (Dv, index c*D + j): writes tA (D
// arrays), tC (D) and P_cj (D*D), all real (imaginary part 0).
template <int D>
__global__ void k_tr_products(const double2* __restrict__ U, const double2* __restrict__ Dv, double2* __restrict__ tA,
                              double2* __restrict__ tC, double2* __restrict__ P, size_t n) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        double u[D], d[D][D];
#pragma unroll
        for (int c = 0; c < D; ++c) {
            u[c] = U[c * n + p].x;
#pragma unroll
            for (int j = 0; j < D; ++j) d[c][j] = Dv[(size_t)(c * D + j) * n + p].x;
        }
        double th = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) th += d[j][j];
#pragma unroll
        for (int c = 0; c < D; ++c) {
            double a = 0;
#pragma unroll
            for (int j = 0; j < D; ++j) a -= u[j] * d[c][j];
            tA[c * n + p] = make_double2(a, 0.0);
            tC[c * n + p] = make_double2(u[c] * th, 0.0);
#pragma unroll
            for (int j = 0; j < D; ++j) P[(size_t)(c * D + j) * n + p] = make_double2(u[c] * u[j], 0.0);
        }
    }
}

// Per stored mode (weight 2 for kx > 0): trans, trans1, trans2 -> tr[mode][3] (mode numbering of
// the shell lists: ((kx*KY + kyi)*KZ + kzi)).
template <int D>
__global__ void k_tr_modes(const double2* __restrict__ U0, Geo g, const double2* __restrict__ tA,
                           const double2* __restrict__ tC, const double2* __restrict__ P, double* __restrict__ tr,
                           size_t nfull) {
    const size_t nmodes = (size_t)g.K * g.KY * g.KZ;
    const size_t cst = D == 2 ? 1 : (size_t)g.ps;
    for (size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x; m < nmodes; m += (size_t)gridDim.x * blockDim.x) {
        const int kzi = (int)(m % g.KZ), kyi = (int)((m / g.KZ) % g.KY), kx = (int)(m / ((size_t)g.KZ * g.KY));
        const int ky = trunc_k(kyi, g.K, g.KY), kz = D == 3 ? trunc_k(kzi, g.K, g.KZ) : 0;
        const size_t o = D == 2 ? ((size_t)kx * g.KY + kyi) * 2 : m;
        const size_t q = ((size_t)((kz + g.nz) % g.nz) * g.ny + (ky + g.ny) % g.ny) * g.nx + kx;
        const double kv[3] = {(double)kx, (double)ky, (double)kz};
        double t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const double2 u = U0[o + c * cst];
            const double2 a = tA[c * nfull + q], b = tC[c * nfull + q];
            t0 += u.x * a.x + u.y * a.y;   // Re(conj(u) a)
            t2 += u.x * b.x + u.y * b.y;
#pragma unroll
            for (int j = 0; j < D; ++j) {
                const double2 pj = P[(size_t)(c * D + j) * nfull + q];
                // Im(k_j pj conj(u)) = k_j (pj.y u.x - pj.x u.y)
                t1 += kv[j] * (pj.y * u.x - pj.x * u.y);
            }
        }
        const double w = kx == 0 ? 1.0 : 2.0;
        tr[m * 3 + 0] = w * t0;
        tr[m * 3 + 1] = w * t1;
        tr[m * 3 + 2] = w * t2;
    }
}

// Shell sums of tr over the shell lists: one block per work item (partials), then per shell in
// fixed order.  out: [3][nshell].
template <int NT>
__global__ void __launch_bounds__(NT) k_tr_items(const double* __restrict__ tr, const int* __restrict__ modes,
                                                 const int* __restrict__ item_lo, double* __restrict__ part) {
    __shared__ double scratch[3 * NT];
    const int lo = item_lo[blockIdx.x], hi = item_lo[blockIdx.x + 1];
    double acc[3] = {0, 0, 0};
    for (int i = lo + threadIdx.x; i < hi; i += NT) {
        const size_t m = (size_t)modes[i];
#pragma unroll
        for (int k = 0; k < 3; ++k) acc[k] += tr[m * 3 + k];
    }
    block_sum<3, NT>(acc, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) part[(size_t)blockIdx.x * 3 + k] = acc[k];
    }
}

__global__ void k_tr_shells(const double* __restrict__ part, const int* __restrict__ shell_item, int nshell,
                            double* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshell) return;
    double a[3] = {0, 0, 0};
    for (int it = shell_item[s]; it < shell_item[s + 1]; ++it) {
#pragma unroll
        for (int k = 0; k < 3; ++k) a[k] += part[(size_t)it * 3 + k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) out[(size_t)k * nshell + s] = a[k];
}

}  // namespace bastr
