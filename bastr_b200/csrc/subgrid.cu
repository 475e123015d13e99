// Filtered fields and the subgrid term of a handle's state, on the device (closure training data).
//
// For a fine state u (the handle's truncated spectral state, FP64) and a box filter of width r
// (mean over r^d cells, decimation r), with spectral derivatives on both grids:
//
//   ub    = filter(u)                                   coarse grid n/r
//   tau_i = filter(u_j d_j u_i) - ub_j d_j ub_i        d_j: i k_j in Fourier space
//
// Fine products: for each component i, sum_j u_j * IFFT(i k_j u^_i) accumulates on the fine grid
// (one complex grid of scratch: the derivative of u^_i scattered from the state with its
// Hermitian partners, then the full-grid inverse transforms of fullfft.cu), and is box-filtered.
// Coarse products: ub_i goes to Fourier space with the forward full-grid transform (scaled 1/N),
// each derivative comes back with the inverse one.  No reference counterpart: the reference has
// no closure; this is the data path of the learned closure, restating in kernels the host
// pipeline it replaces (box_filter and the spectral u.grad u in bastr_b200/closure.py).
#pragma once
#include "solver.cuh"

namespace bastr {

__device__ __forceinline__ int sg_wave(int i, int n) { return i <= n / 2 ? i : i - n; }

// W = i k_axis u^_comp (axis < 0: u^_comp itself) of the truncated state on the full complex grid
// [nz][ny][nx], with the conjugate partner of every kx > 0 mode.  W must be zero elsewhere.
template <int D>
__global__ void k_sg_scatter(const double2* __restrict__ U0, Geo g, int comp, int axis, double2* __restrict__ W) {
    const size_t nmodes = (size_t)g.K * g.KY * g.KZ;
    const size_t cst = D == 2 ? 1 : (size_t)g.ps;
    for (size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x; m < nmodes; m += (size_t)gridDim.x * blockDim.x) {
        const int kzi = (int)(m % g.KZ), kyi = (int)((m / g.KZ) % g.KY), kx = (int)(m / ((size_t)g.KZ * g.KY));
        const int ky = trunc_k(kyi, g.K, g.KY), kz = D == 3 ? trunc_k(kzi, g.K, g.KZ) : 0;
        const size_t o = D == 2 ? ((size_t)kx * g.KY + kyi) * 2 : m;
        double2 v = U0[o + comp * cst];
        if (axis >= 0) {
            const double k = axis == 0 ? kx : axis == 1 ? ky : kz;
            v = make_double2(-k * v.y, k * v.x);
        }
        const int iy = (ky + g.ny) % g.ny, iz = (kz + g.nz) % g.nz;
        W[((size_t)iz * g.ny + iy) * g.nx + kx] = v;
        if (kx > 0) {
            const int jy = (g.ny - ky) % g.ny, jz = (g.nz - kz) % g.nz, jx = g.nx - kx;
            W[((size_t)jz * g.ny + jy) * g.nx + jx] = make_double2(v.x, -v.y);
        }
    }
}

// acc = (first ? 0 : acc) + u * Re(W), over n points.
__global__ void k_sg_accum(double* __restrict__ acc, const double* __restrict__ u, const double2* __restrict__ W,
                           size_t n, int first) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const double t = u[p] * W[p].x;
        acc[p] = first ? t : acc[p] + t;
    }
}

// Box filter: dst[cell] = mean of the r^d fine points of the cell; fine [nz][ny][nx], coarse
// [nz/r][ny/r][nx/r] (nz = 1 in 2D).
__global__ void k_sg_filter(const double* __restrict__ src, int nx, int ny, int nz, int r, int d,
                            double* __restrict__ dst) {
    const int cx = nx / r, cy = ny / r, cz = d == 3 ? nz / r : 1;
    const size_t nc = (size_t)cx * cy * cz;
    const int rz = d == 3 ? r : 1;
    const double w = 1.0 / ((double)r * r * rz);
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(c % cx), iy = (int)((c / cx) % cy), iz = (int)(c / ((size_t)cx * cy));
        double s = 0.0;
        for (int a = 0; a < rz; ++a)
            for (int b = 0; b < r; ++b) {
                const double* row = src + (((size_t)iz * rz + a) * ny + (size_t)iy * r + b) * nx + (size_t)ix * r;
                for (int e = 0; e < r; ++e) s += row[e];
            }
        dst[c] = s * w;
    }
}

// Real field -> complex grid (imaginary part zero).
__global__ void k_sg_complex(const double* __restrict__ src, double2* __restrict__ dst, size_t n) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        dst[p] = make_double2(src[p], 0.0);
}

// dst = i k_axis src on a full complex grid [nz][ny][nx].
__global__ void k_sg_deriv(const double2* __restrict__ src, double2* __restrict__ dst, int nx, int ny, int nz,
                           int axis) {
    const size_t n = (size_t)nx * ny * nz;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(p % nx), iy = (int)((p / nx) % ny), iz = (int)(p / ((size_t)nx * ny));
        const double k = axis == 0 ? sg_wave(ix, nx) : axis == 1 ? sg_wave(iy, ny) : sg_wave(iz, nz);
        const double2 v = src[p];
        dst[p] = make_double2(-k * v.y, k * v.x);
    }
}

// tau = fadv - cadv and ub, as FP32 outputs.
__global__ void k_sg_finish(const double* __restrict__ fadv, const double* __restrict__ cadv,
                            const double* __restrict__ ub, float* __restrict__ tau, float* __restrict__ ubar,
                            size_t n) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        if (tau) tau[p] = (float)(fadv[p] - cadv[p]);
        if (ubar) ubar[p] = (float)ub[p];
    }
}

}  // namespace bastr
