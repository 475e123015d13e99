// Initial-field generators of Bastrpp (commands hitgen2d, hitgen2dbis, hitgen3d):
// create_initial_field_2d (Bastrpp.F90:601-696), create_initial_field_3d (:698-808) and
// create_initial_field_2d_bis (:810-1005), FP64 on full complex grids [nz][ny][nx].
//
//   r = uniform (0,1) per grid point;  R = FFT(r) (forward, scaled 1/N)
//   per mode k != 0:  theta = atan2(Im R, Re R),  u^_c = A(|k|) k_c/|k| (sin theta + i cos theta)
//        A = sqrt(E(|k|) / (2 pi |k|)) in 2D, sqrt(E(|k|) / (4 pi |k|^2)) in 3D,
//        E(k) = k^4 exp(-2 (k/forcek)^2) for k >= forcek, forcek^6 / k^2 exp(-2) below
//        (the _bis generator uses the first branch for every k)
//   u_c = Re IFFT(u^_c);  factor = sqrt(target / mean(sum_c u_c^2));  u_c *= factor
// The reference keeps `random_angle` = theta on every mode and the uniform value at k = 0.
//
// _bis draws two such fields A and B (with theta_X = Re IFFT(i k.u^_X)), forms the grid means
// QX = <|uA|^2 thA>, QY = <2 uB.uA thA + |uA|^2 thB>, QZ = <2 uA.uB thB + |uB|^2 thA>,
// QW = <|uB|^2 thB>, takes the real root alpha of QX + QY a + QZ a^2 + QW a^3 = 0 by the
// reference's Cardano / trigonometric formulas and returns u = uA + alpha uB, scaled as above
// (so that <|u|^2 theta> = 0).
//
// The uniform numbers come from Philox-4x32-10 (key = the 64-bit seed, counter = (point index
// lo, hi, draw, tag)) instead of gfortran's random_number: the spectrum of every mode is
// the reference's exactly; the phases agree with it in distribution only.
#pragma once
#include "diag.cu"
#include "solver.cuh"
#include "transfer.cu"

namespace bastr {

constexpr uint32_t HITGEN_TAG = 0x48475431u;

// 53-bit uniform in (0, 1) of point p of draw `draw`.
__host__ __device__ inline double hitgen_uniform(unsigned long long p, int draw, unsigned long long seed) {
    uint32_t c[4] = {(uint32_t)p, (uint32_t)(p >> 32), (uint32_t)draw, HITGEN_TAG};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const unsigned long long x = ((unsigned long long)c[0] << 32) | c[1];
    return ((double)(x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

__global__ void k_hg_uniform(double2* __restrict__ R, double* __restrict__ angle, size_t n, int draw,
                             unsigned long long seed) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const double u = hitgen_uniform(p, draw, seed);
        R[p] = make_double2(u, 0.0);
        angle[p] = u;
    }
}

// Modes of one draw: F[c] (c < D) = u^_c, and with `with_theta` F[D] = i (kx u^_1 + ky u^_2).
template <int D>
__global__ void k_hg_modes(const double2* __restrict__ R, double2* __restrict__ F, double* __restrict__ angle, Geo g,
                           double forcek, int bis, int with_theta) {
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    const double pi = 3.14159265358979323846;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(p % g.nx), iy = (int)((p / g.nx) % g.ny), iz = (int)(p / ((size_t)g.nx * g.ny));
        const double k[3] = {(double)full_k(ix, g.nx), (double)full_k(iy, g.ny), D == 3 ? (double)full_k(iz, g.nz) : 0.0};
        double kk2 = 0.0;
#pragma unroll
        for (int c = 0; c < D; ++c) kk2 += k[c] * k[c];
        if (kk2 == 0.0) {
#pragma unroll
            for (int c = 0; c < D; ++c) F[(size_t)c * n + p] = make_double2(0.0, 0.0);
            if (with_theta) F[(size_t)D * n + p] = make_double2(0.0, 0.0);
            continue;   // angle keeps the uniform value here, as in the reference
        }
        const double kk = sqrt(kk2);
        const double var1 = (bis || kk >= forcek) ? kk * kk * kk * kk * exp(-2.0 * (kk / forcek) * (kk / forcek))
                                                  : forcek * forcek * forcek * forcek * forcek * forcek / (kk * kk) * exp(-2.0);
        const double var2 = D == 2 ? sqrt(var1 / 2.0 / pi / kk) : sqrt(var1 / 4.0 / pi / (kk * kk));
        const double2 r = R[p];
        const double th = atan2(r.y, r.x);
        angle[p] = th;
        double s, co;
        sincos(th, &s, &co);
        double2 u[D];
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const double a = var2 * k[c] / kk;
            u[c] = make_double2(a * s, a * co);
            F[(size_t)c * n + p] = u[c];
        }
        if (with_theta) {
            // (0, 1) * (kx u1 + ky u2)
            const double re = k[0] * u[0].x + k[1] * u[1].x, im = k[0] * u[0].y + k[1] * u[1].y;
            F[(size_t)D * n + p] = make_double2(-im, re);
        }
    }
}

// Per-block partial sums over grid points of real parts: mode 0 -> sum_c Re(A_c)^2 (+ alpha B_c
// combined first when B != null); mode 1 -> the four Q sums of the _bis generator (2D).
template <int NT>
__global__ void __launch_bounds__(NT) k_hg_sums(const double2* __restrict__ A, const double2* __restrict__ B,
                                                double alpha, int ncomp, size_t n, int mode, double* __restrict__ part) {
    __shared__ double scratch[4 * NT];
    double acc[4] = {0, 0, 0, 0};
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        if (mode == 0) {
            for (int c = 0; c < ncomp; ++c) {
                double v = A[(size_t)c * n + p].x;
                if (B) v = v + alpha * B[(size_t)c * n + p].x;
                acc[0] += v * v;
            }
        } else {
            const double a1 = A[p].x, a2 = A[n + p].x, ta = A[2 * n + p].x;
            const double b1 = B[p].x, b2 = B[n + p].x, tb = B[2 * n + p].x;
            const double aa = a1 * a1 + a2 * a2, bb = b1 * b1 + b2 * b2, ab = b1 * a1 + b2 * a2;
            acc[0] += aa * ta;
            acc[1] += 2.0 * ab * ta + aa * tb;
            acc[2] += 2.0 * (a1 * b1 + a2 * b2) * tb + bb * ta;
            acc[3] += bb * tb;
        }
    }
    block_sum<4, NT>(acc, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) part[(size_t)blockIdx.x * 4 + i] = acc[i];
    }
}

// out[c][p] = factor * (Re A_c + alpha Re B_c) (B may be null).
__global__ void k_hg_finish(const double2* __restrict__ A, const double2* __restrict__ B, double alpha, double factor,
                            int ncomp, size_t n, double* __restrict__ out) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        for (int c = 0; c < ncomp; ++c) {
            double v = A[(size_t)c * n + p].x;
            if (B) v = v + alpha * B[(size_t)c * n + p].x;
            out[(size_t)c * n + p] = v * factor;
        }
    }
}

// The real root the reference takes of QX + QY a + QZ a^2 + QW a^3 = 0 (Bastrpp.F90:951-973):
// depressed cubic, Cardano with real cube roots when the discriminant is >= 0, else the
// trigonometric form.
inline double hitgen_cubic_root(double QX, double QY, double QZ, double QW) {
    const double QP = QY / QW - (1.0 / 3.0) * (QZ / QW) * (QZ / QW);
    const double QQ = 2.0 / 27.0 * (QZ / QW) * (QZ / QW) * (QZ / QW) - (1.0 / 3.0) * (QZ * QY) / (QW * QW) + QX / QW;
    const double QDELTA = (QQ / 2.0) * (QQ / 2.0) + (QP / 3.0) * (QP / 3.0) * (QP / 3.0);
    if (QDELTA >= 0.0) {
        const double t1 = -QQ / 2.0 + std::sqrt(QDELTA), t2 = -QQ / 2.0 - std::sqrt(QDELTA);
        return std::copysign(std::cbrt(std::fabs(t1)), t1) + std::copysign(std::cbrt(std::fabs(t2)), t2) -
               QZ / (3.0 * QW);
    }
    return 2.0 * std::sqrt(-QP / 3.0) * std::cos((1.0 / 3.0) * std::acos(3.0 * QQ / (2.0 * QP) * std::sqrt(-3.0 / QP))) -
           QZ / (3.0 * QW);
}

}  // namespace bastr
