// Full-grid complex-to-complex transforms in FP64 (fft2d/fft3d/ifft2d/ifft3d,
// fftwlink.F90:324-368): forward e^{-ikx} scaled by 1/N, backward e^{+ikx} unscaled, in place on
// a complex grid [nz][ny][nx] (x fastest, the Fortran order of the reference's arrays).
//
// One pass per axis.  A block owns G lines of one axis; the G lines x0..x0+G-1 of the y or z
// axis are neighbours in x, so the block moves its G x N tile between global and shared
// memory in runs of G consecutive elements (x lines are contiguous and move as whole lines).
// Each line is then transformed by a register Stockham transform (regfft.cuh) of one group of
// N/EPT threads.  The scale 1/N is folded into the last axis of a forward transform.
#pragma once
#include "regfft.cuh"
#include "solver.cuh"

namespace bastr {

template <int N> struct FullLine {
    static constexpr int EPT = N < 8 ? N : 8;
    static constexpr int NTR = N / EPT;
    // lines per block: a tile of at most 64 KB and at least 128 threads
    static constexpr int GT = 65536 / (N * 16) < 1 ? 1 : 65536 / (N * 16);
    static constexpr int GMIN = NTR >= 128 ? 1 : 128 / NTR;
    static constexpr int G = GT > GMIN ? GT : GMIN;
    static constexpr int NT = G * NTR;
    template <bool INV> using FFT = RegFFT<double, N, EPT, 1, INV>;
    static constexpr size_t TILE = (size_t)G * N * sizeof(double2);
    static constexpr size_t SMEM = TILE + (size_t)G * FFT<true>::SMEM_ELEMS * sizeof(double2);
};

// Axis with element stride S (1, nx or nx*ny): line L has x = L % nx, r = L / nx and starts at
// x + r*R (R = nx*ny for the y axis, nx for the z axis); for the x axis (S = 1) line L starts at
// L*nx.  nlines lines; scale multiplies the result.
template <int N, bool INV>
__global__ void __launch_bounds__(FullLine<N>::NT)
k_full_axis(double2* __restrict__ A, int nx, long long S, long long R, int nlines, double scale,
            const double2* __restrict__ tw) {
    using P = FullLine<N>;
    using FFT = typename P::template FFT<INV>;
    constexpr int G = P::G, NT = P::NT, EPT = P::EPT;
    extern __shared__ __align__(16) unsigned char smraw[];
    double2* tile = reinterpret_cast<double2*>(smraw);                         // [g][N]
    double2* xch = reinterpret_cast<double2*>(smraw + P::TILE);
    pdl_wait();
    const int gi = threadIdx.x / P::NTR, t = threadIdx.x % P::NTR;
    double2* sm = xch + gi * FFT::SMEM_ELEMS;
    const int nitems = (nlines + G - 1) / G;
    auto base = [&](int L) -> long long {
        return S == 1 ? (long long)L * nx : (long long)(L % nx) + (long long)(L / nx) * R;
    };
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int L0 = item * G;
        // tile in: x lines whole; y/z lines element by element, the G lines side by side
        for (int i = threadIdx.x; i < G * N; i += NT) {
            int g, j;
            if (S == 1) { g = i / N; j = i - g * N; }
            else { j = i / G; g = i - j * G; }
            if (L0 + g < nlines) tile[g * N + j] = A[base(L0 + g) + (long long)j * S];
        }
        __syncthreads();
        double2 v[EPT];
#pragma unroll
        for (int e = 0; e < EPT; ++e) v[e] = tile[gi * N + FFT::in_pos(t, e)];
        FFT::run(v, sm, tw, t);
#pragma unroll
        for (int e = 0; e < EPT; ++e) {
            double2 r = v[e];
            tile[gi * N + FFT::out_pos(t, e)] = make_double2(r.x * scale, r.y * scale);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < G * N; i += NT) {
            int g, j;
            if (S == 1) { g = i / N; j = i - g * N; }
            else { j = i / G; g = i - j * G; }
            if (L0 + g < nlines) A[base(L0 + g) + (long long)j * S] = tile[g * N + j];
        }
        __syncthreads();
    }
}

}  // namespace bastr
