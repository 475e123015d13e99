// Building blocks of a slab-decomposed 3D transform over several GPUs (the reference's
// FFTW-MPI decomposition, fftwlink.F90:63-77, with the transforms of fftwlink.F90:324-368), on
// caller-owned device arrays:
//
//   bastr_fft_lines  in-place complex-to-complex transforms of every line along one axis of a
//                    complex FP64 array [nz][ny][nx] (x fastest), e^{-ikx} forward / e^{+ikx}
//                    backward, times a scale (the full-grid axis kernel of fullfft.cu)
//   bastr_slab_pack  out[q][zl][yl][x] = in[zl][q*nyl + yl][x]: a z-slab [nzl][ny][nx] cut into
//                    the nparts blocks the all-to-all sends, rank q's block contiguous
//   bastr_slab_unpack  the inverse: in[zl][q*nyl + yl][x] = out[q][zl][yl][x]
//
// A forward transform of the grid held as z-slabs (rank r: planes r*nzl .. r*nzl+nzl-1) is then
// x and y lines on each slab, pack, one all-to-all of equal blocks (rank r receives
// [q][zl][yl][x] = [z][yl][x] for its y range: a y-slab), z lines on the y-slab.  The result
// stays y-slab distributed (the reference's transposed layout); the backward transform runs the
// same steps in reverse.  The communication is the caller's (NCCL all_to_all in
// bastr_b200/slabfft.py): every block crosses NVLink once into the receiver's own memory.
#pragma once
#include <map>
#include <mutex>
#include "fullfft.cu"

namespace bastr {

// out[q][zl][yl][x] = in[zl][q*nyl + yl][x] (pack) or the inverse (unpack), x fastest.
template <bool PACK>
__global__ void k_slab_move(const double2* __restrict__ in, double2* __restrict__ out, int nx, int ny, int nzl,
                            int nparts) {
    const int nyl = ny / nparts;
    const size_t total = (size_t)nzl * ny * nx;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        // i enumerates the packed layout [q][zl][yl][x]
        const int x = (int)(i % nx);
        const size_t r = i / nx;
        const int yl = (int)(r % nyl);
        const size_t r2 = r / nyl;
        const int zl = (int)(r2 % nzl), q = (int)(r2 / nzl);
        const size_t s = ((size_t)zl * ny + (size_t)q * nyl + yl) * nx + x;   // slab layout [zl][y][x]
        if (PACK) out[i] = in[s];
        else out[s] = in[i];
    }
}

// Device twiddle table w^m = exp(-2 pi i m/n), m < n, per (device, n): made on first use and
// kept until the process exits.
inline cudaError_t lines_twiddles(int n, const double2** out) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, double2*> tabs;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    auto it = tabs.find({dev, n});
    if (it == tabs.end()) {
        std::vector<double2> t64;
        std::vector<float2> t32;
        host_twiddles(n, t64, t32);
        double2* d = nullptr;
        e = cudaMalloc(&d, n * sizeof(double2));
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, t64.data(), n * sizeof(double2), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(d);
            return e;
        }
        it = tabs.emplace(std::make_pair(dev, n), d).first;
    }
    *out = it->second;
    return cudaSuccess;
}

template <bool INV>
cudaError_t lines_launch(double2* A, const int ns[3], int axis, double scale, const double2* tw, cudaStream_t st) {
    const long long total = (long long)ns[0] * ns[1] * ns[2];
    const int N = ns[axis];
    const int nlines = (int)(total / N);
    const long long S = axis == 0 ? 1 : axis == 1 ? ns[0] : (long long)ns[0] * ns[1];
    const long long R = axis == 1 ? (long long)ns[0] * ns[1] : ns[0];
    SIZE_CASES(N, {
        using P = FullLine<NN>;
        auto k = k_full_axis<NN, INV>;
        int nb = 1;
        cudaError_t e = prep(k, P::SMEM, P::NT, &nb);
        if (e != cudaSuccess) return e;
        int dev = 0;
        cudaGetDevice(&dev);
        const int sms = (dev >= 0 && dev < 64 && g_num_sms[dev] > 0) ? g_num_sms[dev] : 148;
        const int grid = std::max(1, std::min(cdiv(nlines, P::G), nb * sms));
        k<<<grid, P::NT, P::SMEM, st>>>(A, ns[0], S, R, nlines, scale, tw);
    });
    return cudaGetLastError();
}

inline bool lines_extent(int n) { return n >= 16 && n <= 2048 && (n & (n - 1)) == 0; }

}  // namespace bastr

extern "C" {

int bastr_fft_lines(double* d_a, int32_t nx, int32_t ny, int32_t nz, int32_t axis, int32_t dir, double scale,
                    void* stream) {
    using namespace bastr;
    if (!d_a || axis < 0 || axis > 2 || (dir != 1 && dir != -1) || nx < 1 || ny < 1 || nz < 1)
        return BASTR_E_INVALID;
    const int ns[3] = {nx, ny, nz};
    if (!lines_extent(ns[axis])) return BASTR_E_UNSUPPORTED;   // power-of-two lines of 16..2048 points
    if ((long long)nx * ny * nz / ns[axis] > (1LL << 31) - 1) return BASTR_E_UNSUPPORTED;
    const double2* tw = nullptr;
    if (lines_twiddles(ns[axis], &tw) != cudaSuccess) return BASTR_E_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const cudaError_t e = dir < 0 ? lines_launch<false>((double2*)d_a, ns, axis, scale, tw, st)
                                  : lines_launch<true>((double2*)d_a, ns, axis, scale, tw, st);
    return e == cudaSuccess ? BASTR_OK : BASTR_E_CUDA;
}

static int slab_move(bool pack, const double* d_in, double* d_out, int32_t nx, int32_t ny, int32_t nzl,
                     int32_t nparts, void* stream) {
    using namespace bastr;
    if (!d_in || !d_out || d_in == d_out || nx < 1 || ny < 1 || nzl < 1 || nparts < 1 || ny % nparts)
        return BASTR_E_INVALID;
    const size_t total = (size_t)nzl * ny * nx;
    const int grid = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    if (pack)
        k_slab_move<true><<<grid, 256, 0, (cudaStream_t)stream>>>((const double2*)d_in, (double2*)d_out, nx, ny,
                                                                   nzl, nparts);
    else
        k_slab_move<false><<<grid, 256, 0, (cudaStream_t)stream>>>((const double2*)d_in, (double2*)d_out, nx, ny,
                                                                    nzl, nparts);
    return cudaGetLastError() == cudaSuccess ? BASTR_OK : BASTR_E_CUDA;
}

int bastr_slab_pack(const double* d_slab, double* d_blocks, int32_t nx, int32_t ny, int32_t nzl, int32_t nparts,
                    void* stream) {
    return slab_move(true, d_slab, d_blocks, nx, ny, nzl, nparts, stream);
}

int bastr_slab_unpack(const double* d_blocks, double* d_slab, int32_t nx, int32_t ny, int32_t nzl, int32_t nparts,
                      void* stream) {
    return slab_move(false, d_blocks, d_slab, nx, ny, nzl, nparts, stream);
}

}  // extern "C"
