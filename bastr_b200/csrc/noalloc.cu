// Shell spectra of a caller-owned spectrum without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: a Fortran post-processing code whose GPU
// memory is owned by CUDA Fortran / OpenACC data regions, or a driver that runs under a
// memory-capped pool, can hold its spectrum on the device but cannot create a handle (which
// allocates the solver's buffers).  bastr_spectra_noalloc gives them the shell spectra of
// spectra_compute2D/3D (solution.F90:930-1108) on their own arrays.  Its only workspace, the
// per-shell partial sums, lives in the file-scope device array g_noalloc_shell below, of fixed
// size: every GPU that loads the library holds those 128 KiB until the process exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "../../include/bastr_gpu.h"
#include "solver.cuh"

namespace {

using namespace bastr;

constexpr int kNoallocMaxShells = BASTR_NOALLOC_MAX_SHELLS;
constexpr int kNoallocThreads = 256;
constexpr int kMaxDevices = 64;

// Per-shell partial sums (Es, Ed, k2Ed, kMEd) of one call.  In host code this name is only a
// host-side stand-in for the device symbol: its device address comes from
// cudaGetSymbolAddress (noalloc_scratch below) and is what the kernels receive.
static __device__ __align__(256) double g_noalloc_shell[kNoallocMaxShells * 4];

// The address is valid only in the CUDA context that resolved it: another context on the same
// device (one a driver-API or CUDA Fortran caller made current, or the primary context created
// anew after a cudaDeviceReset) has its own copy of the array.  So the cache is keyed on the
// context's unique id (cuCtxGetId, reached through cudaGetDriverEntryPoint so the library needs
// no link to libcuda), and an address is looked up again in a context not seen before.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

struct ScratchEntry {
    unsigned long long ctx_id;
    double* ptr;
};

std::mutex g_mu;
std::vector<ScratchEntry> g_scratch;
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
bool g_ctx_fns_tried = false;

// Id of the calling thread's current context, or 0 when there is none yet or the driver does
// not offer the query.  Called with g_mu held.
unsigned long long current_ctx_id() {
    if (!g_ctx_fns_tried) {
        g_ctx_fns_tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_id = reinterpret_cast<CtxGetIdFn>(f);
    }
    if (!g_ctx_current || !g_ctx_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    if (g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_noalloc_shell in the current context: looked up once per context (every
// call, when the context cannot be identified).  The lookup is not a stream operation, but the
// first call in a context should come before any stream capture.
cudaError_t noalloc_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    unsigned long long id = current_ctx_id();
    if (id != 0) {
        for (const ScratchEntry& s : g_scratch)
            if (s.ctx_id == id) {
                *out = s.ptr;
                return cudaSuccess;
            }
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_shell);   // also makes the device's primary context current
    if (e != cudaSuccess) return e;
    if (id == 0) id = current_ctx_id();
    if (id != 0) g_scratch.push_back({id, static_cast<double*>(p)});
    *out = static_cast<double*>(p);
    return cudaSuccess;
}

__device__ __forceinline__ long long isqrt_floor_na(long long v) {
    if (v <= 0) return 0;
    long long r = (long long)sqrt((double)v);
    while (r * r > v) --r;
    while ((r + 1) * (r + 1) <= v) ++r;
    return r;
}
__device__ __forceinline__ long long isqrt_ceil_na(long long v) {
    if (v <= 0) return 0;
    long long r = isqrt_floor_na(v);
    return r * r == v ? r : r + 1;
}

struct FullGrid {
    int nx, ny, nz, d;
};

// Wavenumber range of one axis of a full grid: [-(n/2-1), n/2] (Nyquist carries +n/2).
__device__ __forceinline__ bool in_axis(int k, int n) { return k > -(n / 2) && k <= n / 2; }
__device__ __forceinline__ int axis_index(int k, int n) { return k >= 0 ? k : k + n; }

template <int D>
__device__ __forceinline__ void mode_full(const double2* __restrict__ u1, const double2* __restrict__ u2,
                                          const double2* __restrict__ u3, const FullGrid& g, int kx, int ky,
                                          int kz, double acc[4]) {
    const long long m = (long long)kx * kx + (long long)ky * ky + (long long)kz * kz;
    if (m == 0) return;
    const double kk = sqrt((double)m);
    const double k1 = kx, k2 = ky, k3 = kz;
    const size_t o = ((size_t)axis_index(kz, g.nz) * g.ny + axis_index(ky, g.ny)) * g.nx + axis_index(kx, g.nx);
    const double2 a = u1[o], b = u2[o];
    double es, ed;
    if constexpr (D == 2) {
        const double usx = a.x * k2 / kk - b.x * k1 / kk, usy = a.y * k2 / kk - b.y * k1 / kk;
        const double udx = a.x * k1 / kk + b.x * k2 / kk, udy = a.y * k1 / kk + b.y * k2 / kk;
        es = (usx * usx + usy * usy) / 2;
        ed = (udx * udx + udy * udy) / 2;
    } else {
        const double2 c = u3[o];
        const double udx = a.x * k1 / kk + b.x * k2 / kk + c.x * k3 / kk;
        const double udy = a.y * k1 / kk + b.y * k2 / kk + c.y * k3 / kk;
        const double s1x = a.x - udx * k1 / kk, s1y = a.y - udy * k1 / kk;
        const double s2x = b.x - udx * k2 / kk, s2y = b.y - udy * k2 / kk;
        const double s3x = c.x - udx * k3 / kk, s3y = c.y - udy * k3 / kk;
        es = (s1x * s1x + s1y * s1y) / 2 + (s2x * s2x + s2y * s2y) / 2 + (s3x * s3x + s3y * s3y) / 2;
        ed = (udx * udx + udy * udy) / 2;
    }
    acc[0] += es;
    acc[1] += ed;
    acc[2] += ed * (kk * kk);
    acc[3] += ed / kk;
}

// One block per shell s: every full-grid mode with |k|^2 in [s^2-s+1, s^2+s] (nint(|k|) = s),
// partial sums written to scratch[s] (every slot in [0, nshell) is written, none is read first).
template <int D>
__global__ void __launch_bounds__(kNoallocThreads)
k_spectra_full(const double2* __restrict__ u1, const double2* __restrict__ u2, const double2* __restrict__ u3,
               FullGrid g, double* __restrict__ scratch) {
    __shared__ double red[4 * kNoallocThreads];
    const int s = blockIdx.x;
    const long long lo = s == 0 ? 0 : (long long)s * s - s + 1;
    const long long hi = s == 0 ? 0 : (long long)s * s + s;
    double acc[4] = {0, 0, 0, 0};
    const int kxm = s < g.nx / 2 ? s : g.nx / 2;
    const int nkx = 2 * kxm + 1;
    if constexpr (D == 2) {
        for (int e = threadIdx.x; e < nkx; e += kNoallocThreads) {
            const int kx = e - kxm;
            if (!in_axis(kx, g.nx)) continue;
            const long long rlo = lo - (long long)kx * kx, rhi = hi - (long long)kx * kx;
            if (rhi < 0) continue;
            const int a = (int)isqrt_ceil_na(rlo), b = (int)isqrt_floor_na(rhi);
            for (int t = a; t <= b; ++t) {
                if (in_axis(t, g.ny)) mode_full<2>(u1, u2, u3, g, kx, t, 0, acc);
                if (t != 0 && in_axis(-t, g.ny)) mode_full<2>(u1, u2, u3, g, kx, -t, 0, acc);
            }
        }
    } else {
        const int kym = s < g.ny / 2 ? s : g.ny / 2;
        const int nky = 2 * kym + 1;
        for (int e = threadIdx.x; e < nkx * nky; e += kNoallocThreads) {
            const int kx = e / nky - kxm, ky = e % nky - kym;
            if (!in_axis(kx, g.nx) || !in_axis(ky, g.ny)) continue;
            const long long rr = (long long)kx * kx + (long long)ky * ky;
            const long long rlo = lo - rr, rhi = hi - rr;
            if (rhi < 0) continue;
            const int a = (int)isqrt_ceil_na(rlo), b = (int)isqrt_floor_na(rhi);
            for (int t = a; t <= b; ++t) {
                if (in_axis(t, g.nz)) mode_full<3>(u1, u2, u3, g, kx, ky, t, acc);
                if (t != 0 && in_axis(-t, g.nz)) mode_full<3>(u1, u2, u3, g, kx, ky, -t, acc);
            }
        }
    }
    block_sum<4, kNoallocThreads>(acc, red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) scratch[(size_t)s * 4 + i] = acc[i];
    }
}

// Totals over all shells in fixed order and the copy of shells 0..allkmax.
__global__ void __launch_bounds__(kNoallocThreads)
k_spectra_full_final(const double* __restrict__ scratch, int nshell, int allkmax, double* __restrict__ es,
                     double* __restrict__ ed, double* __restrict__ totals) {
    __shared__ double red[4 * kNoallocThreads];
    double acc[4] = {0, 0, 0, 0};
    for (int s = threadIdx.x; s < nshell; s += kNoallocThreads) {
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i] += scratch[(size_t)s * 4 + i];
    }
    block_sum<4, kNoallocThreads>(acc, red);
    if (threadIdx.x == 0 && totals) {
#pragma unroll
        for (int i = 0; i < 4; ++i) totals[i] = acc[i];
    }
    for (int s = threadIdx.x; s <= allkmax; s += kNoallocThreads) {
        es[s] = s < nshell ? scratch[(size_t)s * 4 + 0] : 0.0;
        ed[s] = s < nshell ? scratch[(size_t)s * 4 + 1] : 0.0;
    }
}

bool pow2_extent(int n) { return n >= 2 && (n & (n - 1)) == 0; }

}  // namespace

extern "C" BASTR_API int bastr_spectra_noalloc(int32_t ia, int32_t ja, int32_t ka, int32_t kmax,
                                              const double* d_u1spe, const double* d_u2spe,
                                              const double* d_u3spe, double* d_Es, double* d_Ed,
                                              double* d_totals, void* stream) {
    const int d = ka == 0 ? 2 : 3;
    if (!pow2_extent(ia) || !pow2_extent(ja) || (d == 3 && !pow2_extent(ka))) return BASTR_E_INVALID;
    if (!d_u1spe || !d_u2spe || (d == 3 && !d_u3spe) || !d_Es || !d_Ed) return BASTR_E_INVALID;
    const int nz = d == 3 ? ka : 1;
    // every mode of the grid lies in a shell <= nint(|k|max): the totals cover them all
    const double kmax_grid = std::sqrt((double)(ia / 2) * (ia / 2) + (double)(ja / 2) * (ja / 2) +
                                       (d == 3 ? (double)(nz / 2) * (nz / 2) : 0.0));
    const int nshell = (int)std::floor(kmax_grid + 0.5) + 1;
    if (nshell > kNoallocMaxShells) return BASTR_E_TOO_LARGE;   // the fixed workspace holds fewer shells
    int allkmax = std::min(ia / 3, (int)kmax);
    if (allkmax < 0) allkmax = 0;
    double* scratch = nullptr;
    if (noalloc_scratch(&scratch) != cudaSuccess) return BASTR_E_CUDA;
    const FullGrid g{ia, ja, nz, d};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double2* u1 = reinterpret_cast<const double2*>(d_u1spe);
    const double2* u2 = reinterpret_cast<const double2*>(d_u2spe);
    const double2* u3 = reinterpret_cast<const double2*>(d == 3 ? d_u3spe : d_u1spe);
    // launch statuses are taken from the launches themselves, so that an error the caller left
    // pending in the runtime's last-error state is neither cleared nor blamed on this call
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(kNoallocThreads);
    cfg.stream = st;
    cfg.gridDim = dim3(nshell);
    cudaError_t e = d == 2 ? cudaLaunchKernelEx(&cfg, k_spectra_full<2>, u1, u2, u3, g, scratch)
                           : cudaLaunchKernelEx(&cfg, k_spectra_full<3>, u1, u2, u3, g, scratch);
    if (e != cudaSuccess) return BASTR_E_CUDA;
    cfg.gridDim = dim3(1);
    e = cudaLaunchKernelEx(&cfg, k_spectra_full_final, (const double*)scratch, nshell, allkmax, d_Es, d_Ed, d_totals);
    return e == cudaSuccess ? BASTR_OK : BASTR_E_CUDA;
}
