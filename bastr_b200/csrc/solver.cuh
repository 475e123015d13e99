// Geometry, layouts and launch helpers shared by the 2D/3D pass kernels.
//
// Spectral layout ("truncated half spectrum").  A real field has a Hermitian spectrum, so
// only kx >= 0 is stored.  The spherical 2/3 rule of the reference (tool.F90:175-217) zeroes
// every mode with |k| >= K = floor(ia/3); the state and every right-hand side therefore live
// on kx in [0,K), ky and kz in (-K,K).  Those are the only modes kept in HBM:
//
//   S[kx][kyi][c]          2D, kyi in [0,KY), KY = 2K-1, c = velocity component (interleaved)
//   S[c][kx][kyi][kzi]     3D, kzi in [0,KZ), KZ = 2K-1, component planes ps elements apart
//
// with index i < K meaning wavenumber i and i >= K meaning i - (2K-1) (negative side).
// Modes outside this set are exactly zero in the reference's arithmetic up to round-off.
#pragma once
#include "fft_engine.cuh"

namespace bastr {

// ---------------------------------------------------------------------------------------------
// Index-checking build (-DBASTR_CHECKED): the library's own memory checker.  A handle registers
// every device buffer it allocates in a CheckTable in device memory (Geo::chk); the checked
// accesses (the passes' staging copies and output stores, the stage epilogue's state reads and
// writes, the spectra and forcing gathers) verify that their bytes lie inside one registered
// buffer.  An access that does not sets ERR_INDEX in the handle's error word and goes to a
// scratch line instead, so the kernel runs on and the batch reports BASTR_E_CUDA.  In the normal
// build the checks compile to nothing and Geo::chk is null.
// ---------------------------------------------------------------------------------------------
constexpr int kCheckRanges = 64;
struct CheckTable {
    int n;
    unsigned long long lo[kCheckRanges], hi[kCheckRanges];   // [lo, hi) byte ranges
};
constexpr unsigned int ERR_INDEX = 2u;   // error-word bit (bit 1 is a TMA wait that gave up)

struct Geo {
    int nx, ny, nz;     // grid (nz == 1 in 2D)
    int d;              // 2 or 3
    int K;              // dealias cutoff floor(nx/3); kept kx in [0,K)
    int KY, KZ;         // truncated counts along y and z: 2K-1 (KZ == 1 in 2D)
    int lproject;       // dilatational projection on the right-hand side
    long long ps;       // 3D: stride between the component planes of a spectral field (elements)
    double nu, dt;
    double inv_n;       // 1 / (nx*ny*nz)
    // Stop word of a batch of steps (null outside bastr_step batches): the spectra kernel of a
    // step whose Es+Ed is NaN stores that step's slot + 1 there (solution.F90:69-81, `stop '"E" is
    // a NaN'`), and every kernel launched after it in the batch returns without touching data, so
    // the state stays the one that produced the NaN.
    unsigned int* halt;
    // Error word of the handle (never null in a handle's launches): kernels record failures
    // there (e.g. a TMA completion wait that gave up), and the host reports them after the batch.
    unsigned int* err;
    const CheckTable* chk;   // the handle's buffers (index-checking build), else null
};

#ifdef BASTR_CHECKED
static __device__ __align__(16) unsigned char g_check_scratch[64];
// p if [p, p + bytes) lies inside one buffer of the table (or there is no table), else records
// ERR_INDEX and returns the scratch line (at most 64 bytes are accessed through it).
template <typename P>
__device__ __forceinline__ P* checked_ptr(P* p, size_t bytes, const CheckTable* t, unsigned int* err) {
    if (!t) return p;
    const unsigned long long a = reinterpret_cast<unsigned long long>(p), b = a + bytes;
    for (int i = 0; i < t->n; ++i)
        if (a >= t->lo[i] && b <= t->hi[i]) return p;
    if (err) atomicOr(err, ERR_INDEX);
    return reinterpret_cast<P*>(g_check_scratch);
}
// the checked address of an access of `bytes` bytes at p; c: anything with .chk and .err
#define BASTR_CHK(p, bytes, c) ::bastr::checked_ptr((p), (size_t)(bytes), (c).chk, (c).err)
#else
#define BASTR_CHK(p, bytes, c) (p)
#endif
// element i of array a, checked
#define BASTR_AT(a, i, c) (*BASTR_CHK(&(a)[i], sizeof((a)[0]), c))

// True when an earlier kernel of the batch found a NaN energy; the same for every thread of the
// grid (the word is written by a kernel that completed before this one's pdl_wait returned).
__device__ __forceinline__ bool halted(const Geo& g) {
    return g.halt != nullptr && *reinterpret_cast<volatile const unsigned int*>(g.halt) != 0u;
}

// truncated index -> wavenumber
__device__ __forceinline__ int trunc_k(int i, int K, int KT) { return i < K ? i : i - KT; }
// position in a length-n transform -> truncated index, or -1 outside the kept set
__device__ __forceinline__ int pos_trunc(int p, int K, int KT, int n) {
    return p < K ? p : (p > n - K ? p - (n - KT) : -1);
}

template <typename A, typename B> __device__ __forceinline__ B cvt(A a);
template <> __device__ __forceinline__ float2 cvt<double2, float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __device__ __forceinline__ double2 cvt<float2, double2>(float2 a) { return make_double2(a.x, a.y); }
template <> __device__ __forceinline__ double2 cvt<double2, double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 cvt<float2, float2>(float2 a) { return a; }

__host__ __device__ constexpr int pow2_floor(int n) {
    int p = 1;
    while (p * 2 <= n) p *= 2;
    return p;
}

// Fixed-order block reduction of NV doubles (sum) into every thread's v[]; the tree shape
// depends only on the block size, so results are bitwise reproducible run to run.  Blocks of
// whole warps reduce within each warp by butterfly shuffles (lanes l and l^m add the same two
// values, so every lane holds the same bits), then the warps' sums the same way in warp 0: two
// barriers instead of log2(NT).  Other block sizes use a shared-memory tree, their tail folded
// onto the leading power of two first.
template <int NV, int NT>
__device__ __forceinline__ void block_sum(double* v, double* scratch /* NV*NT doubles */) {
    const int t = threadIdx.x;
    if constexpr (NT % 32 == 0 && NT <= 1024) {
        constexpr int NW = NT / 32;
        const int lane = t & 31, w = t >> 5;
#pragma unroll
        for (int i = 0; i < NV; ++i)
#pragma unroll
            for (int m = 16; m > 0; m >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], m);
        if (lane == 0) {
#pragma unroll
            for (int i = 0; i < NV; ++i) scratch[i * NW + w] = v[i];
        }
        __syncthreads();
        if (w == 0) {
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                double x = lane < NW ? scratch[i * NW + lane] : 0.0;
#pragma unroll
                for (int m = 16; m > 0; m >>= 1) x += __shfl_xor_sync(0xffffffffu, x, m);
                v[i] = x;
            }
        }
        __syncthreads();   // every warp has read its partials: the totals go where they were
        if (w == 0 && lane == 0) {
#pragma unroll
            for (int i = 0; i < NV; ++i) scratch[i * NW] = v[i];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] = scratch[i * NW];
        __syncthreads();
    } else {
        constexpr int P2 = pow2_floor(NT);
#pragma unroll
        for (int i = 0; i < NV; ++i) scratch[i * NT + t] = v[i];
        __syncthreads();
        if constexpr (P2 != NT) {
            if (t >= P2) {
#pragma unroll
                for (int i = 0; i < NV; ++i) scratch[i * NT + t - P2] += scratch[i * NT + t];
            }
            __syncthreads();
        }
#pragma unroll
        for (int s = P2 / 2; s > 0; s >>= 1) {
            if (t < s) {
#pragma unroll
                for (int i = 0; i < NV; ++i) scratch[i * NT + t] += scratch[i * NT + t + s];
            }
            __syncthreads();
        }
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] = scratch[i * NT];
        __syncthreads();
    }
}

template <int NT>
__device__ __forceinline__ double block_min(double v, double* scratch) {
    const int t = threadIdx.x;
    if constexpr (NT % 32 == 0 && NT <= 1024) {
        constexpr int NW = NT / 32;
        const int lane = t & 31, w = t >> 5;
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, m));
        if (lane == 0) scratch[w] = v;
        __syncthreads();
        double r = scratch[0];
#pragma unroll
        for (int i = 1; i < NW; ++i) r = fmin(r, scratch[i]);
        __syncthreads();
        return r;
    } else {
        constexpr int P2 = pow2_floor(NT);
        scratch[t] = v;
        __syncthreads();
        if constexpr (P2 != NT) {
            if (t >= P2) scratch[t - P2] = fmin(scratch[t - P2], scratch[t]);
            __syncthreads();
        }
#pragma unroll
        for (int s = P2 / 2; s > 0; s >>= 1) {
            if (t < s) scratch[t] = fmin(scratch[t], scratch[t + s]);
            __syncthreads();
        }
        double r = scratch[0];
        __syncthreads();
        return r;
    }
}

// Programmatic dependent launch: the kernels of a step are launched with
// cudaLaunchAttributeProgrammaticStreamSerialization, so a kernel's blocks are scheduled as the
// previous kernel's blocks exit, and each kernel waits here for the previous kernel to complete
// (and its writes to be visible) before it touches any data that kernel wrote or reads.  An
// explicit early trigger (griddepcontrol.launch_dependents) measured slower: the waiting blocks
// then hold SM resources the running kernel could use.  Without the launch attribute this is a
// no-op.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Completion ticket of a reduction whose per-block partials are finished by one block: every
// block calls this after writing its partials (thread 0 wrote them); it returns true in the one
// block that arrives last, which then sees all partials and must reset *done to 0 when it is
// through.  `flag` is one shared word.  No block waits for another.
__device__ __forceinline__ bool last_block_arrives(unsigned int* done, unsigned int* flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        *flag = atomicAdd(done, 1u) == gridDim.x - 1 ? 1u : 0u;
    }
    __syncthreads();
    const bool last = *flag != 0;
    if (last) __threadfence();
    return last;
}

// Epilogue modes of the forward pass that closes a right-hand side evaluation.
enum EpiMode : int {
    EPI_STORE = 0,   // state <- dealiased spectrum (set_state)
    EPI_RK1 = 1,     // k1; acc = k1; us = u0 + dt*k1/2
    EPI_RK2 = 2,     // k2; us = u0 - dt*acc + 2dt*k2; acc += 4 k2
    EPI_RK3 = 3,     // k3; u0 += dt*(acc + k3)/6
    EPI_CN_MID = 4,  // Crank-Nicolson sweep 1..5: w = 0.5*((u0 + dt*k) + u0)
    EPI_CN_LAST = 5, // sweep 6: u0 += dt*k
};

// Pointers a stage epilogue reads and writes (types per precision form).
template <typename T>
struct StageIO {
    double2* u0;         // state, always FP64
    cplx<T>* us;         // stage input of the next evaluation
    cplx<T>* acc;        // RK accumulator k1 + 4 k2
    double* energy_part; // per-block sum of w*|u0_new|^2 (RK3 / CN_LAST), or null
    const CheckTable* chk;   // Geo::chk and Geo::err, for the checked accesses
    unsigned int* err;
};

__device__ __forceinline__ double2 dscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// State values one mode's epilogue reads: the FP64 state a = u0, the stage input s (us; equal to
// a when the stage starts from u0) and the RK accumulator p.  Loading them for several modes
// before any store lets those loads overlap instead of paying one memory latency per mode.
template <typename T, int D> struct EpiIn {
    double2 a[D];
    cplx<T> s[D];
    cplx<T> p[D];
};

template <typename T, int D, int EPI>
__device__ __forceinline__ void epi_load(EpiIn<T, D>& in, size_t o, size_t cst, const StageIO<T>& io,
                                         bool from_u0) {
    if constexpr (EPI != EPI_STORE) {
#pragma unroll
        for (int c = 0; c < D; ++c) {
            in.a[c] = BASTR_AT(io.u0, o + c * cst, io);
            // RK2 re-forms its stage input u0 + dt/2 k1 from a and p instead of reading it
            if (!from_u0 && EPI != EPI_RK2) in.s[c] = BASTR_AT(io.us, o + c * cst, io);
            if constexpr (EPI == EPI_RK2 || EPI == EPI_RK3) in.p[c] = BASTR_AT(io.acc, o + c * cst, io);
        }
    }
}

// Spectral epilogue of one mode (compute_ut, solution.F90:841-861 / 903-926, and the time
// integrators, solution.F90:172-301).  v[c] holds the dealiased, 1/N-normalised transform of
// the advective product; k[c] the wavenumbers, m2 = |k|^2; in the mode's state values
// (epi_load); o the state offset of component 0; cst the stride between components; w the
// Hermitian weight of the mode (1 on kx = 0, else 2); en accumulates w*|u0_new|^2.
// With NEXT, the new stage input that RK1, RK2 and CN_MID store to io.us is also returned in
// next[c] (the value stored, in T), for a pass that transforms it on the spot; RK1 then need
// not store it at all (STORE_US = false), since RK2 re-forms it.
template <typename T, int D, int EPI, bool NEXT = false, bool STORE_US = true>
__device__ __forceinline__ void rk_apply(double2* v, const double* k, double m2, const EpiIn<T, D>& in,
                                         size_t o, size_t cst, const StageIO<T>& io, bool from_u0,
                                         const Geo& g, double w, double& en, cplx<T>* next = nullptr) {
    if constexpr (EPI == EPI_STORE) {
#pragma unroll
        for (int c = 0; c < D; ++c) BASTR_AT(io.u0, o + c * cst, io) = v[c];
        return;
    } else {
        const double nu = g.nu, dt = g.dt;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            // + nu * FFT(lap u) with lap u^ = -|k|^2 u^ of the stage input (RK2: u0 + dt/2 k1,
            // the value RK1 formed, exactly so in FP64)
            double2 s;
            if constexpr (EPI == EPI_RK2) {
                const double2 p = cvt<cplx<T>, double2>(in.p[c]);
                s = make_double2(in.a[c].x + g.dt * p.x / 2.0, in.a[c].y + g.dt * p.y / 2.0);
            } else {
                s = from_u0 ? in.a[c] : cvt<cplx<T>, double2>(in.s[c]);
            }
            v[c].x += nu * (-(s.x * m2));
            v[c].y += nu * (-(s.y * m2));
        }
        if (g.lproject) {   // projection2D/3D, tool.F90:219-270
            if (m2 > 0.25) {
                // u_d = (k/|k|) (k/|k|) . v, with one reciprocal per mode
                const double ik = 1.0 / sqrt(m2);
                double kh[D];
#pragma unroll
                for (int c = 0; c < D; ++c) kh[c] = k[c] * ik;
                double2 ud = make_double2(0, 0);
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    ud.x += v[c].x * kh[c];
                    ud.y += v[c].y * kh[c];
                }
#pragma unroll
                for (int c = 0; c < D; ++c) v[c] = make_double2(ud.x * kh[c], ud.y * kh[c]);
            } else {
#pragma unroll
                for (int c = 0; c < D; ++c) v[c] = make_double2(0, 0);
            }
        }
        const double dt2 = 2.0 * dt;
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const double2 a = in.a[c];
            if constexpr (EPI == EPI_RK1) {
                BASTR_AT(io.acc, o + c * cst, io) = cvt<double2, cplx<T>>(v[c]);
                const cplx<T> u = cvt<double2, cplx<T>>(make_double2(a.x + dt * v[c].x / 2.0, a.y + dt * v[c].y / 2.0));
                if constexpr (STORE_US) BASTR_AT(io.us, o + c * cst, io) = u;
                if constexpr (NEXT) next[c] = u;
            } else if constexpr (EPI == EPI_RK2) {
                const double2 p = cvt<cplx<T>, double2>(in.p[c]);
                const cplx<T> u = cvt<double2, cplx<T>>(
                    make_double2(a.x - dt * p.x + dt2 * v[c].x, a.y - dt * p.y + dt2 * v[c].y));
                BASTR_AT(io.us, o + c * cst, io) = u;
                if constexpr (NEXT) next[c] = u;
                BASTR_AT(io.acc, o + c * cst, io) = cvt<double2, cplx<T>>(make_double2(p.x + 4.0 * v[c].x, p.y + 4.0 * v[c].y));
            } else if constexpr (EPI == EPI_RK3) {
                const double2 p = cvt<cplx<T>, double2>(in.p[c]);
                const double2 n = make_double2(a.x + dt * (p.x + v[c].x) / 6.0, a.y + dt * (p.y + v[c].y) / 6.0);
                BASTR_AT(io.u0, o + c * cst, io) = n;
                en += w * (n.x * n.x + n.y * n.y);
            } else if constexpr (EPI == EPI_CN_MID) {
                const cplx<T> u = cvt<double2, cplx<T>>(
                    make_double2(0.5 * ((a.x + dt * v[c].x) + a.x), 0.5 * ((a.y + dt * v[c].y) + a.y)));
                BASTR_AT(io.us, o + c * cst, io) = u;
                if constexpr (NEXT) next[c] = u;
            } else if constexpr (EPI == EPI_CN_LAST) {
                const double2 n = make_double2(a.x + dt * v[c].x, a.y + dt * v[c].y);
                BASTR_AT(io.u0, o + c * cst, io) = n;
                en += w * (n.x * n.x + n.y * n.y);
            }
        }
    }
}

// Modes per thread whose state is fetched together before the epilogue math: more overlap
// against more live registers (measured best: FP32 2D 4, FP64 2D 2, FP32 3D 2, FP64 3D 4).
template <typename T, int D> struct EpiChunk {
    static constexpr int v = D == 2 ? (sizeof(T) == 4 ? 4 : 2) : (sizeof(T) == 4 ? 2 : 4);
};

// Asynchronous 16-byte global -> shared copies (cp.async, bypassing L1), used to stage whole
// contiguous lines one iteration ahead of the transform that consumes them.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPEND> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND) : "memory");
}

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}

// Copies `bytes` (a multiple of 8, both ends 8-byte aligned) from global to shared memory with
// all threads of the block, in 16-byte chunks when both ends and the length allow it and in
// 8-byte chunks otherwise; returns without waiting.
// g: the handle's geometry (its check table in the index-checking build).
__device__ __forceinline__ void stage_line(void* smem_dst, const void* gmem_src, int bytes, const Geo& g) {
    char* d = static_cast<char*>(smem_dst);
    const char* s = static_cast<const char*>(gmem_src);
    if ((((unsigned long long)d | (unsigned long long)s | (unsigned long long)bytes) & 15ull) == 0) {
        const int n16 = bytes >> 4;
        for (int i = threadIdx.x; i < n16; i += blockDim.x) cp_async16(d + 16 * i, BASTR_CHK(s + 16 * i, 16, g));
    } else {
        const int n8 = bytes >> 3;
        for (int i = threadIdx.x; i < n8; i += blockDim.x) cp_async8(d + 8 * i, BASTR_CHK(s + 8 * i, 8, g));
    }
    (void)g;
}

}  // namespace bastr
