// Register-resident Stockham FFT for sm_100a.
//
// A group of NTR = N/EPT threads transforms UPT units (independent length-N complex sequences
// that share one index map) of which every thread holds EPT elements per unit in registers.
// Stage s of radix R works on butterflies b = t + q*NTR (q < EPT/R) reading x[b + j*N/R]:
// twiddle, DFT-R in registers, and the outputs land at (b-k)*R + k + j*P (k = b mod P, P the
// product of the earlier radices), the Stockham autosort order.  Only the hand-over between two
// stages goes through shared memory; the first stage takes its inputs from the caller's
// registers (filled straight from global memory by `in_pos`) and the last stage leaves its
// outputs in registers at `out_pos`, so a pass needs no shared-memory copy of its input or
// output.  The inverse plan uses radix EPT first and the remainder last; the forward plan is
// its mirror, so an inverse transform followed by a forward one of the same shape hands its
// registers over directly (out_pos of the first == in_pos of the second).
//
// Twiddles w^m = exp(-2 pi i m/N) come from a table generated on the host in extended
// precision and rounded once to T; per butterfly only w^1, w^2, w^4, w^8 are loaded and the
// other powers are formed by at most two multiplications, and they are shared by all units.
#pragma once
#include "fft_engine.cuh"

namespace bastr {

__host__ __device__ constexpr int ilog2c(int n) {
    int r = 0;
    while ((1 << r) < n) ++r;
    return r;
}

template <int N, int EPT> struct RPlan {
    static constexpr int n = ilog2c(N), e = ilog2c(EPT);
    static constexpr int NFULL = n / e, REM = n % e;
    static constexpr int NS = NFULL + (REM ? 1 : 0);
    static constexpr int inv_radix(int s) { return s < NFULL ? EPT : (1 << REM); }
    static constexpr int fwd_radix(int s) { return inv_radix(NS - 1 - s); }
    static constexpr int radix(bool inv, int s) { return inv ? inv_radix(s) : fwd_radix(s); }
    // product of the radices before stage s
    static constexpr int sub(bool inv, int s) { return s == 0 ? 1 : sub(inv, s - 1) * radix(inv, s - 1); }
};

template <typename T, int N, int EPT, int UPT, bool INV>
struct RegFFT {
    using PL = RPlan<N, EPT>;
    static constexpr int NTR = N / EPT;
    static constexpr int NS = PL::NS;
    static constexpr int R0 = PL::radix(INV, 0);
    static constexpr int RL = PL::radix(INV, NS - 1);
    static constexpr int US = padded_len(N);                // shared elements per unit
    static constexpr int SMEM_ELEMS = UPT * US;
    static_assert((N & (N - 1)) == 0 && N >= EPT, "power-of-two length");

    // position of register element e of thread t before the first stage / after the last
    __device__ static __forceinline__ int in_pos(int t, int e) {
        return t + (e / R0) * NTR + (e % R0) * (N / R0);
    }
    __device__ static __forceinline__ int out_pos(int t, int e) {
        return t + (e / RL) * NTR + (e % RL) * (N / RL);
    }

    // True when register element e lies, for every thread, in the open band (lo, N - lo) of
    // positions before the first stage (in_pos) / after the last stage (out_pos): known at
    // compile time once the loops are unrolled, so a caller can leave such inputs at zero and
    // skip such outputs, and the compiler folds the arithmetic they would take.
    __host__ __device__ static constexpr bool in_band(int e, int lo) {
        const int b = (e / R0) * NTR + (e % R0) * (N / R0);
        return b >= lo && b + NTR - 1 <= N - lo;
    }
    __host__ __device__ static constexpr bool out_band(int e, int lo) {
        const int b = (e / RL) * NTR + (e % RL) * (N / RL);
        return b >= lo && b + NTR - 1 <= N - lo;
    }

    // Twiddles by stage, an alternative layout of the same values: for every stage s >= 1 the
    // base powers w^(j k S), j = 1, 2, 4, 8 (as many as the stage's radix uses), k = 0..PS-1,
    // j-major.  The threads of a warp take consecutive k, so they read consecutive elements;
    // in the linear table w^m they read with stride j*S, a multiple of the bank width for most
    // stages.  Same values, same arithmetic: results are bitwise those of the linear table.
    static constexpr int nbase(int R) { return R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4; }
    static constexpr int tws_off(int s) {
        return s <= 1 ? 0 : tws_off(s - 1) + PL::sub(INV, s - 1) * nbase(PL::radix(INV, s - 1));
    }
    static constexpr int TWS_ELEMS = NS > 1 ? tws_off(NS) : 0;

    // Block-wide copy of the linear table `lin` (w^m, m < N/2) into the by-stage layout at dst
    // (TWS_ELEMS elements); the caller's next __syncthreads() publishes it.
    template <int S = 1>
    __device__ static __forceinline__ void fill_stage_twiddles(cplx<T>* dst, const cplx<T>* __restrict__ lin) {
        if constexpr (S < NS) {
            constexpr int R = PL::radix(INV, S), PS = PL::sub(INV, S), NB = nbase(R), TS = N / (PS * R);
            for (int i = threadIdx.x; i < NB * PS; i += blockDim.x) {
                const int jb = i / PS, k = i - jb * PS;
                dst[tws_off(S) + i] = lin[(1 << jb) * k * TS];
            }
            fill_stage_twiddles<S + 1>(dst, lin);
        }
    }

    template <int R, int PS, int S_, bool STAGED>
    __device__ static __forceinline__ void compute(cplx<T>* v, const cplx<T>* __restrict__ tw, int t) {
#pragma unroll
        for (int q = 0; q < EPT / R; ++q) {
            const int b = t + q * NTR;
            if constexpr (PS > 1) {
                constexpr int S = N / (PS * R);
                const int k = b & (PS - 1);
                // w[j] = w^(j k S): read for j = 1, 2, 4, 8, products for the rest
                auto base = [&](int jb) -> cplx<T> {
                    if constexpr (STAGED) return tw[tws_off(S_) + jb * PS + k];
                    else return tw[(1 << jb) * k * S];
                };
                cplx<T> w[R];
                w[1] = base(0);
                if constexpr (R >= 4) {
                    w[2] = base(1);
                    w[3] = cmul<T>(w[2], w[1]);
                }
                if constexpr (R >= 8) {
                    w[4] = base(2);
                    w[5] = cmul<T>(w[4], w[1]);
                    w[6] = cmul<T>(w[4], w[2]);
                    w[7] = cmul<T>(w[4], w[3]);
                }
                if constexpr (R >= 16) {
                    w[8] = base(3);
#pragma unroll
                    for (int j = 9; j < 16; ++j) w[j] = cmul<T>(w[8], w[j - 8]);
                }
#pragma unroll
                for (int j = 1; j < R; ++j) {
                    const cplx<T> ww = INV ? cconj<T>(w[j]) : w[j];
#pragma unroll
                    for (int u = 0; u < UPT; ++u) v[u * EPT + q * R + j] = cmul<T>(v[u * EPT + q * R + j], ww);
                }
            }
#pragma unroll
            for (int u = 0; u < UPT; ++u) dftR<T, INV, R>(v + u * EPT + q * R);
        }
    }

    // Shared-memory position of element a of a unit during the exchanges.  The padded map pidx
    // leaves the warps of the radix-8 FP32 plans and the radix-4 and -8 FP64 plans with 1.2-1.3x the
    // ideal number of shared-memory wavefronts (bank conflicts of the stride-PS writes); for
    // those plans an XOR of the low bank bits with higher bits spreads every exchange over all
    // banks.  Each swizzle changes bit i only by bits above i, so it is a bijection within every
    // aligned block of 16 (8) elements and stays inside the unit.  For FP32 lines longer than
    // 512 the conflicts are fewer (1.1x) and the extra index arithmetic measured slower.
    __device__ static __forceinline__ int sidx(int a) {
        if constexpr (sizeof(T) == 4 && EPT == 8 && N <= 512) return a ^ (((a >> 3) ^ (a >> 5)) & 15);
        else if constexpr (sizeof(T) == 8 && EPT == 4) return a ^ (((a >> 2) ^ (a >> 5)) & 7);
        else if constexpr (sizeof(T) == 8 && EPT == 8) return a ^ (((a >> 3) ^ (a >> 4)) & 7);
        else return pidx(a);
    }

    template <int R, int PS, int R2>
    __device__ static __forceinline__ void exchange(cplx<T>* v, cplx<T>* sm, int t) {
#pragma unroll
        for (int q = 0; q < EPT / R; ++q) {
            const int b = t + q * NTR;
            const int k = b & (PS - 1);
            const int base = (b - k) * R + k;
#pragma unroll
            for (int j = 0; j < R; ++j) {
#pragma unroll
                for (int u = 0; u < UPT; ++u) sm[u * US + sidx(base + j * PS)] = v[u * EPT + q * R + j];
            }
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < EPT / R2; ++q) {
#pragma unroll
            for (int j = 0; j < R2; ++j) {
                const int p = t + q * NTR + j * (N / R2);
#pragma unroll
                for (int u = 0; u < UPT; ++u) v[u * EPT + q * R2 + j] = sm[u * US + sidx(p)];
            }
        }
        __syncthreads();
    }

    template <int S, bool STAGED>
    __device__ static __forceinline__ void stages(cplx<T>* v, cplx<T>* sm, const cplx<T>* __restrict__ tw, int t) {
        if constexpr (S < NS) {
            constexpr int R = PL::radix(INV, S);
            constexpr int PS = PL::sub(INV, S);
            compute<R, PS, S, STAGED>(v, tw, t);
            if constexpr (S + 1 < NS) {
                exchange<R, PS, PL::radix(INV, S + 1)>(v, sm, t);
            }
            stages<S + 1, STAGED>(v, sm, tw, t);
        }
    }

    // v: UPT*EPT registers (unit-major); sm: this group's SMEM_ELEMS shared elements; tw: the
    // linear table w^m, or with STAGED the by-stage table of fill_stage_twiddles.
    // The caller fills v in in_pos order; on return v holds the transform in out_pos order.
    // Contains __syncthreads(): every thread of the block must call it.
    template <bool STAGED = false>
    __device__ static __forceinline__ void run(cplx<T>* v, cplx<T>* sm, const cplx<T>* __restrict__ tw, int t) {
        stages<0, STAGED>(v, sm, tw, t);
    }
};

// Twiddles a length-N RegFFT reads: w^m for m < N/2 (the largest index any stage forms is
// R/2 * k * N/(PS*R) < N/2).  With BASTR_TW_SMEM the kernels keep them in shared memory in the
// by-stage layout (fill_stage_twiddles); otherwise the transforms read the linear table.
#ifndef BASTR_TW_SMEM
#define BASTR_TW_SMEM 1
#endif
// Shared bytes of the by-stage tables of the transforms F... (one after the other).
template <typename T, class... F> constexpr size_t tw_stage_bytes() {
    return BASTR_TW_SMEM ? (size_t)(0 + ... + F::TWS_ELEMS) * sizeof(cplx<T>) : 0;
}

}  // namespace bastr
