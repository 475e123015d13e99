// 3D right-hand side as five fused passes (compute_ut3D, solution.F90:865-928, with the RK3/CN
// combinations of solution.F90:233-301 folded into the last pass).  Every pass is a persistent
// loop over groups of G lines staged through shared memory with cp.async, transformed in
// registers, and written transposed for the next pass:
//
//   A  zinv : lines (kx,ky) along kz of the truncated state -> MA[kx][kyi][f][z]
//             f = g_c = IFFT_z(u_c^), h_c = IFFT_z(i kz u_c^)       (+ q_c = IFFT_z(kz^2 u_c^),
//             t = IFFT_z(lap(theta)^) when velocity-gradient statistics are due)
//   B  yinv : lines (kx,z) along ky -> MB[z][kx][f][y] (each line's outputs contiguous per field)
//             f = G_c = IFFT_y(g_c), Dy_c = IFFT_y(i ky g_c), Dz_c = IFFT_y(h_c)  (+ lap u_c, lap theta)
//   C  xpass: rows (y,z): six packed complex inverse x transforms give u_c and all nine
//             du_i/dx_j in registers; N_i = -(u_j du_i/dx_j) (solution.F90:903-908); two packed
//             forward transforms -> MC[z][kx][y][c]
//   D  yfwd : lines (kx,z) along y, truncated to |ky| < K -> MD[kx][kyi][z][c]
//   E  zfwd : lines (kx,ky) along z, truncated to |kz| < K, 1/N, spherical dealias
//             (tool.F90:196-217), viscous term, projection (tool.F90:245-270), RK/CN combination.
#include "regfft.cuh"
#include "solver.cuh"
#include "tma.cuh"

// Units of the 3D x pass's inverse transforms that share one shared-memory exchange (the rest
// run as further transforms through the same buffer), and the blocks per SM asked of the
// register allocator for the FP32 product passes (0: no request).
#ifndef BASTR_X3_ZA
#define BASTR_X3_ZA 8
#endif
#ifndef BASTR_MINB_X3
#define BASTR_MINB_X3 0
#endif
// Line pairing of the 3D x and y-inverse passes (0: one line per warp; 1: a line per half-warp;
// 2: lines alternating every 8 lanes, the fastest at 256^3 FP32).
#ifndef BASTR_X3_PAIR
#define BASTR_X3_PAIR 2
#endif

namespace bastr {

// Passes that hold many units at once use 32 bytes per unit per thread.
template <typename T> struct EptWide { static constexpr int v = sizeof(T) == 8 ? 4 : 8; };

// ---------------------------------------------------------------------------------------
// Pass A
// ---------------------------------------------------------------------------------------
enum ZInvSet : int { ZI_STATE = 0, ZI_RHS = 1, ZI_VG = 2 };

template <typename T, typename TIN, int NZ, int SET> struct ZInv3D {
    static constexpr int F = SET == ZI_STATE ? 3 : SET == ZI_RHS ? 6 : 4;
    static constexpr int F0 = SET == ZI_VG ? 6 : 0;
    static constexpr int UG = SET == ZI_STATE ? 3 : 2;
    static constexpr int NG = (F + UG - 1) / UG;
    static constexpr int EPT = ept_fit<NZ, EptWide<T>::v>();
    using FFT = RegFFT<T, NZ, EPT, UG, true>;
    static constexpr int G = groups_per_block<FFT::NTR>();
    static constexpr int NT = G * FFT::NTR;
    static constexpr size_t XCH = (size_t)G * FFT::SMEM_ELEMS * sizeof(cplx<T>);
    // staging of G lines of KZ modes for each of the 3 component planes, sized at run time
    __host__ __device__ static size_t plane_bytes(int KZ) {
        return ((size_t)G * KZ * sizeof(cplx<TIN>) + 15) & ~(size_t)15;
    }
    __host__ __device__ static size_t stage_bytes(int KZ) { return 3 * plane_bytes(KZ); }
    static size_t smem(int KZ) { return stage_bytes(KZ) + XCH; }
};

template <typename T, typename TIN, int NZ, int SET>
__global__ void __launch_bounds__(ZInv3D<T, TIN, NZ, SET>::NT)
k3d_zinv(const cplx<TIN>* __restrict__ S, cplx<T>* __restrict__ MA, int ftot, Geo g,
         const cplx<T>* __restrict__ tw) {
    pdl_wait();
    if (halted(g)) return;
    using P = ZInv3D<T, TIN, NZ, SET>;
    using FFT = typename P::FFT;
    constexpr int EPT = P::EPT, UG = P::UG, F = P::F, G = P::G;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<TIN>* stg = reinterpret_cast<cplx<TIN>*>(smraw);
    const int gi = threadIdx.x / FFT::NTR, t = threadIdx.x % FFT::NTR;
    const int K = g.K, KY = g.KY, KZ = g.KZ;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw + P::stage_bytes(KZ)) + gi * FFT::SMEM_ELEMS;
    const int nlines = K * KY;                 // line = kx*KY + kyi
    const int nitems = (nlines + G - 1) / G;
    const size_t pe = P::plane_bytes(KZ) / sizeof(cplx<TIN>);   // staged elements per plane
    auto issue = [&](int item) {
        const int l0 = item * G;
        const int nl = min(G, nlines - l0);
#pragma unroll
        for (int c = 0; c < 3; ++c)
            stage_line(stg + c * pe, S + c * g.ps + (size_t)l0 * KZ, nl * KZ * (int)sizeof(cplx<TIN>), g);
        cp_async_commit();
    };
    int item = blockIdx.x;
    if (item < nitems) issue(item);
    for (; item < nitems; item += gridDim.x) {
        cp_async_wait<0>();
        __syncthreads();
        const int l = item * G + gi;
        const bool valid = l < nlines;
        const int kx = l / KY, kyi = l - kx * KY;
        const T kxt = (T)kx, kyt = (T)trunc_k(kyi, K, KY);
        const cplx<TIN>* line = stg + (size_t)gi * KZ;
        cplx<T> r[3][EPT];
#pragma unroll
        for (int e = 0; e < EPT; ++e) {
            const int kzi = pos_trunc(FFT::in_pos(t, e), K, KZ, NZ);
            const bool on = valid && kzi >= 0;
#pragma unroll
            for (int c = 0; c < 3; ++c) r[c][e] = on ? cvt<cplx<TIN>, cplx<T>>(line[c * pe + kzi]) : mk<T>(0, 0);
        }
        __syncthreads();   // the staging buffer is free: fetch the next line group now
        if (item + (int)gridDim.x < nitems) issue(item + gridDim.x);
#pragma unroll
        for (int grp = 0; grp < P::NG; ++grp) {
            cplx<T> v[UG * EPT];
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                const int kzi = pos_trunc(FFT::in_pos(t, e), K, KZ, NZ);
                const T kz = (T)(kzi >= 0 ? trunc_k(kzi, K, KZ) : 0);
                if constexpr (SET == ZI_STATE) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) v[c * EPT + e] = r[c][e];
                } else if constexpr (SET == ZI_RHS) {
                    v[e] = r[grp][e];
                    v[EPT + e] = cscale<T>(cmuli<T>(r[grp][e]), kz);
                } else {
                    const T kz2 = kz * kz;
                    if (grp == 0) {
                        v[e] = cscale<T>(r[0][e], kz2);
                        v[EPT + e] = cscale<T>(r[1][e], kz2);
                    } else {
                        v[e] = cscale<T>(r[2][e], kz2);
                        // lap(theta)^ = -i |k|^2 (k . u^)   (solution.F90:1216)
                        const T kk = kxt * kxt + kyt * kyt + kz2;
                        const cplx<T> dv = cadd<T>(cadd<T>(cscale<T>(r[0][e], kxt), cscale<T>(r[1][e], kyt)),
                                                   cscale<T>(r[2][e], kz));
                        v[EPT + e] = cscale<T>(cmulni<T>(dv), kk);
                    }
                }
            }
            FFT::run(v, sm, tw, t);
            if (valid) {
                // MA[kx][kyi][f][z]: each line's field is a contiguous run along z
                cplx<T>* dst = MA + ((size_t)l * ftot + P::F0 + grp * UG) * NZ;
#pragma unroll
                for (int u = 0; u < UG; ++u) {
                    if (grp * UG + u < F) {
#pragma unroll
                        for (int e = 0; e < EPT; ++e) BASTR_AT(dst, (size_t)u * NZ + FFT::out_pos(t, e), g) = v[u * EPT + e];
                    }
                }
            }
        }
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------------
// Pass B
// ---------------------------------------------------------------------------------------
enum YInv3Set : int { YB_STATE = 0, YB_RHS = 1, YB_RHS_VG = 2 };

template <typename T, int NY, int SET> struct YInv3D {
    static constexpr int FIN = SET == YB_STATE ? 3 : SET == YB_RHS ? 6 : 10;
    static constexpr int F = SET == YB_STATE ? 3 : SET == YB_RHS ? 9 : 13;
    static constexpr int UG = 3;
    static constexpr int NG = (F + UG - 1) / UG;
    static constexpr int EPT = ept_fit<NY, EptWide<T>::v>();
    using FFT = RegFFT<T, NY, EPT, UG, true>;
    // lines of one block: consecutive z of one kx (every extent is a power of two >= 16)
    static constexpr int G = groups_per_block<FFT::NTR>() > 16 ? 16 : groups_per_block<FFT::NTR>();
    static constexpr int NT = G * FFT::NTR;
    static constexpr size_t XCH = (size_t)G * FFT::SMEM_ELEMS * sizeof(cplx<T>);
    // lines served in pairs by pairs of warps, as in the x pass (one warp's worth of threads per
    // line, an even number of lines, exchange buffers a multiple of 128 bytes long)
    static constexpr bool PAIRED = BASTR_X3_PAIR > 0 && FFT::NTR == 32 && G % 2 == 0 &&
                                   (FFT::SMEM_ELEMS * (int)sizeof(cplx<T>)) % 128 == 0;
    // TMA staging of the product fields (FP32): the group's [kyi][f][4 lines] values as one box of
    // a 4-D tensor map over MA (KY < NY <= 256 modes in one box) with the 32-byte swizzle and one
    // field more than MA holds (read as zeros), an odd number of 32-byte rows per mode: a model of
    // the banks gives conflict-free 8-byte reads for the paired lines (the dense unswizzled layout
    // of 6 or 10 fields is 8-way conflicted)
    static constexpr bool TMA = PAIRED && sizeof(T) == 4 && G == 4 && SET != YB_STATE && NY <= 256;
    static constexpr int FB = TMA ? FIN + 1 : FIN;                 // staged fields per mode
    // staging [kyi][f][line] of KY modes x FB fields, sized at run time
    __host__ __device__ static size_t stage_bytes(int KY) {
        const size_t b = (size_t)G * KY * FB * sizeof(cplx<T>);
        return TMA ? 1024 + ((b + 1023) & ~(size_t)1023) : (b + 15) & ~(size_t)15;
    }
    static size_t smem(int KY) { return stage_bytes(KY) + XCH; }
};

template <typename T, int NY, int SET>
__global__ void __launch_bounds__(YInv3D<T, NY, SET>::NT)
k3d_yinv(const cplx<T>* __restrict__ MA, cplx<T>* __restrict__ MB, Geo g, const cplx<T>* __restrict__ tw,
         const __grid_constant__ CUtensorMap tma_map) {
    pdl_wait();
    if (halted(g)) return;
    using P = YInv3D<T, NY, SET>;
    using FFT = typename P::FFT;
    constexpr int EPT = P::EPT, UG = P::UG, F = P::F, FIN = P::FIN, G = P::G;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* stg = reinterpret_cast<cplx<T>*>(smraw);
    // line of this thread: pairs of lines served by pairs of warps, alternating every 8 lanes
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int gi = !P::PAIRED ? threadIdx.x / FFT::NTR
                 : BASTR_X3_PAIR == 1 ? 2 * (wp >> 1) + ((wp & 1) ^ (lane >> 4))
                                      : 2 * (wp >> 1) + (((lane >> 3) & 1) ^ (wp & 1));
    const int t = P::PAIRED ? lane : threadIdx.x % FFT::NTR;
    const int K = g.K, KY = g.KY, NZ = g.nz;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw + P::stage_bytes(KY)) + gi * FFT::SMEM_ELEMS;
    const int nlines = K * NZ;                 // line = kx*NZ + z
    const int nitems = (nlines + G - 1) / G;
    // TMA tile at the first 1024-byte boundary of the staging area
    unsigned char* tmat = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    __shared__ __align__(8) uint64_t bar;
    if constexpr (P::TMA) {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
    }
    uint32_t phase = 0;
    bool lost = false;   // a TMA completion wait gave up (recorded in g.err)
    auto issue = [&](int item) {
        // gather [kyi][f][z] from MA[kx][kyi][f][z]: G consecutive z per (kyi, f)
        const int l0 = item * G, kx0 = l0 / NZ, z0 = l0 - kx0 * NZ;
        if constexpr (P::TMA) {
            if (threadIdx.x == 0) {
                mbar_expect_tx(&bar, (uint32_t)(G * KY * P::FB * (int)sizeof(cplx<T>)));
                tma_load_4d(tmat, &tma_map, 2 * z0, 0, 0, kx0, &bar);
            }
            return;
        }
        constexpr int RB = G * (int)sizeof(cplx<T>);
        constexpr int CH = RB % 16 == 0 ? 16 : 8;
        constexpr int NCH = RB / CH;
        const int total = KY * FIN * NCH;
        char* d = reinterpret_cast<char*>(stg);
        const char* src = reinterpret_cast<const char*>(MA + (size_t)kx0 * KY * FIN * NZ + z0);
        for (int i = threadIdx.x; i < total; i += P::NT) {
            const int kf = i / NCH, c = i - kf * NCH;
            const char* sp = src + (size_t)kf * NZ * sizeof(cplx<T>) + c * CH;
            if constexpr (CH == 16) cp_async16(d + (size_t)kf * RB + c * CH, BASTR_CHK(sp, 16, g));
            else cp_async8(d + (size_t)kf * RB + c * CH, BASTR_CHK(sp, 8, g));
        }
        cp_async_commit();
    };
    int item = blockIdx.x;
    if (item < nitems) issue(item);
    for (; item < nitems; item += gridDim.x) {
        if constexpr (P::TMA) {
            const bool ok = mbar_wait(&bar, phase, g.err);
            if (__syncthreads_or(!ok)) {   // block-uniform: stop, and drain below
                lost = true;
                break;
            }
            phase ^= 1u;
        } else {
            cp_async_wait<0>();
            __syncthreads();
        }
        const int l = item * G + gi;
        const bool valid = l < nlines;
        const int kx = l / NZ, z = l - kx * NZ;
        // field f of mode kyi for this line at stg[(kyi*FIN + f)*G + gi]
        const cplx<T>* line = stg + gi;
#pragma unroll
        for (int grp = 0; grp < P::NG; ++grp) {
            cplx<T> v[UG * EPT];
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                const int kyi = pos_trunc(FFT::in_pos(t, e), K, KY, NY);
                cplx<T> f[UG];
#pragma unroll
                for (int u = 0; u < UG; ++u) f[u] = mk<T>(0, 0);
                if (valid && kyi >= 0) {
                    const T ky = (T)trunc_k(kyi, K, KY);
                    const cplx<T>* src0 = line + (size_t)kyi * FIN * G;
                    auto src = [&](int fi) -> cplx<T> {
                        if constexpr (P::TMA)
                            return *reinterpret_cast<const cplx<T>*>(
                                tmat + swz<32>((uint32_t)((kyi * P::FB + fi) * G + gi) * (uint32_t)sizeof(cplx<T>)));
                        else return src0[fi * G];
                    };
                    if constexpr (SET == YB_STATE) {
                        f[0] = src(0); f[1] = src(1); f[2] = src(2);
                    } else {
                        if (grp < 3) {   // component grp: G, Dy, Dz
                            const cplx<T> gc = src(2 * grp), hc = src(2 * grp + 1);
                            f[0] = gc;
                            f[1] = cscale<T>(cmuli<T>(gc), ky);
                            f[2] = hc;
                        } else if (grp == 3) {
                            // lap u_c without its kx^2 part (added in pass C): -ky^2 g_c - IFFT_z(kz^2 u_c^)
                            const T ky2 = ky * ky;
#pragma unroll
                            for (int c = 0; c < 3; ++c) f[c] = csub<T>(cscale<T>(src(2 * c), -ky2), src(6 + c));
                        } else {
                            f[0] = src(9);
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < UG; ++u) v[u * EPT + e] = f[u];
            }
            if (grp == P::NG - 1) {
                __syncthreads();   // staging buffer consumed: fetch the next line group
                if (item + (int)gridDim.x < nitems) issue(item + gridDim.x);
            }
            FFT::run(v, sm, tw, t);
            if (valid) {
                cplx<T>* dst = MB + ((size_t)(z * K + kx) * F + grp * UG) * NY;
#pragma unroll
                for (int u = 0; u < UG; ++u) {
                    if (grp * UG + u < F) {
#pragma unroll
                        for (int e = 0; e < EPT; ++e) BASTR_AT(dst, (size_t)u * NY + FFT::out_pos(t, e), g) = v[u * EPT + e];
                    }
                }
            }
        }
    }
    cp_async_wait<0>();
    if constexpr (P::TMA) {
        if (lost && threadIdx.x == 0) mbar_wait(&bar, phase, nullptr);   // bounded drain
    }
    (void)lost;
}

// ---------------------------------------------------------------------------------------
// Pass C
// ---------------------------------------------------------------------------------------
enum X3Mode : int { X3_RHS = 1, X3_RHS_VG = 2, X3_TO_PHYS = 3, X3_FROM_PHYS = 4 };


template <typename T, int NX, int MODE> struct XPass3D {
    static constexpr int FIN = MODE == X3_RHS ? 9 : MODE == X3_RHS_VG ? 13 : MODE == X3_TO_PHYS ? 3 : 0;
    static constexpr int ZU = MODE == X3_RHS ? 6 : MODE == X3_RHS_VG ? 8 : 2;
    static constexpr int EPT = ept_fit<NX, (MODE == X3_RHS || MODE == X3_RHS_VG) ? EptWide<T>::v : EptOf<T>::v>();
    static constexpr int ZA = ZU < BASTR_X3_ZA ? ZU : (BASTR_X3_ZA < 2 ? 2 : BASTR_X3_ZA);
    using IFFT = RegFFT<T, NX, EPT, ZA, true>;
    static constexpr int MINB = (BASTR_MINB_X3 > 0 && sizeof(T) == 4 && (MODE == X3_RHS || MODE == X3_RHS_VG))
                                    ? BASTR_MINB_X3 : 1;
    using FFFT = RegFFT<T, NX, EPT, 2, false>;
    static constexpr int NTR = IFFT::NTR;
    // rows of one block: consecutive y of one z plane (every extent is a power of two >= 16)
    static constexpr int G = groups_per_block<NTR>() > 16 ? 16 : groups_per_block<NTR>();
    static constexpr int NT = G * NTR;
    static constexpr int KMAX = NX / 3;
    // staging [kx][f][row]: the threads of a warp touch consecutive wavenumbers, so one
    // wavenumber's run is made an odd number of 16-byte units long (a multiple of 32 bytes puts
    // the threads a multiple of the bank width apart), and in FP32 a tile row of one wavenumber
    // an odd number of elements (4-way conflicts otherwise; FP64 has 2-way ones and keeps its
    // tile unpadded, which leaves the velocity-gradient variant two blocks per SM)
    static constexpr int KPAD = (FIN * G * (int)sizeof(cplx<T>) / 16) % 2 == 0 ? 16 / (int)sizeof(cplx<T>) : 0;
    static constexpr int KSTR = FIN * G + KPAD;        // staged elements per kx
    // rows served in pairs by pairs of warps (see k3d_xpass): with one warp's worth of threads
    // per row, an even number of rows and exchange buffers a multiple of 128 bytes long
    static constexpr bool PAIRED = BASTR_X3_PAIR > 0 && NTR == 32 && G % 2 == 0 &&
                                   (IFFT::SMEM_ELEMS * (int)sizeof(cplx<T>)) % 128 == 0;
    // tile elements per kx in FP32: for paired rows an even stride twice an odd number (the two
    // rows on opposite bank parities: conflict-free split stores), otherwise odd; the
    // velocity-gradient variant keeps the odd one, since two more elements per kx would leave it
    // one block per SM
    static constexpr int TSTR = sizeof(T) != 4 ? 3 * G : (PAIRED && MODE == X3_RHS) ? 3 * G + 2 : ((3 * G) | 1);
    // TMA staging (the FP32 product passes with paired rows): the row group's [kx][f][4 rows]
    // values as one box of a 4-D tensor map over MB, unpadded and swizzled at 32 bytes, which
    // keeps the paired rows' 8-byte reads conflict-free; one elected thread issues it
    static constexpr bool TMA = PAIRED && sizeof(T) == 4 && G == 4 && (MODE == X3_RHS || MODE == X3_RHS_VG) &&
                                KMAX <= 256;
    static constexpr uint32_t TX_BYTES = (uint32_t)(KMAX * FIN * G * sizeof(cplx<T>));
    static constexpr size_t STAGE = TMA ? 1024 + (((size_t)TX_BYTES + 1023) & ~(size_t)1023)
                                  : MODE == X3_FROM_PHYS ? (size_t)G * 3 * NX * sizeof(double)
                                                         : (size_t)KMAX * KSTR * sizeof(cplx<T>);
    static constexpr size_t TILE = (size_t)KMAX * TSTR * sizeof(cplx<T>);   // output tile [kx][row][c]
    static constexpr size_t XCH = (size_t)G * IFFT::SMEM_ELEMS * sizeof(cplx<T>);
    static constexpr size_t XCHR = XCH > (size_t)9 * NT * 8 ? XCH : (size_t)9 * NT * 8;
    static constexpr size_t SMEM = STAGE + TILE + XCHR;
};

// Inverse transforms of units [U0, ZU) in runs of at most ZA units through one exchange buffer.
template <typename T, int NX, int EPT, int ZU, int ZA, int U0 = 0>
__device__ __forceinline__ void x3_inverse_runs(cplx<T>* v, cplx<T>* sm, const cplx<T>* __restrict__ tw, int t) {
    if constexpr (U0 < ZU) {
        constexpr int NU = ZU - U0 < ZA ? ZU - U0 : ZA;
        RegFFT<T, NX, EPT, NU, true>::run(v + U0 * EPT, sm, tw, t);
        x3_inverse_runs<T, NX, EPT, ZU, ZA, U0 + NU>(v, sm, tw, t);
    }
}

template <typename T, int NX, int MODE>
__global__ void __launch_bounds__(XPass3D<T, NX, MODE>::NT, XPass3D<T, NX, MODE>::MINB)
k3d_xpass(const cplx<T>* __restrict__ MB, cplx<T>* __restrict__ MC, const double* __restrict__ phys_in,
          double* __restrict__ phys_out, double* __restrict__ vg_part, Geo g, const cplx<T>* __restrict__ tw,
          const __grid_constant__ CUtensorMap tmb) {
    pdl_wait();
    if (halted(g)) return;
    using P = XPass3D<T, NX, MODE>;
    using IFFT = typename P::IFFT;
    using FFFT = typename P::FFFT;
    constexpr int ZU = P::ZU, EPT = P::EPT, NT = P::NT, NTR = P::NTR, FIN = P::FIN, G = P::G;
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* stg = smraw;
    cplx<T>* tile = reinterpret_cast<cplx<T>*>(smraw + P::STAGE);
    // Row of this thread.  With one warp's worth of threads per row, the rows are taken in pairs
    // by pairs of warps, alternating every 8 lanes (lanes with bit 3 clear serve row 2p + h, the
    // others row 2p + 1 - h, for warp 2p + h; t = lane either way).  The two rows' staged values
    // sit in opposite halves of each 16-byte chunk, so each half-warp's 8-byte loads of
    // consecutive wavenumbers reach all 32 banks once (one row alone reaches only the banks of one
    // half: 2-way conflicts).  The rows' exchange buffers are a multiple of 128 bytes apart, so the
    // exchanges keep their bank pattern.
    constexpr bool PAIRED = P::PAIRED;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int gi = !PAIRED ? threadIdx.x / NTR
                 : BASTR_X3_PAIR == 1 ? 2 * (wp >> 1) + ((wp & 1) ^ (lane >> 4))
                                      : 2 * (wp >> 1) + (((lane >> 3) & 1) ^ (wp & 1));
    const int t = PAIRED ? lane : threadIdx.x % NTR;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw + P::STAGE + P::TILE) + gi * IFFT::SMEM_ELEMS;
    const int K = g.K, NY = g.ny;
    const int rows = NY * g.nz;
    const size_t npts = (size_t)NX * rows;
    const int nitems = (rows + G - 1) / G;
    // TMA tile at the first 1024-byte boundary of the staging area
    unsigned char* tmat = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    __shared__ __align__(8) uint64_t bar;
    if constexpr (P::TMA) {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
    }
    uint32_t phase = 0;
    bool lost = false;   // a TMA completion wait gave up (recorded in g.err)
    auto issue = [&](int item) {
        const int r0 = item * G;   // G consecutive y rows of one z plane
        if constexpr (P::TMA) {
            if (threadIdx.x == 0) {
                const int z0 = r0 / NY, y0 = r0 - z0 * NY;
                mbar_expect_tx(&bar, P::TX_BYTES);
                tma_load_4d(tmat, &tmb, 2 * y0, 0, 0, z0, &bar);
            }
            return;
        } else if constexpr (MODE == X3_FROM_PHYS) {
            double* d = reinterpret_cast<double*>(stg);
#pragma unroll
            for (int c = 0; c < 3; ++c) stage_line(d + (size_t)c * G * NX, phys_in + c * npts + (size_t)r0 * NX, G * NX * 8, g);
        } else {
            // gather [kx][f][row] from MB[z][kx][f][y]: G consecutive y per (kx, f)
            const int z0 = r0 / NY, y0 = r0 - z0 * NY;
            constexpr int RB = G * (int)sizeof(cplx<T>);           // bytes per (kx, f)
            constexpr int CH = RB % 16 == 0 ? 16 : 8;              // copy granule
            constexpr int NCH = RB / CH;
            const int total = K * FIN * NCH;
            char* d = reinterpret_cast<char*>(stg);
            const char* src = reinterpret_cast<const char*>(MB + (size_t)z0 * K * FIN * NY + y0);
            for (int i = threadIdx.x; i < total; i += NT) {
                const int kf = i / NCH, c = i - kf * NCH;
                const int k = kf / FIN;
                const char* sp = src + ((size_t)kf * NY * sizeof(cplx<T>)) + c * CH;
                char* dp = d + (size_t)k * P::KSTR * sizeof(cplx<T>) + (size_t)(kf - k * FIN) * RB + c * CH;
                if constexpr (CH == 16) cp_async16(dp, BASTR_CHK(sp, 16, g));
                else cp_async8(dp, BASTR_CHK(sp, 8, g));
            }
        }
        cp_async_commit();
    };
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double divmax = 0.0;
    int item = blockIdx.x;
    if (item < nitems) issue(item);
    for (; item < nitems; item += gridDim.x) {
        if constexpr (P::TMA) {
            const bool ok = mbar_wait(&bar, phase, g.err);
            if (__syncthreads_or(!ok)) {   // block-uniform: stop, and drain below
                lost = true;
                break;
            }
            phase ^= 1u;
        } else {
            cp_async_wait<0>();
            __syncthreads();
        }
        const int row = item * G + gi;   // row = z*NY + y
        const bool valid = row < rows;
        cplx<T> v[ZU * EPT];
        if constexpr (MODE == X3_FROM_PHYS) {
            const double* d = reinterpret_cast<const double*>(stg) + (size_t)gi * NX;
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                const int x = FFFT::in_pos(t, e);
                v[e] = valid ? mk<T>((T)d[x], (T)d[(size_t)G * NX + x]) : mk<T>(0, 0);
                v[EPT + e] = valid ? mk<T>((T)d[(size_t)2 * G * NX + x], (T)0) : mk<T>(0, 0);
            }
        } else {
            // staged as [kx][f][row]: field f of wavenumber k for this row at (k*FIN + f)*G + gi
            const cplx<T>* rw = reinterpret_cast<const cplx<T>*>(stg) + gi;
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                const int p = IFFT::in_pos(t, e);
                const bool lo = p < K, hi = p > NX - K;
                const int k = lo ? p : NX - p;
#pragma unroll
                for (int u = 0; u < ZU; ++u) v[u * EPT + e] = mk<T>(0, 0);
                // K = floor(NX/3): these elements are dealiased zeros for every thread
                if (IFFT::in_band(e, NX / 3 + 1)) continue;
                if (valid && (lo || hi)) {
                    const cplx<T>* src0 = rw + (size_t)k * P::KSTR;
                    auto src = [&](int f) -> cplx<T> {
                        if constexpr (P::TMA)
                            return *reinterpret_cast<const cplx<T>*>(
                                tmat + swz<32>((uint32_t)((k * FIN + f) * G + gi) * (uint32_t)sizeof(cplx<T>)));
                        else return src0[f * G];
                    };
                    const bool z0 = p == 0;
                    if constexpr (MODE == X3_TO_PHYS) {
                        v[e] = pack_at<T>(src(0), src(1), hi, z0);
                        v[EPT + e] = pack_at<T>(src(2), mk<T>(0, 0), hi, z0);
                    } else {
                        const T kx = (T)k;
                        const cplx<T> G1 = src(0), Dy1 = src(1), Dz1 = src(2);
                        const cplx<T> G2 = src(3), Dy2 = src(4), Dz2 = src(5);
                        const cplx<T> G3 = src(6), Dy3 = src(7), Dz3 = src(8);
                        const cplx<T> X1 = cscale<T>(cmuli<T>(G1), kx), X2 = cscale<T>(cmuli<T>(G2), kx),
                                      X3 = cscale<T>(cmuli<T>(G3), kx);
                        v[e] = pack_at<T>(G1, G2, hi, z0);                 // u1, u2
                        v[EPT + e] = pack_at<T>(G3, X1, hi, z0);           // u3, du1/dx
                        v[2 * EPT + e] = pack_at<T>(X2, X3, hi, z0);       // du2/dx, du3/dx
                        v[3 * EPT + e] = pack_at<T>(Dy1, Dy2, hi, z0);     // du1/dy, du2/dy
                        v[4 * EPT + e] = pack_at<T>(Dy3, Dz1, hi, z0);     // du3/dy, du1/dz
                        v[5 * EPT + e] = pack_at<T>(Dz2, Dz3, hi, z0);     // du2/dz, du3/dz
                        if constexpr (MODE == X3_RHS_VG) {
                            const T kx2 = kx * kx;
                            v[6 * EPT + e] = pack_at<T>(csub<T>(src(9), cscale<T>(G1, kx2)),
                                                        csub<T>(src(10), cscale<T>(G2, kx2)), hi, z0);
                            v[7 * EPT + e] = pack_at<T>(csub<T>(src(11), cscale<T>(G3, kx2)), src(12), hi, z0);
                        }
                    }
                }
            }
        }
        __syncthreads();   // the staging buffer is free: fetch the next row group now
        if (item + (int)gridDim.x < nitems) issue(item + gridDim.x);
        if constexpr (MODE != X3_FROM_PHYS) x3_inverse_runs<T, NX, EPT, ZU, P::ZA>(v, sm, tw, t);

        if constexpr (MODE == X3_TO_PHYS) {
            if (valid) {
#pragma unroll
                for (int e = 0; e < EPT; ++e) {
                    const int x = IFFT::out_pos(t, e);
                    const size_t o = (size_t)row * NX + x;
                    BASTR_AT(phys_out, o, g) = (double)v[e].x;
                    BASTR_AT(phys_out, npts + o, g) = (double)v[e].y;
                    BASTR_AT(phys_out, 2 * npts + o, g) = (double)v[EPT + e].x;
                }
            }
        } else {
            if constexpr (MODE == X3_RHS || MODE == X3_RHS_VG) {
                const double nu = g.nu;
#pragma unroll
                for (int e = 0; e < EPT; ++e) {
                    const cplx<T> z0 = v[e], z1 = v[EPT + e], z2 = v[2 * EPT + e];
                    const cplx<T> z3 = v[3 * EPT + e], z4 = v[4 * EPT + e], z5 = v[5 * EPT + e];
                    const T u1 = z0.x, u2 = z0.y, u3 = z1.x;
                    const T d11 = z1.y, d21 = z2.x, d31 = z2.y;   // d_ij = du_i/dx_j
                    const T d12 = z3.x, d22 = z3.y, d32 = z4.x;
                    const T d13 = z4.y, d23 = z5.x, d33 = z5.y;
                    const T n1 = -u1 * d11 - u2 * d12 - u3 * d13;
                    const T n2 = -u1 * d21 - u2 * d22 - u3 * d23;
                    const T n3 = -u1 * d31 - u2 * d32 - u3 * d33;
                    v[e] = mk<T>(n1, n2);
                    v[EPT + e] = mk<T>(n3, (T)0);
                    if constexpr (MODE == X3_RHS_VG) {
                        if (valid) {
                            // velgrad_calculate3D (solution.F90:1240-1266): per-point terms in the
                            // compute precision, sums in FP64, eta_min from the largest |theta|
                            const cplx<T> z6 = v[6 * EPT + e], z7 = v[7 * EPT + e];
                            const T nuT = (T)nu;
                            const T div = d11 + d22 + d33;
                            const T uu = u1 * u1 + u2 * u2 + u3 * u3;
                            acc[0] += (double)(div * div * uu);
                            acc[1] += (double)((d11 * d11 + d22 * d22 + d33 * d33 + (T)2 * d12 * d21 +
                                                (T)2 * d13 * d31 + (T)2 * d23 * d32) * uu);
                            acc[2] += (double)(div * uu);
                            acc[3] += (double)((T)2 * u1 * div * z6.x + (T)2 * u2 * div * z6.y +
                                               (T)2 * u3 * div * z7.x + uu * z7.y);
                            acc[4] += (double)(nuT * (d12 - d21) * (d12 - d21) + nuT * (d23 - d32) * (d23 - d32) +
                                               nuT * (d13 - d31) * (d13 - d31) + nuT * div * div);
                            divmax = fmax(divmax, (double)fabs(div));
                            acc[5] += (double)uu;
                            acc[6] += (double)(d11 * d11 + d22 * d22 + d33 * d33);
                        }
                    }
                }
            }
            FFFT::run(v, sm, tw, t);
            // split: unit 0 -> components 0, 1; unit 1 -> component 2
            constexpr int US = IFFT::US;
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                if (FFFT::out_band(e, NX / 3 + 1)) continue;   // never read by the split below
                const int x = FFFT::out_pos(t, e);
                sm[pidx(x)] = v[e];
                sm[US + pidx(x)] = v[EPT + e];
            }
            __syncthreads();
            for (int k = t; k < K; k += NTR) {
                const int km = k == 0 ? 0 : NX - k;
                cplx<T>* dst = tile + (size_t)k * P::TSTR + gi * 3;
                const cplx<T> Z = sm[pidx(k)], Zc = cconj<T>(sm[pidx(km)]);
                const cplx<T> W = sm[US + pidx(k)], Wc = cconj<T>(sm[US + pidx(km)]);
                dst[0] = cscale<T>(cadd<T>(Z, Zc), (T)0.5);
                dst[1] = cscale<T>(cmulni<T>(csub<T>(Z, Zc)), (T)0.5);
                dst[2] = cscale<T>(cadd<T>(W, Wc), (T)0.5);
            }
            __syncthreads();
            // MC[z][kx][y][c]: the block's G rows of one kx are G*3 contiguous values
            const int r0 = item * G, z0 = r0 / NY, y0 = r0 - z0 * NY;
            for (int i = threadIdx.x; i < K * G * 3; i += NT) {
                const int k = i / (G * 3), rem = i - k * (G * 3);
                BASTR_AT(MC, (((size_t)z0 * K + k) * NY + y0) * 3 + rem, g) = tile[(size_t)k * P::TSTR + rem];
            }
        }
    }
    cp_async_wait<0>();
    if constexpr (P::TMA) {
        if (lost && threadIdx.x == 0) mbar_wait(&bar, phase, nullptr);   // bounded drain
    }
    (void)lost;
    if constexpr (MODE == X3_RHS_VG) {
        __syncthreads();
        double* scratch = reinterpret_cast<double*>(smraw + P::STAGE + P::TILE);
        block_sum<7, NT>(acc, scratch);
        const double dm = -block_min<NT>(-divmax, scratch);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int i = 0; i < 7; ++i) BASTR_AT(vg_part, (size_t)blockIdx.x * 8 + i, g) = acc[i];
            BASTR_AT(vg_part, (size_t)blockIdx.x * 8 + 7, g) = dm;
        }
    }
}

// ---------------------------------------------------------------------------------------
// Pass D: forward y transforms, truncation to |ky| < K.
// ---------------------------------------------------------------------------------------
template <typename T, int NY> struct YFwd3D {
    static constexpr int EPT = ept_fit<NY, EptWide<T>::v>();
    using FFT = RegFFT<T, NY, EPT, 3, false>;
    // lines of one block: consecutive z of one kx (every extent is a power of two >= 16)
    static constexpr int G = groups_per_block<FFT::NTR>() > 16 ? 16 : groups_per_block<FFT::NTR>();
    static constexpr int NT = G * FFT::NTR;
    static constexpr size_t STAGE = (size_t)G * NY * 3 * sizeof(cplx<T>);
    // output tile [kyi][line][c] of the KY kept modes, TS elements per mode: an odd number in
    // FP32, so that the 8-byte stores of consecutive kyi by a warp reach distinct banks
    // (G*3 = 12 elements gave 4-way conflicts), sized at run time
    static constexpr int TS = sizeof(T) == 4 ? ((G * 3) | 1) : G * 3;
    __host__ __device__ static size_t tile_bytes(int KY) { return (((size_t)KY * TS * sizeof(cplx<T>)) + 15) & ~(size_t)15; }
    static constexpr size_t XCH = (size_t)G * FFT::SMEM_ELEMS * sizeof(cplx<T>);
    static size_t smem(int KY) { return STAGE + tile_bytes(KY) + XCH; }
};

template <typename T, int NY>
__global__ void __launch_bounds__(YFwd3D<T, NY>::NT)
k3d_yfwd(const cplx<T>* __restrict__ MC, cplx<T>* __restrict__ MD, Geo g, const cplx<T>* __restrict__ tw) {
    pdl_wait();
    if (halted(g)) return;
    using P = YFwd3D<T, NY>;
    using FFT = typename P::FFT;
    constexpr int EPT = P::EPT, G = P::G;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* stg = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* tile = reinterpret_cast<cplx<T>*>(smraw + P::STAGE);
    const int gi = threadIdx.x / FFT::NTR, t = threadIdx.x % FFT::NTR;
    const int K = g.K, KY = g.KY, NZ = g.nz;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw + P::STAGE + P::tile_bytes(KY)) + gi * FFT::SMEM_ELEMS;
    const int nlines = K * NZ;                 // line = kx*NZ + z
    const int nitems = (nlines + G - 1) / G;
    auto issue = [&](int item) {
        const int l0 = item * G;
        const int nl = min(G, nlines - l0);
        for (int j = 0; j < nl; ++j) {
            const int l = l0 + j, kx = l / NZ, z = l - kx * NZ;
            stage_line(stg + (size_t)j * NY * 3, MC + ((size_t)z * K + kx) * NY * 3, NY * 3 * (int)sizeof(cplx<T>), g);
        }
        cp_async_commit();
    };
    int item = blockIdx.x;
    if (item < nitems) issue(item);
    for (; item < nitems; item += gridDim.x) {
        cp_async_wait<0>();
        __syncthreads();
        const int l = item * G + gi;
        const bool valid = l < nlines;
        const int kx = l / NZ, z = l - kx * NZ;
        const cplx<T>* line = stg + (size_t)gi * NY * 3;
        cplx<T> v[3 * EPT];
#pragma unroll
        for (int e = 0; e < EPT; ++e) {
            const int y = FFT::in_pos(t, e);
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c * EPT + e] = valid ? line[3 * y + c] : mk<T>(0, 0);
        }
        __syncthreads();
        if (item + (int)gridDim.x < nitems) issue(item + gridDim.x);
        FFT::run(v, sm, tw, t);
#pragma unroll
        for (int e = 0; e < EPT; ++e) {
            const int kyi = pos_trunc(FFT::out_pos(t, e), K, KY, NY);
            if (kyi < 0) continue;
            cplx<T>* dst = tile + (size_t)kyi * P::TS + gi * 3;
#pragma unroll
            for (int c = 0; c < 3; ++c) dst[c] = v[c * EPT + e];
        }
        __syncthreads();
        // MD[kx][kyi][z][c]: the block's G lines of one kx are G*3 contiguous values per kyi
        {
            const int l0 = item * G, kx0 = l0 / NZ, z0 = l0 - kx0 * NZ;
            for (int i = threadIdx.x; i < KY * G * 3; i += P::NT) {
                const int kyi = i / (G * 3), rem = i - kyi * (G * 3);
                BASTR_AT(MD, (((size_t)kx0 * KY + kyi) * NZ + z0) * 3 + rem, g) = tile[(size_t)kyi * P::TS + rem];
            }
        }
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------------
// Pass E: forward z transforms + spectral epilogue.
// ---------------------------------------------------------------------------------------
template <typename T, int NZ> struct ZFwd3D {
    static constexpr int EPT = ept_fit<NZ, EptWide<T>::v>();
    using FFT = RegFFT<T, NZ, EPT, 3, false>;
    static constexpr int G = groups_per_block<FFT::NTR>();
    static constexpr int NT = G * FFT::NTR;
    static constexpr size_t STAGE = (size_t)G * NZ * 3 * sizeof(cplx<T>);
    static constexpr size_t XCH = (size_t)G * FFT::SMEM_ELEMS * sizeof(cplx<T>);
    static constexpr size_t XCHR = XCH > (size_t)NT * 8 ? XCH : (size_t)NT * 8;
    static constexpr size_t SMEM = STAGE + XCHR;
};

template <typename T, int NZ, int EPI>
__global__ void __launch_bounds__(ZFwd3D<T, NZ>::NT)
k3d_zfwd(const cplx<T>* __restrict__ MD, StageIO<T> io, int input_is_u0, Geo g, const cplx<T>* __restrict__ tw) {
    pdl_wait();
    if (halted(g)) return;
    using P = ZFwd3D<T, NZ>;
    using FFT = typename P::FFT;
    constexpr int EPT = P::EPT, NT = P::NT, G = P::G;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* stg = reinterpret_cast<cplx<T>*>(smraw);
    const int gi = threadIdx.x / FFT::NTR, t = threadIdx.x % FFT::NTR;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw + P::STAGE) + gi * FFT::SMEM_ELEMS;
    const int K = g.K, KY = g.KY, KZ = g.KZ;
    const int nlines = K * KY;                 // line = kx*KY + kyi
    const int nitems = (nlines + G - 1) / G;
    auto issue = [&](int item) {
        const int l0 = item * G;
        stage_line(stg, MD + (size_t)l0 * NZ * 3, min(G, nlines - l0) * NZ * 3 * (int)sizeof(cplx<T>), g);
        cp_async_commit();
    };
    const double inv_n = g.inv_n;
    const long long K2 = (long long)K * K;
    double en = 0.0;
    int item = blockIdx.x;
    if (item < nitems) issue(item);
    for (; item < nitems; item += gridDim.x) {
        cp_async_wait<0>();
        __syncthreads();
        const int l = item * G + gi;
        const bool valid = l < nlines;
        const int kx = l / KY, kyi = l - kx * KY;
        const cplx<T>* line = stg + (size_t)gi * NZ * 3;
        cplx<T> v[3 * EPT];
#pragma unroll
        for (int e = 0; e < EPT; ++e) {
            const int z = FFT::in_pos(t, e);
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c * EPT + e] = valid ? line[3 * z + c] : mk<T>(0, 0);
        }
        __syncthreads();
        if (item + (int)gridDim.x < nitems) issue(item + gridDim.x);
        if (valid) epi_prefetch<T, 3, EPI>(io, (size_t)l * KZ, KZ, (size_t)g.ps, input_is_u0 != 0, t, FFT::NTR);
        FFT::run(v, sm, tw, t);
        if (valid) {
            const int ky = trunc_k(kyi, K, KY);
            const double w = kx == 0 ? 1.0 : 2.0;
            const bool from_u0 = input_is_u0 != 0;
            constexpr int CH = EPT < EpiChunk<T, 3>::v ? EPT : EpiChunk<T, 3>::v;
#pragma unroll
            for (int e0 = 0; e0 < EPT; e0 += CH) {
                EpiIn<T, 3> in[CH];
#pragma unroll
                for (int j = 0; j < CH; ++j) {
                    const int kzi = pos_trunc(FFT::out_pos(t, e0 + j), K, KZ, NZ);
                    if (kzi >= 0) epi_load<T, 3, EPI>(in[j], (size_t)l * KZ + kzi, (size_t)g.ps, io, from_u0);
                }
#pragma unroll
                for (int j = 0; j < CH; ++j) {
                    const int e = e0 + j;
                    const int kzi = pos_trunc(FFT::out_pos(t, e), K, KZ, NZ);
                    if (kzi < 0) continue;
                    const int kz = trunc_k(kzi, K, KZ);
                    const size_t o = (size_t)l * KZ + kzi;   // component planes g.ps apart
                    const long long m2i = (long long)kx * kx + (long long)ky * ky + (long long)kz * kz;
                    double2 vv[3];
                    if (m2i < K2) {   // spherical 2/3 rule, tool.F90:206-214
#pragma unroll
                        for (int c = 0; c < 3; ++c) vv[c] = dscale(cvt<cplx<T>, double2>(v[c * EPT + e]), inv_n);
                    } else {
#pragma unroll
                        for (int c = 0; c < 3; ++c) vv[c] = make_double2(0, 0);
                    }
                    const double kv[3] = {(double)kx, (double)ky, (double)kz};
                    rk_apply<T, 3, EPI>(vv, kv, (double)m2i, in[j], o, (size_t)g.ps, io, from_u0, g, w, en);
                }
            }
        }
    }
    cp_async_wait<0>();
    if constexpr (EPI == EPI_RK3 || EPI == EPI_CN_LAST) {
        if (io.energy_part) {
            __syncthreads();
            double* scratch = reinterpret_cast<double*>(smraw + P::STAGE);
            double r[1] = {en};
            block_sum<1, NT>(r, scratch);
            if (threadIdx.x == 0) BASTR_AT(io.energy_part, blockIdx.x, io) = r[0];
        }
    }
}

}  // namespace bastr
