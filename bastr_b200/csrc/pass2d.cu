// 2D right-hand side as three fused passes over HBM (the hot path of compute_ut2D,
// solution.F90:816-863, with the RK3/CN combinations of solution.F90:172-231 folded into the
// last pass).
//
//   A  yinv : per kx column, inverse y transforms of the truncated spectrum -> mixed (kx, y)
//             MA[kx][group][y][W]: the fields f = g1,h1,g2,h2 (| q1,q2,t,0 when velocity-gradient
//             statistics are due) in records of W = 4 fields, so that a warp's store of one
//             sub-pass covers 32 consecutive y and the x pass gathers whole 32-byte sectors
//             g = IFFT_y(u^), h = IFFT_y(i ky u^), q = IFFT_y(ky^2 u^), t = IFFT_y(lap(theta)^)
//   B  xpass: per y row, three (five) packed complex inverse x transforms give u, du/dx, du/dy
//             (and lap u, lap theta) in registers; the advective product
//             N_i = -(u1 d1 u_i + u2 d2 u_i) is formed there and handed, still in registers,
//             to one packed forward x transform.  Output MB[y/2][kx][y%2][c]: a warp's store
//             covers consecutive kx of its row, and the y pass gathers whole 32-byte records of
//             two rows.
//   C  yfwd : per kx column, forward y transforms, 1/N normalisation, truncation (= the
//             spherical 2/3 dealias, tool.F90:175-194), viscous term -nu k^2 u^, dilatational
//             projection (tool.F90:219-243) and the time-integrator combination.
//
// Two real fields share one complex transform (z = a + i b), so the six real inverse and two
// real forward x transforms of the reference become three plus one complex transforms.
//
// Every pass is a persistent loop over groups of G contiguous lines, staged through shared memory
// with cp.async (16-byte chunks, fully coalesced): as soon as a group's values sit in registers,
// the copy of the next group is issued, so it lands while the current group is transformed.
#include "regfft.cuh"
#include "solver.cuh"
#include "tma.cuh"

namespace bastr {

// Elements per thread per unit: 64 bytes of data per unit per thread in both precisions.
#ifndef BASTR_EPT_F32
#define BASTR_EPT_F32 16
#endif
#ifndef BASTR_EPT_F64
#define BASTR_EPT_F64 8
#endif
// Minimum resident blocks per SM asked of the register allocator for the 2D passes.
#ifndef BASTR_MINB_2D
#define BASTR_MINB_2D 1
#endif
template <typename T> struct EptOf { static constexpr int v = sizeof(T) == 8 ? BASTR_EPT_F64 : BASTR_EPT_F32; };
// The forward y pass (two units, FP64 epilogue) runs best with more, lighter threads.
#ifndef BASTR_EPT_YFWD_F32
#define BASTR_EPT_YFWD_F32 8
#endif
// The inverse y pass (the step's first pass, from the FP64 state) runs best at 8 points per
// thread since its lines are TMA-staged: 2048^2 FP32 k2d_yinv_rhs_vg 49.6 -> 43.5 us (16: 248
// registers, 8: 117-128 and twice the threads).
#ifndef BASTR_EPT_YINV_F32
#define BASTR_EPT_YINV_F32 8
#endif
#ifndef BASTR_MINB_YINV
#define BASTR_MINB_YINV 0
#endif
// Modes per thread whose state the fused y pass fetches together (its registers also hold the
// next stage input).
#ifndef BASTR_EPI_CHUNK_YFI
#define BASTR_EPI_CHUNK_YFI 2
#endif
#ifndef BASTR_MINB_YFI
#define BASTR_MINB_YFI 2
#endif
#ifndef BASTR_MINB_XPASS
#define BASTR_MINB_XPASS 0
#endif
#ifndef BASTR_XPASS_TW_SMEM
#define BASTR_XPASS_TW_SMEM 1
#endif
#ifndef BASTR_XPASS_ROWS
#define BASTR_XPASS_ROWS 0
#endif
#ifndef BASTR_EPT_XPASS_F32
#define BASTR_EPT_XPASS_F32 16
#endif
#ifndef BASTR_XPASS_ZA
#define BASTR_XPASS_ZA 3
#endif
// Blocks per SM asked of the register allocator: two once an FP32 block has 256 threads.
template <typename T, int NT> constexpr int minb_for() { return sizeof(T) == 4 && NT >= 256 ? 2 : BASTR_MINB_2D; }
template <int N, int EPT> constexpr int ept_fit() { return N < EPT ? N : EPT; }
// Lines handled by one block: at least 128 threads per block.
template <int NTR> constexpr int groups_per_block() { return NTR >= 128 ? 1 : 128 / NTR; }

// Two adjacent complex values as one vector store.
template <typename T> __device__ __forceinline__ void st2(cplx<T>* dst, cplx<T> a, cplx<T> b) {
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(dst) = make_float4(a.x, a.y, b.x, b.y);
    } else {
        dst[0] = a;
        dst[1] = b;
    }
}

// Two adjacent complex values (16-byte aligned in FP32) as one vector load: half the load
// instructions, and a warp's 16-byte loads of consecutive pairs fill every bank once.
template <typename T> __device__ __forceinline__ void ld2(const cplx<T>* src, cplx<T>& a, cplx<T>& b) {
    if constexpr (sizeof(T) == 4) {
        const float4 q = *reinterpret_cast<const float4*>(src);
        a = make_float2(q.x, q.y);
        b = make_float2(q.z, q.w);
    } else {
        a = src[0];
        b = src[1];
    }
}

// ---------------------------------------------------------------------------------------
// Pass A: inverse transforms along y of kx columns.
// ---------------------------------------------------------------------------------------
// Field sets: the state (u1, u2), the product's fields (g1, h1, g2, h2), the velocity-gradient
// fields (q1, q2 = ky^2 u^), or both of the last two from one read of the column (YI_RHS_VG).
enum YInvSet : int { YI_STATE = 0, YI_RHS = 1, YI_VG = 2, YI_RHS_VG = 3 };

template <typename T, typename TIN, int NY, int SET> struct YInv2D {
    static constexpr int F = SET == YI_STATE ? 2 : SET == YI_RHS ? 4 : SET == YI_VG ? 2 : 6;   // fields produced
    static constexpr int F0 = SET == YI_VG ? 4 : 0;                                             // offset in MA
    static constexpr int UG = 2;                                             // units per sub-pass
    static constexpr int NG = (F + UG - 1) / UG;
    static constexpr int EPT = ept_fit<NY, sizeof(T) == 8 ? EptOf<T>::v : BASTR_EPT_YINV_F32>();
    using FFT = RegFFT<T, NY, EPT, UG, true>;
    static constexpr int G = groups_per_block<FFT::NTR>();
    static constexpr int NT = G * FFT::NTR;
    static constexpr int MINB = (BASTR_MINB_YINV > 0 && sizeof(T) == 4) ? BASTR_MINB_YINV : minb_for<T, NT>();
    static constexpr size_t XCH = (size_t)G * FFT::SMEM_ELEMS * sizeof(cplx<T>);
    // staging of G columns of KY modes x 2 components, sized at run time
    __host__ __device__ static size_t stage_bytes(int KY) {
        return ((size_t)G * KY * 2 * sizeof(cplx<TIN>) + 15) & ~(size_t)15;
    }
    static constexpr size_t TWB = tw_stage_bytes<T, FFT>();
    static size_t smem(int KY) { return stage_bytes(KY) + XCH + TWB; }
    // one column per block: staged by one bulk copy (TMA, contiguous run) on an mbarrier
    static constexpr bool TMA = G == 1;
};

template <typename T, typename TIN, int NY, int SET>
__global__ void __launch_bounds__(YInv2D<T, TIN, NY, SET>::NT, YInv2D<T, TIN, NY, SET>::MINB)
k2d_yinv(const cplx<TIN>* __restrict__ S, cplx<T>* __restrict__ MA, int ftot, Geo g,
         const cplx<T>* tw) {
    using P = YInv2D<T, TIN, NY, SET>;
    using FFT = typename P::FFT;
    constexpr int EPT = P::EPT, UG = P::UG, F = P::F, G = P::G;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<TIN>* stg = reinterpret_cast<cplx<TIN>*>(smraw);
    const int gi = threadIdx.x / FFT::NTR, t = threadIdx.x % FFT::NTR;
    const int K = g.K, KY = g.KY;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw + P::stage_bytes(KY)) + gi * FFT::SMEM_ELEMS;
    constexpr bool STW = P::TWB > 0;   // twiddles by stage in shared memory
    if constexpr (STW) {
        cplx<T>* d = reinterpret_cast<cplx<T>*>(smraw + P::stage_bytes(KY) + P::XCH);
        FFT::fill_stage_twiddles(d, tw);
        tw = d;
    }
    pdl_wait();
    if (halted(g)) return;
    const int nitems = (K + G - 1) / G;
    const int colbytes = KY * 2 * (int)sizeof(cplx<TIN>);   // a multiple of 16
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
        const int kx0 = item * G;
        const int ncol = min(G, K - kx0);
        if constexpr (P::TMA) {
            if (threadIdx.x == 0) {
                mbar_expect_tx(&bar, (uint32_t)colbytes);
                bulk_load(stg, S + (size_t)kx0 * KY * 2, (uint32_t)colbytes, &bar);
            }
        } else {
            stage_line(stg, S + (size_t)kx0 * KY * 2, ncol * colbytes, g);
            cp_async_commit();
        }
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
        const cplx<TIN>* col = stg + (size_t)gi * KY * 2;
        const int kx = item * G + gi;
        const bool valid = kx < K;
        // the column's two components, in the register order of the first transform stage
        cplx<T> ra[EPT], rb[EPT];
#pragma unroll
        for (int e = 0; e < EPT; ++e) {
            const int kyi = pos_trunc(FFT::in_pos(t, e), K, KY, NY);
            const bool on = valid && kyi >= 0;
            ra[e] = on ? cvt<cplx<TIN>, cplx<T>>(col[2 * kyi]) : mk<T>(0, 0);
            rb[e] = on ? cvt<cplx<TIN>, cplx<T>>(col[2 * kyi + 1]) : mk<T>(0, 0);
        }
        __syncthreads();   // the staging buffer is free: fetch the next column group now
        if (item + (int)gridDim.x < nitems) issue(item + gridDim.x);
#pragma unroll
        for (int grp = 0; grp < P::NG; ++grp) {
            cplx<T> v[UG * EPT];
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                const int kyi = pos_trunc(FFT::in_pos(t, e), K, KY, NY);
                const T ky = (T)(kyi >= 0 ? trunc_k(kyi, K, KY) : 0);
                const cplx<T> a = ra[e], b = rb[e];
                cplx<T> f[8];
                if constexpr (SET == YI_STATE) {
                    f[0] = a; f[1] = b; f[2] = f[3] = mk<T>(0, 0);
                } else if constexpr (SET == YI_RHS || SET == YI_RHS_VG) {
                    f[0] = a; f[1] = cscale<T>(cmuli<T>(a), ky);
                    f[2] = b; f[3] = cscale<T>(cmuli<T>(b), ky);
                }
                if constexpr (SET == YI_VG || SET == YI_RHS_VG) {
                    // ky^2 u^: the x pass forms lap(u) = -(kx^2 u^ + this) per point
                    constexpr int o = SET == YI_VG ? 0 : 4;
                    const T ky2 = ky * ky;
                    f[o + 0] = cscale<T>(a, ky2);
                    f[o + 1] = cscale<T>(b, ky2);
                }
#pragma unroll
                for (int u = 0; u < UG; ++u) v[u * EPT + e] = f[grp * UG + u];
            }
            FFT::template run<STW>(v, sm, tw, t);
            if (valid) {
                // record width W = min(4, ftot) fields: MA[kx][group][y][W]
                const int W = ftot < 4 ? ftot : 4;
                const int f0 = P::F0 + grp * UG;
                cplx<T>* dst = MA + ((size_t)kx * (ftot / W) + f0 / W) * NY * W + (f0 % W);
#pragma unroll
                for (int e = 0; e < EPT; ++e) {
                    const int y = FFT::out_pos(t, e);
                    st2<T>(BASTR_CHK(dst + (size_t)y * W, 2 * sizeof(cplx<T>), g), v[e],
                           grp * UG + 1 < F ? v[EPT + e] : mk<T>(0, 0));
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
// Pass B: x transforms of whole rows, with the advective product in registers.
// ---------------------------------------------------------------------------------------
enum XMode : int { XM_RHS = 1, XM_RHS_VG = 2, XM_TO_PHYS = 3, XM_FROM_PHYS = 4 };

template <typename T, int NX, int MODE> struct XPass2D {
    static constexpr int ZU = MODE == XM_RHS ? 3 : MODE == XM_RHS_VG ? 4 : 1;   // units per row
    // fields in the staged records (records of 4), and how many of them are read
    static constexpr int FIN = MODE == XM_RHS ? 4 : MODE == XM_RHS_VG ? 8 : MODE == XM_TO_PHYS ? 2 : 0;
    static constexpr int FLIVE = MODE == XM_RHS_VG ? 6 : FIN;
    static constexpr int EPT = ept_fit<NX, sizeof(T) == 8 ? EptOf<T>::v : BASTR_EPT_XPASS_F32>();
    // at most BASTR_XPASS_ZA units share one shared-memory exchange; more run as a second transform
    static constexpr int ZA = ZU > BASTR_XPASS_ZA ? BASTR_XPASS_ZA : ZU, ZB = ZU - ZA;
    // the second transform runs through the exchange buffer sized for the first
    static_assert(ZB <= ZA, "BASTR_XPASS_ZA: the remaining units must fit the exchange of the first transform");
    using IFFT = RegFFT<T, NX, EPT, ZA, true>;
    using IFFTB = RegFFT<T, NX, EPT, (ZB > 0 ? ZB : 1), true>;
    using FFFT = RegFFT<T, NX, EPT, 1, false>;
    static constexpr int NTR = IFFT::NTR;
    // rows per block: enough for 128 threads, and BASTR_XPASS_ROWS rows so that the gathered
    // (kx, pair) pieces of consecutive rows fill whole 32-byte sectors
    static constexpr int G0 = groups_per_block<NTR>();
    static constexpr int SR = BASTR_XPASS_ROWS ? 32 / (2 * (int)sizeof(cplx<T>)) : 1;
    static constexpr int G = (MODE != XM_FROM_PHYS && G0 < SR) ? SR : G0;
    static constexpr int NT = G * NTR;
    static constexpr int MINB = G > G0 ? 1 : (BASTR_MINB_XPASS > 0 && sizeof(T) == 4 && MODE == XM_RHS) ? BASTR_MINB_XPASS : minb_for<T, NT>();
    static constexpr int KMAX = NX / 3;
    // one staged group: G rows of K*FIN mixed values, or G rows of 2 physical components.  The
    // threads of a warp read consecutive wavenumbers, so the staged run of one wavenumber is an
    // odd number of 16-byte units long (padded if need be): a multiple of 32 bytes would put the
    // threads' addresses a multiple of the bank width apart (4- to 8-way conflicts).  With one
    // row per block the dead tail of the last record (fields past FLIVE) is not staged.
    static constexpr int KBASE = (FLIVE < FIN && G == 1) ? FLIVE : FIN * G;
    static constexpr int KPAD = (KBASE * (int)sizeof(cplx<T>) / 16) % 2 == 0 ? 16 / (int)sizeof(cplx<T>) : 0;
    static constexpr int KSTR = KBASE + KPAD;                                // elements per kx
    // TMA staging (one row per block, the product modes): tile A holds the records of the four
    // fields (g1, h1, g2, h2) of every kx, RB bytes each, swizzled at RB bytes so that the threads
    // of a warp (consecutive kx) read their 16-byte pieces from distinct banks; with velocity-
    // gradient fields, tile B holds the (q1, q2) pieces (QB bytes each).  Boxes of BK records.
    static constexpr bool TMA = G == 1 && (MODE == XM_RHS || MODE == XM_RHS_VG);
    static constexpr int RB = 4 * (int)sizeof(cplx<T>);
    static constexpr int QB = 2 * (int)sizeof(cplx<T>);
    static constexpr int SWZA = RB;                     // 32-byte (FP32) or 64-byte (FP64) swizzle
    static constexpr int SWZB = QB == 32 ? 32 : 0;      // FP64 q pieces: 32-byte swizzle
    static constexpr int BK = KMAX < 256 ? KMAX : 256;
    static constexpr int NBOX = (KMAX + BK - 1) / BK;
    static constexpr size_t TILEA = ((size_t)NBOX * BK * RB + 1023) & ~(size_t)1023;
    static constexpr size_t TILEB = MODE == XM_RHS_VG ? (((size_t)NBOX * BK * QB + 1023) & ~(size_t)1023) : 0;
    static constexpr uint32_t TX_BYTES = (uint32_t)(NBOX * BK * (RB + (MODE == XM_RHS_VG ? QB : 0)));
    static constexpr size_t STAGE = TMA ? 1024 + TILEA + TILEB   // 1024: alignment of the tiles
                                  : MODE == XM_FROM_PHYS ? (size_t)G * 2 * NX * sizeof(double)
                                                         : (size_t)KMAX * KSTR * sizeof(cplx<T>);
    static constexpr size_t XCH = (size_t)G * IFFT::SMEM_ELEMS * sizeof(cplx<T>);
    static constexpr size_t XCHR = XCH > (size_t)9 * NT * 8 ? XCH : (size_t)9 * NT * 8;
    static constexpr size_t TWB = BASTR_XPASS_TW_SMEM ? tw_stage_bytes<T, IFFT, FFFT>() : 0;
    static constexpr size_t SMEM = STAGE + XCHR + TWB;
};

// 16-byte chunk c of kx record k of a swizzled TMA tile (RB-byte records).
template <int SWZ, int RB, typename V>
__device__ __forceinline__ V tile_chunk(const unsigned char* tile, int k, int c) {
    return *reinterpret_cast<const V*>(tile + swz<SWZ>((uint32_t)(k * RB + c * 16)));
}

// Packs the half-spectrum values A, B of wavenumber k (0 <= k < K) for one position of a
// length-NX sequence whose inverse transform is a + i b.  `mirror` selects the position NX-k
// (conjugate side); the imaginary parts of the kx = 0 bin are dropped as dreal() does.
template <typename T>
__device__ __forceinline__ cplx<T> pack_at(cplx<T> A, cplx<T> B, bool mirror, bool zero_bin) {
    if (zero_bin) return mk<T>(A.x, B.x);
    return mirror ? mk<T>(A.x + B.y, B.x - A.y) : mk<T>(A.x - B.y, A.y + B.x);
}

template <typename T, int NX, int MODE>
__global__ void __launch_bounds__(XPass2D<T, NX, MODE>::NT, XPass2D<T, NX, MODE>::MINB)
k2d_xpass(const cplx<T>* __restrict__ MA, int ftot, cplx<T>* __restrict__ MB,
          const double* __restrict__ phys_in, double* __restrict__ phys_out,
          double* __restrict__ vg_part, Geo g, const cplx<T>* tw,
          const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB) {
    using P = XPass2D<T, NX, MODE>;
    using IFFT = typename P::IFFT;
    using FFFT = typename P::FFFT;
    constexpr int ZU = P::ZU, EPT = P::EPT, NT = P::NT, NTR = P::NTR, G = P::G, FIN = P::FIN;
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* stg = smraw;
    // TMA tiles start at the first 1024-byte boundary of the staging area
    unsigned char* tileA = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    unsigned char* tileB = tileA + P::TILEA;
    __shared__ __align__(8) uint64_t bar;
    const int gi = threadIdx.x / NTR, t = threadIdx.x % NTR;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw + P::STAGE) + gi * IFFT::SMEM_ELEMS;
    // twiddles by stage in shared memory: the inverse plan (shared by IFFT and IFFTB), then the forward one
    constexpr bool STW = P::TWB > 0;
    static_assert(P::IFFTB::TWS_ELEMS == IFFT::TWS_ELEMS, "one inverse plan");
    const cplx<T>* twi = tw;
    const cplx<T>* twf = tw;
    if constexpr (STW) {
        cplx<T>* d = reinterpret_cast<cplx<T>*>(smraw + P::STAGE + P::XCHR);
        IFFT::fill_stage_twiddles(d, tw);
        FFFT::fill_stage_twiddles(d + IFFT::TWS_ELEMS, tw);
        twi = d;
        twf = d + IFFT::TWS_ELEMS;
    }
    pdl_wait();
    if (halted(g)) return;
    const int K = g.K, NY = g.ny;
    const int nitems = (NY + G - 1) / G;
    if constexpr (P::TMA) {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
    }
    uint32_t phase = 0;
    auto issue = [&](int item) {
        const int y0 = item * G;
        const int nrow = min(G, NY - y0);
        if constexpr (P::TMA) {
            // one thread: the records of row y0 for every kx, as NBOX boxes of BK wavenumbers
            (void)nrow;
            if (threadIdx.x == 0) {
                mbar_expect_tx(&bar, P::TX_BYTES);
#pragma unroll
                for (int b = 0; b < P::NBOX; ++b) {
                    tma_load_4d(tileA + (size_t)b * P::BK * P::RB, &tmA, 0, y0, 0, b * P::BK, &bar);
                    if constexpr (MODE == XM_RHS_VG)
                        tma_load_4d(tileB + (size_t)b * P::BK * P::QB, &tmB, 0, y0, 1, b * P::BK, &bar);
                }
            }
            return;
        } else if constexpr (MODE == XM_FROM_PHYS) {
            double* d = reinterpret_cast<double*>(stg);
            stage_line(d, phys_in + (size_t)y0 * NX, nrow * NX * 8, g);
            stage_line(d + G * NX, phys_in + (size_t)NY * NX + (size_t)y0 * NX, nrow * NX * 8, g);
        } else {
            // rows y0.. of every (kx, pair) -> staging [kx][pair][row][W], KSTR elements per kx
            constexpr int W = FIN < 4 ? FIN : 4;
            constexpr int NPIN = FIN / W, C16 = W * (int)sizeof(cplx<T>) / 16;
            const int total = K * NPIN * G * C16;
            for (int i = threadIdx.x; i < total; i += NT) {
                const int q = i / C16, c = i - q * C16;
                const int kp = q / G, r = q - kp * G;
                const int k = kp / NPIN, pr = kp - k * NPIN;
                // chunks holding only fields past FLIVE are never read
                if (r < nrow && pr * W + c * (16 / (int)sizeof(cplx<T>)) < P::FLIVE) {
                    cp_async16(stg + (size_t)k * P::KSTR * sizeof(cplx<T>) + (size_t)((pr * G + r) * C16 + c) * 16,
                               BASTR_CHK(MA + (((size_t)k * (ftot / W) + pr) * NY + y0 + r) * W +
                                             c * (16 / (int)sizeof(cplx<T>)), 16, g));
                }
            }
        }
        cp_async_commit();
    };
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double divmax = 0.0;
    int item = blockIdx.x;
    if (item < nitems) issue(item);
    bool lost = false;   // a TMA completion wait gave up (recorded in g.err)
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
        const int y = item * G + gi;
        const bool valid = y < NY;
        cplx<T> v[ZU * EPT];
        if constexpr (MODE == XM_FROM_PHYS) {
            const double* row = reinterpret_cast<const double*>(stg) + (size_t)gi * NX;
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                const int x = FFFT::in_pos(t, e);
                v[e] = valid ? mk<T>((T)row[x], (T)row[G * NX + x]) : mk<T>(0, 0);
            }
        } else {
            constexpr int W = FIN < 4 ? FIN : 4;
            const cplx<T>* row = reinterpret_cast<const cplx<T>*>(stg) + (size_t)gi * W;
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                const int p = IFFT::in_pos(t, e);
                const bool lo = p < K, hi = p > NX - K;
                const int k = lo ? p : NX - p;
#pragma unroll
                for (int u = 0; u < ZU; ++u) v[u * EPT + e] = mk<T>(0, 0);
                // K = floor(NX/3) in 2D: these elements are dealiased zeros for every thread
                if (IFFT::in_band(e, NX / 3 + 1)) continue;
                if (valid && (lo || hi)) {
                    // field f of this wavenumber at src0[(f / W) * G * W + f % W]: pairs (0,1), (2,3),
                    // (4,5) are adjacent and 16-byte aligned
                    const cplx<T>* src0 = row + (size_t)k * P::KSTR;
                    const bool z0 = p == 0;
                    cplx<T> g1, h1;
                    if constexpr (P::TMA) {
                        if constexpr (sizeof(T) == 4) {
                            const float4 q = tile_chunk<P::SWZA, P::RB, float4>(tileA, k, 0);
                            g1 = mk<T>(q.x, q.y);
                            h1 = mk<T>(q.z, q.w);
                        } else {
                            g1 = tile_chunk<P::SWZA, P::RB, cplx<T>>(tileA, k, 0);
                            h1 = tile_chunk<P::SWZA, P::RB, cplx<T>>(tileA, k, 1);
                        }
                    } else {
                        ld2<T>(src0, g1, h1);
                    }
                    if constexpr (MODE == XM_TO_PHYS) {
                        v[e] = pack_at<T>(g1, h1, hi, z0);
                    } else {
                        cplx<T> g2, h2;
                        if constexpr (P::TMA) {
                            if constexpr (sizeof(T) == 4) {
                                const float4 q = tile_chunk<P::SWZA, P::RB, float4>(tileA, k, 1);
                                g2 = mk<T>(q.x, q.y);
                                h2 = mk<T>(q.z, q.w);
                            } else {
                                g2 = tile_chunk<P::SWZA, P::RB, cplx<T>>(tileA, k, 2);
                                h2 = tile_chunk<P::SWZA, P::RB, cplx<T>>(tileA, k, 3);
                            }
                        } else {
                            ld2<T>(src0 + 2, g2, h2);
                        }
                        const T kx = (T)k;
                        v[e] = pack_at<T>(g1, g2, hi, z0);
                        v[EPT + e] = pack_at<T>(cscale<T>(cmuli<T>(g1), kx), cscale<T>(cmuli<T>(g2), kx), hi, z0);
                        v[2 * EPT + e] = pack_at<T>(h1, h2, hi, z0);
                        if constexpr (MODE == XM_RHS_VG) {
                            cplx<T> q1, q2;
                            if constexpr (P::TMA) {
                                if constexpr (sizeof(T) == 4) {
                                    const float4 q = tile_chunk<P::SWZB, P::QB, float4>(tileB, k, 0);
                                    q1 = mk<T>(q.x, q.y);
                                    q2 = mk<T>(q.z, q.w);
                                } else {
                                    q1 = tile_chunk<P::SWZB, P::QB, cplx<T>>(tileB, k, 0);
                                    q2 = tile_chunk<P::SWZB, P::QB, cplx<T>>(tileB, k, 1);
                                }
                            } else {
                                ld2<T>(src0 + G * W, q1, q2);
                            }
                            const T kx2 = kx * kx;
                            v[3 * EPT + e] = pack_at<T>(csub<T>(cscale<T>(g1, -kx2), q1),
                                                        csub<T>(cscale<T>(g2, -kx2), q2), hi, z0);
                        }
                    }
                }
            }
        }
        __syncthreads();   // the staging buffer is free: fetch the next row group now
        if (item + (int)gridDim.x < nitems) issue(item + gridDim.x);
        if constexpr (MODE != XM_FROM_PHYS) {
            IFFT::template run<STW>(v, sm, twi, t);
            if constexpr (P::ZB > 0) P::IFFTB::template run<STW>(v + P::ZA * EPT, sm, twi, t);
        }

        if constexpr (MODE == XM_TO_PHYS) {
            if (valid) {
#pragma unroll
                for (int e = 0; e < EPT; ++e) {
                    const int x = IFFT::out_pos(t, e);
                    const size_t o = (size_t)y * NX + x;
                    BASTR_AT(phys_out, o, g) = (double)v[e].x;
                    BASTR_AT(phys_out, (size_t)NY * NX + o, g) = (double)v[e].y;
                }
            }
        } else {
            if constexpr (MODE == XM_RHS || MODE == XM_RHS_VG) {
                // advective product (solution.F90:841-846) at the points this thread holds; the
                // viscous term is added spectrally in pass C
                const double nu = g.nu;
#pragma unroll
                for (int e = 0; e < EPT; ++e) {
                    const cplx<T> a = v[e], b = v[EPT + e], c = v[2 * EPT + e];
                    const T u1 = a.x, u2 = a.y, u1x = b.x, u2x = b.y, u1y = c.x, u2y = c.y;
                    const T n1 = -u1 * u1x - u2 * u1y;
                    const T n2 = -u1 * u2x - u2 * u2y;
                    v[e] = mk<T>(n1, n2);
                    if constexpr (MODE == XM_RHS_VG) {
                        if (valid) {
                            // velgrad_calculate2D (solution.F90:1149-1166): per-point terms in the
                            // compute precision, sums in FP64; eta_min = sqrt(nu/max|theta|) is
                            // formed once from the largest |theta| (the map is monotone).
                            // dissp = <2 u_i theta lap(u_i) + |u|^2 lap(theta)>, with the second
                            // mean taken as <theta lap(|u|^2)> = <theta (2 u_i lap(u_i) +
                            // 2 |grad u_i|^2)>: equal on the grid (every product has degree
                            // 3(K-1) < n per axis, so grid means are exact and integration by
                            // parts holds), and it needs no lap(theta) field
                            const cplx<T> l = v[3 * EPT + e];
                            const T nuT = (T)nu;
                            const T div = u1x + u2y;
                            const T uu = u1 * u1 + u2 * u2;
                            const T gg = u1x * u1x + u1y * u1y + u2x * u2x + u2y * u2y;
                            acc[0] += (double)(div * div * uu);
                            acc[1] += (double)((u1x * u1x + u2y * u2y + (T)2 * u1y * u2x) * uu);
                            acc[2] += (double)(div * uu);
                            acc[3] += (double)(div * ((T)4 * (u1 * l.x + u2 * l.y) + (T)2 * gg));
                            acc[4] += (double)(nuT * (u1y - u2x) * (u1y - u2x) + nuT * div * div);
                            divmax = fmax(divmax, (double)fabs(div));
                            acc[5] += (double)uu;
                            acc[6] += (double)(u1x * u1x + u2y * u2y);
                        }
                    }
                }
            }
            // forward transform of the packed product (or of the packed physical fields)
            FFFT::template run<STW>(v, sm, twf, t);
            // split the packed spectrum into the two half spectra, kx in [0,K): Z[k] and Z[NX-k]
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                // outputs strictly between K-1 and NX-K+1 are never read by the split below
                if (MODE != XM_FROM_PHYS && FFFT::out_band(e, NX / 3 + 1)) continue;
                sm[pidx(FFFT::out_pos(t, e))] = v[e];
            }
            __syncthreads();
            if (valid) {
                for (int k = t; k < K; k += NTR) {
                    const cplx<T> Z = sm[pidx(k)];
                    const cplx<T> Zc = cconj<T>(sm[pidx(k == 0 ? 0 : NX - k)]);
                    st2<T>(BASTR_CHK(MB + (((size_t)(y >> 1) * K + k) * 2 + (y & 1)) * 2, 2 * sizeof(cplx<T>), g),
                           cscale<T>(cadd<T>(Z, Zc), (T)0.5), cscale<T>(cmulni<T>(csub<T>(Z, Zc)), (T)0.5));
                }
            }
        }
    }
    cp_async_wait<0>();
    if constexpr (P::TMA) {
        if (lost && threadIdx.x == 0) mbar_wait(&bar, phase, nullptr);   // bounded drain
    }
    (void)lost;
    if constexpr (MODE == XM_RHS_VG) {
        __syncthreads();
        double* scratch = reinterpret_cast<double*>(smraw + P::STAGE);
        block_sum<7, NT>(acc, scratch);
        const double dm = -block_min<NT>(-divmax, scratch);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int i = 0; i < 7; ++i) BASTR_AT(vg_part, (size_t)blockIdx.x * 8 + i, g) = acc[i];
            BASTR_AT(vg_part, (size_t)blockIdx.x * 8 + 7, g) = dm;
        }
    }
}

// Prefetch of the state a line's epilogue will read (the u0, us and acc values of modes
// first .. first + n - 1 of each of D components cst elements apart; 2D: interleaved, cst = 1
// and 2n values), issued before the line's forward transform so that the loads after it find
// the lines in L2: 0 none, 1 into L1, 2 into L2 with the evict-last priority (the default; 2048^2
// FP32: 0.372 -> 0.367 ms per step, L1 0.368).
#ifndef BASTR_EPI_PREFETCH
#define BASTR_EPI_PREFETCH 2
#endif
template <typename T, int D, int EPI>
__device__ __forceinline__ void epi_prefetch(const StageIO<T>& io, size_t first, int n, size_t cst, bool from_u0,
                                             int t, int nthreads) {
    if constexpr (BASTR_EPI_PREFETCH != 0 && EPI != EPI_STORE) {
        auto pf = [&](const void* base, size_t bytes) {
            for (size_t off = (size_t)t * 128; off < bytes; off += (size_t)nthreads * 128) {
                const char* a = static_cast<const char*>(base) + off;
                if constexpr (BASTR_EPI_PREFETCH == 1) asm volatile("prefetch.global.L1 [%0];" ::"l"(a));
                else asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(a));
            }
        };
        const int runs = D == 2 ? 1 : D;                       // 2D: one interleaved run
        const size_t len = D == 2 ? (size_t)n * 2 : (size_t)n;
#pragma unroll
        for (int c = 0; c < runs; ++c) {
            pf(io.u0 + first + c * cst, len * sizeof(double2));
            if (!from_u0 && EPI != EPI_RK2) pf(io.us + first + c * cst, len * sizeof(cplx<T>));
            if constexpr (EPI == EPI_RK2 || EPI == EPI_RK3) pf(io.acc + first + c * cst, len * sizeof(cplx<T>));
        }
    }
}

// ---------------------------------------------------------------------------------------
// Pass C: forward transforms along y of kx columns + spectral epilogue.
// ---------------------------------------------------------------------------------------
// TMA staging of the forward y passes (one kx column per block): the column's records of two
// rows [y/2][2 rows][2 comps] (RB bytes) for every row pair, as NBOX boxes of BY row pairs.  The
// FP64 records are swizzled at 64 bytes so that the threads of a warp (consecutive y) read their
// 16-byte pieces from distinct banks; the FP32 ones are read as consecutive 16-byte pieces.
template <typename T, int NY, int G> struct YStage2D {
    static constexpr bool TMA = G == 1;
    static constexpr int RB = 4 * (int)sizeof(cplx<T>);
    static constexpr int SWZ = RB == 64 ? 64 : 0;
    static constexpr int NP = NY / 2;
    static constexpr int BY = NP < 256 ? NP : 256;
    static constexpr int NBOX = NP / BY;
    static constexpr uint32_t TX_BYTES = (uint32_t)(NP * RB);
    static constexpr size_t BYTES = 1024 + (((size_t)NP * RB + 1023) & ~(size_t)1023);
    // the two components of row y
    __device__ static __forceinline__ void load(const unsigned char* tile, int y, cplx<T>& a, cplx<T>& b) {
        if constexpr (sizeof(T) == 4) {
            const float4 q = *reinterpret_cast<const float4*>(tile + (size_t)y * 16);
            a = mk<T>(q.x, q.y);
            b = mk<T>(q.z, q.w);
        } else {
            a = *reinterpret_cast<const cplx<T>*>(tile + swz<SWZ>((uint32_t)y * 32));
            b = *reinterpret_cast<const cplx<T>*>(tile + swz<SWZ>((uint32_t)y * 32 + 16));
        }
    }
    // one thread: column kx of every row pair
    __device__ static __forceinline__ void issue(unsigned char* tile, const CUtensorMap* map, int kx, uint64_t* bar) {
        mbar_expect_tx(bar, TX_BYTES);
#pragma unroll
        for (int b = 0; b < NBOX; ++b) tma_load_3d(tile + (size_t)b * BY * RB, map, 0, kx, b * BY, bar);
    }
};

template <typename T, int NY> struct YFwd2D {
    static constexpr int EPT = ept_fit<NY, sizeof(T) == 8 ? EptOf<T>::v : BASTR_EPT_YFWD_F32>();
    using FFT = RegFFT<T, NY, EPT, 2, false>;
    static constexpr int G = groups_per_block<FFT::NTR>();
    static constexpr int NT = G * FFT::NTR;
    static constexpr int MINB = NT >= 256 ? 2 : 1;
    using YS = YStage2D<T, NY, G>;
    static constexpr size_t STAGE = YS::TMA ? YS::BYTES : (size_t)G * NY * 2 * sizeof(cplx<T>);
    static constexpr size_t XCH = (size_t)G * FFT::SMEM_ELEMS * sizeof(cplx<T>);
    static constexpr size_t XCHR = XCH > (size_t)NT * 8 ? XCH : (size_t)NT * 8;
    static constexpr size_t TWB = tw_stage_bytes<T, FFT>();
    static constexpr size_t SMEM = STAGE + XCHR + TWB;
};

template <typename T, int NY, int EPI>
__global__ void __launch_bounds__(YFwd2D<T, NY>::NT, YFwd2D<T, NY>::MINB)
k2d_yfwd(const cplx<T>* __restrict__ MB, StageIO<T> io, int input_is_u0, Geo g,
         const cplx<T>* tw, const __grid_constant__ CUtensorMap tmy) {
    using P = YFwd2D<T, NY>;
    using FFT = typename P::FFT;
    constexpr int EPT = P::EPT, NT = P::NT, G = P::G;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* stg = reinterpret_cast<cplx<T>*>(smraw);
    const int gi = threadIdx.x / FFT::NTR, t = threadIdx.x % FFT::NTR;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw + P::STAGE) + gi * FFT::SMEM_ELEMS;
    constexpr bool STW = P::TWB > 0;   // twiddles by stage in shared memory
    if constexpr (STW) {
        cplx<T>* d = reinterpret_cast<cplx<T>*>(smraw + P::STAGE + P::XCHR);
        FFT::fill_stage_twiddles(d, tw);
        tw = d;
    }
    pdl_wait();
    if (halted(g)) return;
    const int K = g.K, KY = g.KY;
    const int nitems = (K + G - 1) / G;
    using YS = typename P::YS;
    unsigned char* tile = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    __shared__ __align__(8) uint64_t bar;
    if constexpr (YS::TMA) {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
    }
    uint32_t phase = 0;
    bool lost = false;   // a TMA completion wait gave up (recorded in g.err)
    // columns kx0.. of every row (records of two rows in MB) -> staging [col][y][c]
    auto issue = [&](int item) {
        if constexpr (YS::TMA) {
            if (threadIdx.x == 0) YS::issue(tile, &tmy, item, &bar);
            return;
        }
        const int kx0 = item * G;
        const int ncol = min(G, K - kx0);
        constexpr int C16 = 2 * (int)sizeof(cplx<T>) / 16;
        const int total = NY * G * C16;
        for (int i = threadIdx.x; i < total; i += NT) {
            const int q = i / C16, c = i - q * C16;
            const int col = q % G, y = q / G;
            if (col < ncol)
                cp_async16(reinterpret_cast<unsigned char*>(stg) + ((size_t)(col * NY + y) * 2 * sizeof(cplx<T>) + c * 16),
                           BASTR_CHK(MB + (((size_t)(y >> 1) * K + kx0 + col) * 2 + (y & 1)) * 2 +
                                         c * (16 / (int)sizeof(cplx<T>)), 16, g));
        }
        cp_async_commit();
    };
    const double inv_n = g.inv_n;
    const long long K2 = (long long)K * K;
    double en = 0.0;
    int item = blockIdx.x;
    if (item < nitems) issue(item);
    for (; item < nitems; item += gridDim.x) {
        if constexpr (YS::TMA) {
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
        const cplx<T>* col = stg + (size_t)gi * NY * 2;
        const int kx = item * G + gi;
        const bool valid = kx < K;
        cplx<T> v[2 * EPT];
#pragma unroll
        for (int e = 0; e < EPT; ++e) {
            const int y = FFT::in_pos(t, e);
            if (!valid) v[e] = v[EPT + e] = mk<T>(0, 0);
            else if constexpr (YS::TMA) YS::load(tile, y, v[e], v[EPT + e]);
            else ld2<T>(col + 2 * y, v[e], v[EPT + e]);
        }
        __syncthreads();   // the staging buffer is free: fetch the next column group now
        if (item + (int)gridDim.x < nitems) issue(item + gridDim.x);
        if (valid) epi_prefetch<T, 2, EPI>(io, (size_t)kx * KY * 2, KY, 1, input_is_u0 != 0, t, FFT::NTR);
        FFT::template run<STW>(v, sm, tw, t);
        if (valid) {
            const double w = kx == 0 ? 1.0 : 2.0;
            const bool from_u0 = input_is_u0 != 0;
            constexpr int CH = EPT < EpiChunk<T, 2>::v ? EPT : EpiChunk<T, 2>::v;
#pragma unroll
            for (int e0 = 0; e0 < EPT; e0 += CH) {
                EpiIn<T, 2> in[CH];
#pragma unroll
                for (int j = 0; j < CH; ++j) {
                    const int kyi = pos_trunc(FFT::out_pos(t, e0 + j), K, KY, NY);
                    if (kyi >= 0) epi_load<T, 2, EPI>(in[j], ((size_t)kx * KY + kyi) * 2, 1, io, from_u0);
                }
#pragma unroll
                for (int j = 0; j < CH; ++j) {
                    const int e = e0 + j;
                    const int kyi = pos_trunc(FFT::out_pos(t, e), K, KY, NY);
                    if (kyi < 0) continue;
                    const int ky = trunc_k(kyi, K, KY);
                    const size_t o = ((size_t)kx * KY + kyi) * 2;
                    const long long m2i = (long long)kx * kx + (long long)ky * ky;
                    double2 vv[2];
                    if (m2i < K2) {   // spherical 2/3 rule, tool.F90:185-193
                        vv[0] = dscale(cvt<cplx<T>, double2>(v[e]), inv_n);
                        vv[1] = dscale(cvt<cplx<T>, double2>(v[EPT + e]), inv_n);
                    } else {
                        vv[0] = make_double2(0, 0);
                        vv[1] = make_double2(0, 0);
                    }
                    const double kv[2] = {(double)kx, (double)ky};
                    rk_apply<T, 2, EPI>(vv, kv, (double)m2i, in[j], o, 1, io, from_u0, g, w, en);
                }
            }
        }
    }
    cp_async_wait<0>();
    if constexpr (YS::TMA) {
        if (lost && threadIdx.x == 0) mbar_wait(&bar, phase, nullptr);   // bounded drain
    }
    (void)lost;
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


// ---------------------------------------------------------------------------------------
// Pass C + A of the next stage: the forward y pass of RK stage 1 or 2 (or a Crank-Nicolson
// sweep before the last) followed, in the same kernel, by the next stage's inverse y
// transforms of the stage input it has just formed.  Both transforms use EPT = 8, so the
// forward transform's output order in registers is the inverse's input order (mirrored
// plans): the new stage input goes from the epilogue into the inverse without a round trip
// through HBM, and one pass and one launch per stage disappear.  MA is written in the same
// [kx][group][y][4] records as pass A (ftot = 4: the stages after the first carry no
// velocity-gradient fields).
// ---------------------------------------------------------------------------------------
template <typename T, int NY> struct YFwdInv2D {
    static constexpr int EPT = ept_fit<NY, 8>();
    using FFT = RegFFT<T, NY, EPT, 2, false>;
    using IFFT = RegFFT<T, NY, EPT, 2, true>;
    static_assert(FFT::RL == IFFT::R0, "forward output order must be the inverse input order");
    static constexpr int G = groups_per_block<FFT::NTR>();
    static constexpr int NT = G * FFT::NTR;
    static constexpr int MINB = (sizeof(T) == 4 && NT >= 256) ? BASTR_MINB_YFI : 1;
    using YS = YStage2D<T, NY, G>;
    static constexpr size_t STAGE = YS::TMA ? YS::BYTES : (size_t)G * NY * 2 * sizeof(cplx<T>);
    static constexpr size_t XCH = (size_t)G * FFT::SMEM_ELEMS * sizeof(cplx<T>);
    static constexpr size_t XCHR = XCH > (size_t)NT * 8 ? XCH : (size_t)NT * 8;
    static constexpr size_t TWB = tw_stage_bytes<T, FFT, IFFT>();
    static constexpr size_t SMEM = STAGE + XCHR + TWB;
};

template <typename T, int NY, int EPI>
__global__ void __launch_bounds__(YFwdInv2D<T, NY>::NT, YFwdInv2D<T, NY>::MINB)
k2d_yfwd_inv(const cplx<T>* __restrict__ MB, StageIO<T> io, int input_is_u0, Geo g, const cplx<T>* tw,
             cplx<T>* __restrict__ MA, const __grid_constant__ CUtensorMap tmy) {
    static_assert(EPI == EPI_RK1 || EPI == EPI_RK2 || EPI == EPI_CN_MID, "stages that hand on a stage input");
    using P = YFwdInv2D<T, NY>;
    using FFT = typename P::FFT;
    using IFFT = typename P::IFFT;
    constexpr int EPT = P::EPT, NT = P::NT, G = P::G;
    constexpr int W = 4, FTOT = 4;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* stg = reinterpret_cast<cplx<T>*>(smraw);
    const int gi = threadIdx.x / FFT::NTR, t = threadIdx.x % FFT::NTR;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw + P::STAGE) + gi * FFT::SMEM_ELEMS;
    // twiddles by stage in shared memory: the forward plan, then the inverse one
    constexpr bool STW = P::TWB > 0;
    const cplx<T>* twf = tw;
    const cplx<T>* twi = tw;
    if constexpr (STW) {
        cplx<T>* d = reinterpret_cast<cplx<T>*>(smraw + P::STAGE + P::XCHR);
        FFT::fill_stage_twiddles(d, tw);
        IFFT::fill_stage_twiddles(d + FFT::TWS_ELEMS, tw);
        twf = d;
        twi = d + FFT::TWS_ELEMS;
    }
    pdl_wait();
    if (halted(g)) return;
    const int K = g.K, KY = g.KY;
    const int nitems = (K + G - 1) / G;
    using YS = typename P::YS;
    unsigned char* tile = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    __shared__ __align__(8) uint64_t bar;
    if constexpr (YS::TMA) {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
    }
    uint32_t phase = 0;
    bool lost = false;   // a TMA completion wait gave up (recorded in g.err)
    // columns kx0.. of every row (records of two rows in MB) -> staging [col][y][c]
    auto issue = [&](int item) {
        if constexpr (YS::TMA) {
            if (threadIdx.x == 0) YS::issue(tile, &tmy, item, &bar);
            return;
        }
        const int kx0 = item * G;
        const int ncol = min(G, K - kx0);
        constexpr int C16 = 2 * (int)sizeof(cplx<T>) / 16;
        const int total = NY * G * C16;
        for (int i = threadIdx.x; i < total; i += NT) {
            const int q = i / C16, c = i - q * C16;
            const int col = q % G, y = q / G;
            if (col < ncol)
                cp_async16(reinterpret_cast<unsigned char*>(stg) + ((size_t)(col * NY + y) * 2 * sizeof(cplx<T>) + c * 16),
                           BASTR_CHK(MB + (((size_t)(y >> 1) * K + kx0 + col) * 2 + (y & 1)) * 2 +
                                         c * (16 / (int)sizeof(cplx<T>)), 16, g));
        }
        cp_async_commit();
    };
    const double inv_n = g.inv_n;
    const long long K2 = (long long)K * K;
    double en = 0.0;
    int item = blockIdx.x;
    if (item < nitems) issue(item);
    for (; item < nitems; item += gridDim.x) {
        if constexpr (YS::TMA) {
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
        const cplx<T>* col = stg + (size_t)gi * NY * 2;
        const int kx = item * G + gi;
        const bool valid = kx < K;
        cplx<T> v[2 * EPT];
#pragma unroll
        for (int e = 0; e < EPT; ++e) {
            const int y = FFT::in_pos(t, e);
            if (!valid) v[e] = v[EPT + e] = mk<T>(0, 0);
            else if constexpr (YS::TMA) YS::load(tile, y, v[e], v[EPT + e]);
            else ld2<T>(col + 2 * y, v[e], v[EPT + e]);
        }
        __syncthreads();   // the staging buffer is free: fetch the next column group now
        if (item + (int)gridDim.x < nitems) issue(item + gridDim.x);
        if (valid) epi_prefetch<T, 2, EPI>(io, (size_t)kx * KY * 2, KY, 1, input_is_u0 != 0, t, FFT::NTR);
        FFT::template run<STW>(v, sm, twf, t);
        // the next stage input at the positions this thread holds (zero outside the kept set)
        cplx<T> nx[2 * EPT];
#pragma unroll
        for (int e = 0; e < 2 * EPT; ++e) nx[e] = mk<T>(0, 0);
        if (valid) {
            const double w = kx == 0 ? 1.0 : 2.0;
            const bool from_u0 = input_is_u0 != 0;
            constexpr int CH = EPT < BASTR_EPI_CHUNK_YFI ? EPT : BASTR_EPI_CHUNK_YFI;
#pragma unroll
            for (int e0 = 0; e0 < EPT; e0 += CH) {
                EpiIn<T, 2> in[CH];
#pragma unroll
                for (int j = 0; j < CH; ++j) {
                    const int kyi = pos_trunc(FFT::out_pos(t, e0 + j), K, KY, NY);
                    if (kyi >= 0) epi_load<T, 2, EPI>(in[j], ((size_t)kx * KY + kyi) * 2, 1, io, from_u0);
                }
#pragma unroll
                for (int j = 0; j < CH; ++j) {
                    const int e = e0 + j;
                    const int kyi = pos_trunc(FFT::out_pos(t, e), K, KY, NY);
                    if (kyi < 0) continue;
                    const int ky = trunc_k(kyi, K, KY);
                    const size_t o = ((size_t)kx * KY + kyi) * 2;
                    const long long m2i = (long long)kx * kx + (long long)ky * ky;
                    double2 vv[2];
                    if (m2i < K2) {   // spherical 2/3 rule, tool.F90:185-193
                        vv[0] = dscale(cvt<cplx<T>, double2>(v[e]), inv_n);
                        vv[1] = dscale(cvt<cplx<T>, double2>(v[EPT + e]), inv_n);
                    } else {
                        vv[0] = make_double2(0, 0);
                        vv[1] = make_double2(0, 0);
                    }
                    const double kv[2] = {(double)kx, (double)ky};
                    cplx<T> nxt[2];
                    rk_apply<T, 2, EPI, true, EPI != EPI_RK1>(vv, kv, (double)m2i, in[j], o, 1, io, from_u0, g, w,
                                                              en, nxt);
                    nx[e] = nxt[0];
                    nx[EPT + e] = nxt[1];
                }
            }
        }
        // next stage, pass A: g_c = IFFT_y(u_c^), h_c = IFFT_y(i ky u_c^), one sub-pass per component
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            cplx<T> u[2 * EPT];
#pragma unroll
            for (int e = 0; e < EPT; ++e) {
                const int kyi = pos_trunc(IFFT::in_pos(t, e), K, KY, NY);
                const T ky = (T)(kyi >= 0 ? trunc_k(kyi, K, KY) : 0);
                u[e] = nx[c * EPT + e];
                u[EPT + e] = cscale<T>(cmuli<T>(nx[c * EPT + e]), ky);
            }
            IFFT::template run<STW>(u, sm, twi, t);
            if (valid) {
                cplx<T>* dst = MA + (size_t)kx * (FTOT / W) * NY * W + 2 * c;
#pragma unroll
                for (int e = 0; e < EPT; ++e)
                    st2<T>(BASTR_CHK(dst + (size_t)IFFT::out_pos(t, e) * W, 2 * sizeof(cplx<T>), g), u[e], u[EPT + e]);
            }
        }
    }
    cp_async_wait<0>();
    if constexpr (YS::TMA) {
        if (lost && threadIdx.x == 0) mbar_wait(&bar, phase, nullptr);   // bounded drain
    }
    (void)lost;
    (void)en;
}

}  // namespace bastr
