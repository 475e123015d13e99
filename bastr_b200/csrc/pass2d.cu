// 2D right-hand side as three fused passes over HBM (the hot path of compute_ut2D,
// solution.F90:816-863, with the RK3/CN combinations of solution.F90:172-231 folded into the
// last pass).
//
//   A  yinv : per kx column, inverse y transforms of the truncated spectrum -> mixed (kx, y)
//             MA[y][kx][f]  f = g1,h1,g2,h2 (+ q1,q2,t when velocity-gradient statistics are due)
//             g = IFFT_y(u^), h = IFFT_y(i ky u^), q = IFFT_y(ky^2 u^), t = IFFT_y(lap(theta)^)
//   B  xpass: per y row, three (five) packed complex inverse x transforms give u, du/dx, du/dy
//             (and lap u, lap theta) in physical space; the advective product
//             N_i = -(u1 d1 u_i + u2 d2 u_i) is formed in registers and packed back into one
//             forward x transform.  Output MB[kx][y][c].
//   C  yfwd : per kx column, forward y transforms, 1/N normalisation, truncation (= the
//             spherical 2/3 dealias, tool.F90:175-194), viscous term -nu k^2 u^, dilatational
//             projection (tool.F90:219-243) and the time-integrator combination.
//
// Two real fields share one complex transform (z = a + i b), so the six real inverse and two
// real forward x transforms of the reference become three plus one complex transforms.
#include "solver.cuh"

namespace bastr {

// ---------------------------------------------------------------------------------------
// Pass A: inverse transforms along y of one kx column.
// ---------------------------------------------------------------------------------------
enum YInvSet : int { YI_STATE = 0, YI_RHS = 1, YI_VG = 2 };

template <typename T, int NY, int SET> struct YInv2D {
    static constexpr int F = SET == YI_STATE ? 2 : SET == YI_RHS ? 4 : 3;   // fields produced
    static constexpr int F0 = SET == YI_VG ? 4 : 0;                          // offset in MA
    static constexpr int US = padded_len(NY);
    static constexpr int NT = pick_threads<T, F * NY>();
    static constexpr size_t SMEM = (size_t)F * US * sizeof(cplx<T>);
};

template <typename T, typename TIN, int NY, int SET>
__global__ void __launch_bounds__(YInv2D<T, NY, SET>::NT)
k2d_yinv(const cplx<TIN>* __restrict__ S, cplx<T>* __restrict__ MA, int ftot, Geo g,
         const cplx<T>* __restrict__ tw) {
    using P = YInv2D<T, NY, SET>;
    constexpr int F = P::F, US = P::US, NT = P::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    const int kx = blockIdx.x;
    const int K = g.K, KY = g.KY;
    const T kxt = (T)kx;
    for (int p = threadIdx.x; p < NY; p += NT) {
        cplx<T> v[F];
#pragma unroll
        for (int f = 0; f < F; ++f) v[f] = mk<T>(0, 0);
        const int kyi = pos_trunc(p, K, KY, NY);
        if (kyi >= 0) {
            const T ky = (T)trunc_k(kyi, K, KY);
            const size_t o = ((size_t)kx * KY + kyi) * 2;
            cplx<T> a = cvt<cplx<TIN>, cplx<T>>(S[o]);
            cplx<T> b = cvt<cplx<TIN>, cplx<T>>(S[o + 1]);
            if constexpr (SET == YI_STATE) {
                v[0] = a;
                v[1] = b;
            } else if constexpr (SET == YI_RHS) {
                v[0] = a;
                v[1] = cscale<T>(cmuli<T>(a), ky);
                v[2] = b;
                v[3] = cscale<T>(cmuli<T>(b), ky);
            } else {
                const T ky2 = ky * ky;
                v[0] = cscale<T>(a, ky2);
                v[1] = cscale<T>(b, ky2);
                // lap(theta)^ = -i |k|^2 (kx u1^ + ky u2^)   (solution.F90:1131)
                const T kk = kxt * kxt + ky2;
                cplx<T> dv = cadd<T>(cscale<T>(a, kxt), cscale<T>(b, ky));
                v[2] = cscale<T>(cmulni<T>(dv), kk);
            }
        }
#pragma unroll
        for (int f = 0; f < F; ++f) sm[f * US + pidx(p)] = v[f];
    }
    __syncthreads();
    fft_run<T, NY, F, US, NT, true>(sm, tw);
    const size_t rowstride = (size_t)K * ftot;
    for (int e = threadIdx.x; e < NY * F; e += NT) {
        const int y = e / F, f = e - y * F;
        MA[(size_t)y * rowstride + (size_t)kx * ftot + P::F0 + f] = sm[f * US + pidx(y)];
    }
}

// ---------------------------------------------------------------------------------------
// Pass B: x transforms of whole rows, with the advective product in between.
// ---------------------------------------------------------------------------------------
enum XMode : int { XM_RHS = 1, XM_RHS_VG = 2, XM_TO_PHYS = 3, XM_FROM_PHYS = 4 };

template <typename T, int NX, int MODE> struct XPass2D {
    static constexpr int ZU = MODE == XM_RHS ? 3 : MODE == XM_RHS_VG ? 5 : 1;   // units per row
    static constexpr int BR = (sizeof(T) == 8 ? 1 : 2) * (ZU == 1 ? 2 : 1);      // rows per block
    static constexpr int U = ZU * BR;
    static constexpr int US = padded_len(NX);
    static constexpr int NT = pick_threads<T, U * NX>();
    static constexpr size_t SMEM_FFT = (size_t)U * US * sizeof(cplx<T>);
    static constexpr size_t SMEM = SMEM_FFT > (size_t)9 * NT * 8 ? SMEM_FFT : (size_t)9 * NT * 8;
};

// Packs two half spectra A, B (kx in [0,K)) into one length-NX complex sequence whose inverse
// transform is a + i b, a and b the real fields.  The imaginary parts of the kx=0 bins are
// dropped, as the reference's dreal() does.
template <typename T>
__device__ __forceinline__ void pack2(cplx<T>* unit, int k, int NX, cplx<T> A, cplx<T> B) {
    if (k == 0) {
        unit[pidx(0)] = mk<T>(A.x, B.x);
    } else {
        unit[pidx(k)] = mk<T>(A.x - B.y, A.y + B.x);
        unit[pidx(NX - k)] = mk<T>(A.x + B.y, B.x - A.y);
    }
}

template <typename T, int NX, int MODE>
__global__ void __launch_bounds__(XPass2D<T, NX, MODE>::NT)
k2d_xpass(const cplx<T>* __restrict__ MA, int ftot, cplx<T>* __restrict__ MB,
          const double* __restrict__ phys_in, double* __restrict__ phys_out,
          double* __restrict__ vg_part, Geo g, const cplx<T>* __restrict__ tw) {
    using P = XPass2D<T, NX, MODE>;
    constexpr int ZU = P::ZU, BR = P::BR, US = P::US, NT = P::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    const int K = g.K, NY = g.ny;
    const int y0 = blockIdx.x * BR;
    const int tid = threadIdx.x;

    if constexpr (MODE == XM_FROM_PHYS) {
        for (int e = tid; e < BR * NX; e += NT) {
            const int r = e / NX, x = e - r * NX;
            const size_t o = (size_t)(y0 + r) * NX + x;
            sm[r * US + pidx(x)] = mk<T>((T)phys_in[o], (T)phys_in[(size_t)NY * NX + o]);
        }
    } else {
        // zero the untouched middle band of every unit
        for (int e = tid; e < BR * ZU * (NX - 2 * K + 1); e += NT) {
            const int u = e / (NX - 2 * K + 1), x = K + (e - u * (NX - 2 * K + 1));
            sm[u * US + pidx(x)] = mk<T>(0, 0);
        }
        for (int e = tid; e < BR * K; e += NT) {
            const int r = e / K, k = e - r * K;
            const cplx<T>* src = MA + ((size_t)(y0 + r) * K + k) * ftot;
            cplx<T>* z = sm + r * ZU * US;
            const cplx<T> g1 = src[0];
            if constexpr (MODE == XM_TO_PHYS) {
                pack2<T>(z, k, NX, g1, src[1]);
            } else {
                const cplx<T> h1 = src[1], g2 = src[2], h2 = src[3];
                const T kx = (T)k;
                pack2<T>(z, k, NX, g1, g2);
                pack2<T>(z + US, k, NX, cscale<T>(cmuli<T>(g1), kx), cscale<T>(cmuli<T>(g2), kx));
                pack2<T>(z + 2 * US, k, NX, h1, h2);
                if constexpr (MODE == XM_RHS_VG) {
                    const cplx<T> q1 = src[4], q2 = src[5], t = src[6];
                    const T kx2 = kx * kx;
                    cplx<T> l1 = csub<T>(cscale<T>(g1, -kx2), q1);
                    cplx<T> l2 = csub<T>(cscale<T>(g2, -kx2), q2);
                    pack2<T>(z + 3 * US, k, NX, l1, l2);
                    pack2<T>(z + 4 * US, k, NX, t, mk<T>(0, 0));
                }
            }
        }
    }
    __syncthreads();

    if constexpr (MODE == XM_FROM_PHYS) {
        fft_run<T, NX, BR, US, NT, false>(sm, tw);
    } else {
        fft_run<T, NX, BR * ZU, US, NT, true>(sm, tw);
    }

    if constexpr (MODE == XM_TO_PHYS) {
        for (int e = tid; e < BR * NX; e += NT) {
            const int r = e / NX, x = e - r * NX;
            const cplx<T> z = sm[r * US + pidx(x)];
            const size_t o = (size_t)(y0 + r) * NX + x;
            phys_out[o] = (double)z.x;
            phys_out[(size_t)NY * NX + o] = (double)z.y;
        }
        return;
    }

    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double etamin = 1.0 / 0.0;
    if constexpr (MODE == XM_RHS || MODE == XM_RHS_VG) {
        // advective product (solution.F90:841-846); the viscous term is added spectrally in pass C
        const double nu = g.nu;
        for (int e = tid; e < BR * NX; e += NT) {
            const int r = e / NX, x = e - r * NX;
            cplx<T>* z = sm + r * ZU * US;
            const cplx<T> a = z[pidx(x)], b = z[US + pidx(x)], c = z[2 * US + pidx(x)];
            const T u1 = a.x, u2 = a.y, u1x = b.x, u2x = b.y, u1y = c.x, u2y = c.y;
            const T n1 = -u1 * u1x - u2 * u1y;
            const T n2 = -u1 * u2x - u2 * u2y;
            z[pidx(x)] = mk<T>(n1, n2);
            if constexpr (MODE == XM_RHS_VG) {
                // velgrad_calculate2D (solution.F90:1149-1166), accumulated in FP64
                const cplx<T> l = z[3 * US + pidx(x)], th = z[4 * US + pidx(x)];
                const double U1 = u1, U2 = u2, D11 = u1x, D22 = u2y, D12 = u1y, D21 = u2x;
                const double div = D11 + D22;
                const double uu = U1 * U1 + U2 * U2;
                acc[0] += div * div * uu;
                acc[1] += (D11 * D11 + D22 * D22 + 2.0 * D12 * D21) * uu;
                acc[2] += div * uu;
                acc[3] += 2.0 * U1 * div * (double)l.x + 2.0 * U2 * div * (double)l.y + uu * (double)th.x;
                acc[4] += nu * (D12 - D21) * (D12 - D21) + nu * div * div;
                etamin = fmin(etamin, sqrt(nu / fabs(div)));
                acc[5] += uu;
                acc[6] += D11 * D11 + D22 * D22;
            }
        }
        __syncthreads();
        fft_run<T, NX, BR, US, NT, false, 1, ZU * US>(sm, tw);
    }

    // split the packed forward transform into the two half spectra, kx in [0,K)
    for (int e = tid; e < BR * K; e += NT) {
        const int r = e / K, k = e - r * K;
        const cplx<T>* z = sm + r * ZU * US;
        const cplx<T> Z = z[pidx(k)];
        const cplx<T> Zc = cconj<T>(z[pidx(k == 0 ? 0 : NX - k)]);
        const cplx<T> A = cscale<T>(cadd<T>(Z, Zc), (T)0.5);
        const cplx<T> B = cscale<T>(cmulni<T>(csub<T>(Z, Zc)), (T)0.5);
        cplx<T>* dst = MB + ((size_t)k * NY + y0 + r) * 2;
        dst[0] = A;
        dst[1] = B;
    }
    if constexpr (MODE == XM_RHS_VG) {
        __syncthreads();
        double* scratch = reinterpret_cast<double*>(smraw);
        block_sum<7, NT>(acc, scratch);
        const double em = block_min<NT>(etamin, scratch);
        if (tid == 0) {
#pragma unroll
            for (int i = 0; i < 7; ++i) vg_part[(size_t)blockIdx.x * 8 + i] = acc[i];
            vg_part[(size_t)blockIdx.x * 8 + 7] = em;
        }
    }
}

// ---------------------------------------------------------------------------------------
// Pass C: forward transforms along y of one kx column + spectral epilogue.
// ---------------------------------------------------------------------------------------
template <typename T, int NY> struct YFwd2D {
    static constexpr int US = padded_len(NY);
    static constexpr int NT = pick_threads<T, 2 * NY>();
    static constexpr size_t SMEM_FFT = (size_t)2 * US * sizeof(cplx<T>);
    static constexpr size_t SMEM = SMEM_FFT > (size_t)NT * 8 ? SMEM_FFT : (size_t)NT * 8;
};

template <typename T, int NY, int EPI>
__global__ void __launch_bounds__(YFwd2D<T, NY>::NT)
k2d_yfwd(const cplx<T>* __restrict__ MB, StageIO<T> io, int input_is_u0, Geo g,
         const cplx<T>* __restrict__ tw) {
    using P = YFwd2D<T, NY>;
    constexpr int US = P::US, NT = P::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    const int kx = blockIdx.x;
    const int K = g.K, KY = g.KY;
    const int tid = threadIdx.x;
    const cplx<T>* src = MB + (size_t)kx * NY * 2;
    for (int e = tid; e < NY * 2; e += NT) {
        const int y = e >> 1, c = e & 1;
        sm[c * US + pidx(y)] = src[e];
    }
    __syncthreads();
    fft_run<T, NY, 2, US, NT, false>(sm, tw);

    const double inv_n = g.inv_n;
    const long long K2 = (long long)K * K;
    const double w = kx == 0 ? 1.0 : 2.0;
    double en = 0.0;
    for (int kyi = tid; kyi < KY; kyi += NT) {
        const int ky = trunc_k(kyi, K, KY);
        const int p = trunc_pos(kyi, K, KY, NY);
        const size_t o = ((size_t)kx * KY + kyi) * 2;
        const long long m2i = (long long)kx * kx + (long long)ky * ky;
        double2 v[2];
        if (m2i < K2) {   // spherical 2/3 rule, tool.F90:185-193
            v[0] = dscale(cvt<cplx<T>, double2>(sm[pidx(p)]), inv_n);
            v[1] = dscale(cvt<cplx<T>, double2>(sm[US + pidx(p)]), inv_n);
        } else {
            v[0] = make_double2(0, 0);
            v[1] = make_double2(0, 0);
        }
        const double kv[2] = {(double)kx, (double)ky};
        rk_epilogue<T, 2, EPI>(v, kv, (double)m2i, o, io, input_is_u0 != 0, g, w, en);
    }
    if constexpr (EPI == EPI_RK3 || EPI == EPI_CN_LAST) {
        if (io.energy_part) {
            __syncthreads();
            double* scratch = reinterpret_cast<double*>(smraw);
            double v[1] = {en};
            block_sum<1, NT>(v, scratch);
            if (tid == 0) io.energy_part[kx] = v[0];
        }
    }
}

}  // namespace bastr
