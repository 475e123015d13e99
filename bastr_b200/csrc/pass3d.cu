// 3D right-hand side as five fused passes (compute_ut3D, solution.F90:865-928, with the RK3/CN
// combinations of solution.F90:233-301 folded into the last pass).  Every pass reads whole
// contiguous lines and writes its result transposed for the next pass:
//
//   A  zinv : lines (kx,ky) along kz of the truncated state -> MA[kx][z][kyi][f]
//             f = g_c = IFFT_z(u_c^), h_c = IFFT_z(i kz u_c^)       (+ q_c = IFFT_z(kz^2 u_c^),
//             t = IFFT_z(lap(theta)^) when velocity-gradient statistics are due)
//   B  yinv : lines (kx,z) along ky -> MB[z][y][kx][f]
//             f = G_c = IFFT_y(g_c), Dy_c = IFFT_y(i ky g_c), Dz_c = IFFT_y(h_c)  (+ lap u_c, lap theta)
//   C  xpass: rows (y,z): six packed complex inverse x transforms give u_c and all nine
//             du_i/dx_j; N_i = -(u_j du_i/dx_j) (solution.F90:903-908); two packed forward
//             transforms -> MC[z][kx][y][c]
//   D  yfwd : lines (kx,z) along y, truncated to |ky| < K -> MD[kx][kyi][z][c]
//   E  zfwd : lines (kx,ky) along z, truncated to |kz| < K, 1/N, spherical dealias
//             (tool.F90:196-217), viscous term, projection (tool.F90:245-270), RK/CN combination.
#include "solver.cuh"

namespace bastr {

// ---------------------------------------------------------------------------------------
// Pass A
// ---------------------------------------------------------------------------------------
enum ZInvSet : int { ZI_STATE = 0, ZI_RHS = 1, ZI_VG = 2 };

template <typename T, int NZ, int SET> struct ZInv3D {
    static constexpr int F = SET == ZI_STATE ? 3 : SET == ZI_RHS ? 6 : 4;
    static constexpr int F0 = SET == ZI_VG ? 6 : 0;
    static constexpr int L = lines_per_block<T, NZ, F>();
    static constexpr int US = padded_len(NZ);
    static constexpr int NT = pick_threads<T, L * F * NZ>();
    static constexpr size_t SMEM = (size_t)L * F * US * sizeof(cplx<T>);
};

template <typename T, typename TIN, int NZ, int SET>
__global__ void __launch_bounds__(ZInv3D<T, NZ, SET>::NT)
k3d_zinv(const cplx<TIN>* __restrict__ S, cplx<T>* __restrict__ MA, int ftot, Geo g,
         const cplx<T>* __restrict__ tw) {
    using P = ZInv3D<T, NZ, SET>;
    constexpr int F = P::F, L = P::L, US = P::US, NT = P::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    const int K = g.K, KY = g.KY, KZ = g.KZ;
    const int nlines = K * KY;
    const int l0 = blockIdx.x * L;
    for (int e = threadIdx.x; e < L * NZ; e += NT) {
        const int r = e / NZ, p = e - r * NZ;
        const int l = l0 + r;
        cplx<T> v[F];
#pragma unroll
        for (int f = 0; f < F; ++f) v[f] = mk<T>(0, 0);
        const int kzi = pos_trunc(p, K, KZ, NZ);
        if (l < nlines && kzi >= 0) {
            const int kx = l / KY, kyi = l - kx * KY;
            const T kz = (T)trunc_k(kzi, K, KZ);
            const size_t o = ((size_t)l * KZ + kzi) * 3;
            const cplx<T> a = cvt<cplx<TIN>, cplx<T>>(S[o]);
            const cplx<T> b = cvt<cplx<TIN>, cplx<T>>(S[o + 1]);
            const cplx<T> c = cvt<cplx<TIN>, cplx<T>>(S[o + 2]);
            if constexpr (SET == ZI_STATE) {
                v[0] = a; v[1] = b; v[2] = c;
            } else if constexpr (SET == ZI_RHS) {
                v[0] = a; v[1] = cscale<T>(cmuli<T>(a), kz);
                v[2] = b; v[3] = cscale<T>(cmuli<T>(b), kz);
                v[4] = c; v[5] = cscale<T>(cmuli<T>(c), kz);
            } else {
                const T kxt = (T)kx, ky = (T)trunc_k(kyi, K, KY);
                const T kz2 = kz * kz;
                v[0] = cscale<T>(a, kz2);
                v[1] = cscale<T>(b, kz2);
                v[2] = cscale<T>(c, kz2);
                // lap(theta)^ = -i |k|^2 (k . u^)   (solution.F90:1216)
                const T kk = kxt * kxt + ky * ky + kz2;
                const cplx<T> dv = cadd<T>(cadd<T>(cscale<T>(a, kxt), cscale<T>(b, ky)), cscale<T>(c, kz));
                v[3] = cscale<T>(cmulni<T>(dv), kk);
            }
        }
#pragma unroll
        for (int f = 0; f < F; ++f) sm[(r * F + f) * US + pidx(p)] = v[f];
    }
    __syncthreads();
    fft_run<T, NZ, L * F, US, NT, true>(sm, tw);
    for (int e = threadIdx.x; e < NZ * L * F; e += NT) {
        const int z = e / (L * F), rem = e - z * (L * F);
        const int r = rem / F, f = rem - r * F;
        const int l = l0 + r;
        if (l >= nlines) continue;
        const int kx = l / KY, kyi = l - kx * KY;
        MA[(((size_t)kx * NZ + z) * KY + kyi) * ftot + P::F0 + f] = sm[(r * F + f) * US + pidx(z)];
    }
}

// ---------------------------------------------------------------------------------------
// Pass B
// ---------------------------------------------------------------------------------------
enum YInv3Set : int { YB_STATE = 0, YB_RHS = 1, YB_RHS_VG = 2 };

template <typename T, int NY, int SET> struct YInv3D {
    static constexpr int FIN = SET == YB_STATE ? 3 : SET == YB_RHS ? 6 : 10;
    static constexpr int F = SET == YB_STATE ? 3 : SET == YB_RHS ? 9 : 13;
    static constexpr int L = lines_per_block<T, NY, F>();
    static constexpr int US = padded_len(NY);
    static constexpr int NT = pick_threads<T, L * F * NY>();
    static constexpr size_t SMEM = (size_t)L * F * US * sizeof(cplx<T>);
};

template <typename T, int NY, int SET>
__global__ void __launch_bounds__(YInv3D<T, NY, SET>::NT)
k3d_yinv(const cplx<T>* __restrict__ MA, cplx<T>* __restrict__ MB, Geo g, const cplx<T>* __restrict__ tw) {
    using P = YInv3D<T, NY, SET>;
    constexpr int F = P::F, FIN = P::FIN, L = P::L, US = P::US, NT = P::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    const int K = g.K, KY = g.KY, NZ = g.nz;
    const int nlines = K * NZ;
    const int l0 = blockIdx.x * L;
    for (int e = threadIdx.x; e < L * NY; e += NT) {
        const int r = e / NY, p = e - r * NY;
        const int l = l0 + r;
        cplx<T> v[F];
#pragma unroll
        for (int f = 0; f < F; ++f) v[f] = mk<T>(0, 0);
        const int kyi = pos_trunc(p, K, KY, NY);
        if (l < nlines && kyi >= 0) {
            const int z = l / K, kx = l - z * K;
            const T ky = (T)trunc_k(kyi, K, KY);
            const cplx<T>* src = MA + ((((size_t)kx * NZ + z) * KY) + kyi) * FIN;
            if constexpr (SET == YB_STATE) {
                v[0] = src[0]; v[1] = src[1]; v[2] = src[2];
            } else {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const cplx<T> gc = src[2 * c], hc = src[2 * c + 1];
                    v[3 * c] = gc;
                    v[3 * c + 1] = cscale<T>(cmuli<T>(gc), ky);
                    v[3 * c + 2] = hc;
                }
                if constexpr (SET == YB_RHS_VG) {
                    // lap u_c without its kx^2 part, which pass C adds: -ky^2 g_c - IFFT_z(kz^2 u_c^)
                    const T ky2 = ky * ky;
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        v[9 + c] = csub<T>(cscale<T>(src[2 * c], -ky2), src[6 + c]);
                    v[12] = src[9];
                }
            }
        }
#pragma unroll
        for (int f = 0; f < F; ++f) sm[(r * F + f) * US + pidx(p)] = v[f];
    }
    __syncthreads();
    fft_run<T, NY, L * F, US, NT, true>(sm, tw);
    for (int e = threadIdx.x; e < NY * L * F; e += NT) {
        const int y = e / (L * F), rem = e - y * (L * F);
        const int r = rem / F, f = rem - r * F;
        const int l = l0 + r;
        if (l >= nlines) continue;
        const int z = l / K, kx = l - z * K;
        MB[((((size_t)z * NY + y) * K) + kx) * F + f] = sm[(r * F + f) * US + pidx(y)];
    }
}

// ---------------------------------------------------------------------------------------
// Pass C
// ---------------------------------------------------------------------------------------
enum X3Mode : int { X3_RHS = 1, X3_RHS_VG = 2, X3_TO_PHYS = 3, X3_FROM_PHYS = 4 };

template <typename T, int NX, int MODE> struct XPass3D {
    static constexpr int FIN = MODE == X3_RHS ? 9 : MODE == X3_RHS_VG ? 13 : MODE == X3_TO_PHYS ? 3 : 0;
    static constexpr int ZU = MODE == X3_RHS ? 6 : MODE == X3_RHS_VG ? 8 : 2;
    static constexpr int BR = lines_per_block<T, NX, ZU>();
    static constexpr int U = ZU * BR;
    static constexpr int US = padded_len(NX);
    static constexpr int NT = pick_threads<T, U * NX>();
    static constexpr size_t SMEM_FFT = (size_t)U * US * sizeof(cplx<T>);
    static constexpr size_t SMEM = SMEM_FFT > (size_t)9 * NT * 8 ? SMEM_FFT : (size_t)9 * NT * 8;
};

template <typename T>
__device__ __forceinline__ void pack2_3(cplx<T>* unit, int k, int NX, cplx<T> A, cplx<T> B) {
    if (k == 0) {
        unit[pidx(0)] = mk<T>(A.x, B.x);
    } else {
        unit[pidx(k)] = mk<T>(A.x - B.y, A.y + B.x);
        unit[pidx(NX - k)] = mk<T>(A.x + B.y, B.x - A.y);
    }
}

template <typename T, int NX, int MODE>
__global__ void __launch_bounds__(XPass3D<T, NX, MODE>::NT)
k3d_xpass(const cplx<T>* __restrict__ MB, cplx<T>* __restrict__ MC, const double* __restrict__ phys_in,
          double* __restrict__ phys_out, double* __restrict__ vg_part, Geo g, const cplx<T>* __restrict__ tw) {
    using P = XPass3D<T, NX, MODE>;
    constexpr int ZU = P::ZU, BR = P::BR, US = P::US, NT = P::NT, FIN = P::FIN;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    const int K = g.K, NY = g.ny;
    const size_t npts = (size_t)NX * NY * g.nz;
    const int row0 = blockIdx.x * BR;   // row = z*NY + y
    const int tid = threadIdx.x;

    if constexpr (MODE == X3_FROM_PHYS) {
        for (int e = tid; e < BR * NX; e += NT) {
            const int r = e / NX, x = e - r * NX;
            const size_t o = (size_t)(row0 + r) * NX + x;
            sm[(r * ZU) * US + pidx(x)] = mk<T>((T)phys_in[o], (T)phys_in[npts + o]);
            sm[(r * ZU + 1) * US + pidx(x)] = mk<T>((T)phys_in[2 * npts + o], (T)0);
        }
    } else {
        const int mid = NX - 2 * K + 1;
        for (int e = tid; e < BR * ZU * mid; e += NT) {
            const int u = e / mid, x = K + (e - u * mid);
            sm[u * US + pidx(x)] = mk<T>(0, 0);
        }
        for (int e = tid; e < BR * K; e += NT) {
            const int r = e / K, k = e - r * K;
            const cplx<T>* src = MB + ((size_t)(row0 + r) * K + k) * FIN;
            cplx<T>* z = sm + r * ZU * US;
            if constexpr (MODE == X3_TO_PHYS) {
                pack2_3<T>(z, k, NX, src[0], src[1]);
                pack2_3<T>(z + US, k, NX, src[2], mk<T>(0, 0));
            } else {
                const T kx = (T)k;
                const cplx<T> G1 = src[0], Dy1 = src[1], Dz1 = src[2];
                const cplx<T> G2 = src[3], Dy2 = src[4], Dz2 = src[5];
                const cplx<T> G3 = src[6], Dy3 = src[7], Dz3 = src[8];
                const cplx<T> X1 = cscale<T>(cmuli<T>(G1), kx), X2 = cscale<T>(cmuli<T>(G2), kx),
                              X3 = cscale<T>(cmuli<T>(G3), kx);
                pack2_3<T>(z, k, NX, G1, G2);              // u1, u2
                pack2_3<T>(z + US, k, NX, G3, X1);         // u3, du1/dx
                pack2_3<T>(z + 2 * US, k, NX, X2, X3);     // du2/dx, du3/dx
                pack2_3<T>(z + 3 * US, k, NX, Dy1, Dy2);   // du1/dy, du2/dy
                pack2_3<T>(z + 4 * US, k, NX, Dy3, Dz1);   // du3/dy, du1/dz
                pack2_3<T>(z + 5 * US, k, NX, Dz2, Dz3);   // du2/dz, du3/dz
                if constexpr (MODE == X3_RHS_VG) {
                    const T kx2 = kx * kx;
                    const cplx<T> L1 = csub<T>(src[9], cscale<T>(G1, kx2));
                    const cplx<T> L2 = csub<T>(src[10], cscale<T>(G2, kx2));
                    const cplx<T> L3 = csub<T>(src[11], cscale<T>(G3, kx2));
                    pack2_3<T>(z + 6 * US, k, NX, L1, L2);
                    pack2_3<T>(z + 7 * US, k, NX, L3, src[12]);
                }
            }
        }
    }
    __syncthreads();

    if constexpr (MODE == X3_FROM_PHYS) {
        fft_run<T, NX, BR * ZU, US, NT, false>(sm, tw);
    } else {
        fft_run<T, NX, BR * ZU, US, NT, true>(sm, tw);
    }

    if constexpr (MODE == X3_TO_PHYS) {
        for (int e = tid; e < BR * NX; e += NT) {
            const int r = e / NX, x = e - r * NX;
            const cplx<T> a = sm[(r * ZU) * US + pidx(x)], b = sm[(r * ZU + 1) * US + pidx(x)];
            const size_t o = (size_t)(row0 + r) * NX + x;
            phys_out[o] = (double)a.x;
            phys_out[npts + o] = (double)a.y;
            phys_out[2 * npts + o] = (double)b.x;
        }
        return;
    }

    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double etamin = 1.0 / 0.0;
    if constexpr (MODE == X3_RHS || MODE == X3_RHS_VG) {
        const double nu = g.nu;
        for (int e = tid; e < BR * NX; e += NT) {
            const int r = e / NX, x = e - r * NX;
            cplx<T>* z = sm + r * ZU * US;
            const cplx<T> z0 = z[pidx(x)], z1 = z[US + pidx(x)], z2 = z[2 * US + pidx(x)];
            const cplx<T> z3 = z[3 * US + pidx(x)], z4 = z[4 * US + pidx(x)], z5 = z[5 * US + pidx(x)];
            const T u1 = z0.x, u2 = z0.y, u3 = z1.x;
            const T d11 = z1.y, d21 = z2.x, d31 = z2.y;   // d_ij = du_i/dx_j
            const T d12 = z3.x, d22 = z3.y, d32 = z4.x;
            const T d13 = z4.y, d23 = z5.x, d33 = z5.y;
            const T n1 = -u1 * d11 - u2 * d12 - u3 * d13;
            const T n2 = -u1 * d21 - u2 * d22 - u3 * d23;
            const T n3 = -u1 * d31 - u2 * d32 - u3 * d33;
            z[pidx(x)] = mk<T>(n1, n2);
            z[US + pidx(x)] = mk<T>(n3, (T)0);
            if constexpr (MODE == X3_RHS_VG) {
                // velgrad_calculate3D (solution.F90:1240-1266), accumulated in FP64
                const cplx<T> z6 = z[6 * US + pidx(x)], z7 = z[7 * US + pidx(x)];
                const double U1 = u1, U2 = u2, U3 = u3;
                const double D11 = d11, D22 = d22, D33 = d33, D12 = d12, D21 = d21, D13 = d13, D31 = d31,
                             D23 = d23, D32 = d32;
                const double div = D11 + D22 + D33;
                const double uu = U1 * U1 + U2 * U2 + U3 * U3;
                acc[0] += div * div * uu;
                acc[1] += (D11 * D11 + D22 * D22 + D33 * D33 + 2.0 * D12 * D21 + 2.0 * D13 * D31 +
                           2.0 * D23 * D32) * uu;
                acc[2] += div * uu;
                acc[3] += 2.0 * U1 * div * (double)z6.x + 2.0 * U2 * div * (double)z6.y +
                          2.0 * U3 * div * (double)z7.x + uu * (double)z7.y;
                acc[4] += nu * (D12 - D21) * (D12 - D21) + nu * (D23 - D32) * (D23 - D32) +
                          nu * (D13 - D31) * (D13 - D31) + nu * div * div;
                etamin = fmin(etamin, sqrt(nu / fabs(div)));
                acc[5] += uu;
                acc[6] += D11 * D11 + D22 * D22 + D33 * D33;
            }
        }
        __syncthreads();
        fft_run<T, NX, BR * 2, US, NT, false, 2, ZU * US>(sm, tw);
    } else {
        // X3_FROM_PHYS: already transformed
    }

    // split the packed spectra, kx in [0,K): unit 0 -> (c0, c1), unit 1 -> (c2, -)
    for (int e = tid; e < BR * K; e += NT) {
        const int r = e / K, k = e - r * K;
        const int row = row0 + r;
        const int z_ = row / NY, y = row - z_ * NY;
        const cplx<T>* zz = sm + r * ZU * US;
        cplx<T>* dst = MC + (((size_t)z_ * K + k) * NY + y) * 3;
        {
            const cplx<T> Z = zz[pidx(k)];
            const cplx<T> Zc = cconj<T>(zz[pidx(k == 0 ? 0 : NX - k)]);
            dst[0] = cscale<T>(cadd<T>(Z, Zc), (T)0.5);
            dst[1] = cscale<T>(cmulni<T>(csub<T>(Z, Zc)), (T)0.5);
        }
        {
            const cplx<T> Z = zz[US + pidx(k)];
            const cplx<T> Zc = cconj<T>(zz[US + pidx(k == 0 ? 0 : NX - k)]);
            dst[2] = cscale<T>(cadd<T>(Z, Zc), (T)0.5);
        }
    }
    if constexpr (MODE == X3_RHS_VG) {
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
// Pass D: forward y transforms, truncation to |ky| < K.
// ---------------------------------------------------------------------------------------
template <typename T, int NY> struct YFwd3D {
    static constexpr int L = lines_per_block<T, NY, 3>();
    static constexpr int US = padded_len(NY);
    static constexpr int NT = pick_threads<T, L * 3 * NY>();
    static constexpr size_t SMEM = (size_t)L * 3 * US * sizeof(cplx<T>);
};

template <typename T, int NY>
__global__ void __launch_bounds__(YFwd3D<T, NY>::NT)
k3d_yfwd(const cplx<T>* __restrict__ MC, cplx<T>* __restrict__ MD, Geo g, const cplx<T>* __restrict__ tw) {
    using P = YFwd3D<T, NY>;
    constexpr int L = P::L, US = P::US, NT = P::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    const int K = g.K, KY = g.KY, NZ = g.nz;
    const int nlines = K * NZ;    // line = kx*NZ + z
    const int l0 = blockIdx.x * L;
    for (int e = threadIdx.x; e < L * NY * 3; e += NT) {
        const int r = e / (NY * 3), rem = e - r * (NY * 3);
        const int y = rem / 3, c = rem - y * 3;
        const int l = l0 + r;
        cplx<T> v = mk<T>(0, 0);
        if (l < nlines) {
            const int kx = l / NZ, z = l - kx * NZ;
            v = MC[(((size_t)z * K + kx) * NY + y) * 3 + c];
        }
        sm[(r * 3 + c) * US + pidx(y)] = v;
    }
    __syncthreads();
    fft_run<T, NY, L * 3, US, NT, false>(sm, tw);
    for (int e = threadIdx.x; e < KY * L * 3; e += NT) {
        const int kyi = e / (L * 3), rem = e - kyi * (L * 3);
        const int r = rem / 3, c = rem - r * 3;
        const int l = l0 + r;
        if (l >= nlines) continue;
        const int kx = l / NZ, z = l - kx * NZ;
        const int p = trunc_pos(kyi, K, KY, NY);
        MD[(((size_t)kx * KY + kyi) * NZ + z) * 3 + c] = sm[(r * 3 + c) * US + pidx(p)];
    }
}

// ---------------------------------------------------------------------------------------
// Pass E: forward z transforms + spectral epilogue.
// ---------------------------------------------------------------------------------------
template <typename T, int NZ> struct ZFwd3D {
    static constexpr int L = lines_per_block<T, NZ, 3>();
    static constexpr int US = padded_len(NZ);
    static constexpr int NT = pick_threads<T, L * 3 * NZ>();
    static constexpr size_t SMEM_FFT = (size_t)L * 3 * US * sizeof(cplx<T>);
    static constexpr size_t SMEM = SMEM_FFT > (size_t)NT * 8 ? SMEM_FFT : (size_t)NT * 8;
};

template <typename T, int NZ, int EPI>
__global__ void __launch_bounds__(ZFwd3D<T, NZ>::NT)
k3d_zfwd(const cplx<T>* __restrict__ MD, StageIO<T> io, int input_is_u0, Geo g, const cplx<T>* __restrict__ tw) {
    using P = ZFwd3D<T, NZ>;
    constexpr int L = P::L, US = P::US, NT = P::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    const int K = g.K, KY = g.KY, KZ = g.KZ;
    const int nlines = K * KY;    // line = kx*KY + kyi
    const int l0 = blockIdx.x * L;
    for (int e = threadIdx.x; e < L * NZ * 3; e += NT) {
        const int r = e / (NZ * 3), rem = e - r * (NZ * 3);
        const int z = rem / 3, c = rem - z * 3;
        const int l = l0 + r;
        const cplx<T> v = l < nlines ? MD[((size_t)l * NZ + z) * 3 + c] : mk<T>(0, 0);
        sm[(r * 3 + c) * US + pidx(z)] = v;
    }
    __syncthreads();
    fft_run<T, NZ, L * 3, US, NT, false>(sm, tw);

    const double inv_n = g.inv_n;
    const long long K2 = (long long)K * K;
    double en = 0.0;
    for (int e = threadIdx.x; e < L * KZ; e += NT) {
        const int r = e / KZ, kzi = e - r * KZ;
        const int l = l0 + r;
        if (l >= nlines) continue;
        const int kx = l / KY, kyi = l - kx * KY;
        const int ky = trunc_k(kyi, K, KY), kz = trunc_k(kzi, K, KZ);
        const int p = trunc_pos(kzi, K, KZ, NZ);
        const size_t o = ((size_t)l * KZ + kzi) * 3;
        const long long m2i = (long long)kx * kx + (long long)ky * ky + (long long)kz * kz;
        double2 v[3];
        if (m2i < K2) {   // spherical 2/3 rule, tool.F90:206-214
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] = dscale(cvt<cplx<T>, double2>(sm[(r * 3 + c) * US + pidx(p)]), inv_n);
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] = make_double2(0, 0);
        }
        const double kv[3] = {(double)kx, (double)ky, (double)kz};
        const double w = kx == 0 ? 1.0 : 2.0;
        rk_epilogue<T, 3, EPI>(v, kv, (double)m2i, o, io, input_is_u0 != 0, g, w, en);
    }
    if constexpr (EPI == EPI_RK3 || EPI == EPI_CN_LAST) {
        if (io.energy_part) {
            __syncthreads();
            double* scratch = reinterpret_cast<double*>(smraw);
            double v[1] = {en};
            block_sum<1, NT>(v, scratch);
            if (threadIdx.x == 0) io.energy_part[blockIdx.x] = v[0];
        }
    }
}

}  // namespace bastr
