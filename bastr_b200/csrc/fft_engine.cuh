// Complex arithmetic and register DFTs shared by the transforms of sm_100a passes.
//
// cplx<T> is float2 / double2; the single-precision add, subtract and scale use Blackwell's
// packed FP32x2 instructions.  dft2/4/8/16 are in-register DFTs in natural order (the radix
// kernels of the Stockham transforms in regfft.cuh); rot4 is the quarter turn of the
// transform's sign.
//
// Shared-memory addresses of staged lines are padded by one element every 16 (pidx) so that
// strided accesses do not collide on the same banks.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bastr {

template <typename T> struct cvec;
template <> struct cvec<float>  { using t = float2; };
template <> struct cvec<double> { using t = double2; };
template <typename T> using cplx = typename cvec<T>::t;

template <typename T> __device__ __forceinline__ cplx<T> mk(T x, T y) { cplx<T> r; r.x = x; r.y = y; return r; }

// Single-precision complex add/subtract/scale map onto Blackwell's packed FP32x2 instructions
// (add/sub/mul.rn.f32x2): one instruction for both components.
__device__ __forceinline__ unsigned long long f2bits(float2 a) { return *reinterpret_cast<unsigned long long*>(&a); }
__device__ __forceinline__ float2 bitsf2(unsigned long long b) { return *reinterpret_cast<float2*>(&b); }
__device__ __forceinline__ float2 add_f32x2(float2 a, float2 b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2bits(a)), "l"(f2bits(b)));
    return bitsf2(r);
}
__device__ __forceinline__ float2 sub_f32x2(float2 a, float2 b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2bits(a)), "l"(f2bits(b)));
    return bitsf2(r);
}
__device__ __forceinline__ float2 mul_f32x2(float2 a, float2 b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2bits(a)), "l"(f2bits(b)));
    return bitsf2(r);
}

template <typename T> __device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) {
    if constexpr (sizeof(T) == 4) return add_f32x2(a, b);
    else return mk<T>(a.x + b.x, a.y + b.y);
}
template <typename T> __device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) {
    if constexpr (sizeof(T) == 4) return sub_f32x2(a, b);
    else return mk<T>(a.x - b.x, a.y - b.y);
}
template <typename T> __device__ __forceinline__ cplx<T> cscale(cplx<T> a, T s) {
    if constexpr (sizeof(T) == 4) return mul_f32x2(a, make_float2(s, s));
    else return mk<T>(a.x * s, a.y * s);
}
template <typename T> __device__ __forceinline__ cplx<T> cconj(cplx<T> a) { return mk<T>(a.x, -a.y); }
template <typename T> __device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return mk<T>(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// multiply by i and by -i
template <typename T> __device__ __forceinline__ cplx<T> cmuli(cplx<T> a) { return mk<T>(-a.y, a.x); }
template <typename T> __device__ __forceinline__ cplx<T> cmulni(cplx<T> a) { return mk<T>(a.y, -a.x); }

// Rotation by the quarter turn of the transform's sign: forward (sign -1) multiplies by -i,
// inverse (sign +1) by +i.
template <typename T, bool INV> __device__ __forceinline__ cplx<T> rot4(cplx<T> a) {
    return INV ? cmuli<T>(a) : cmulni<T>(a);
}

// Padded shared-memory index: one spare slot every 16 elements.
__device__ __forceinline__ int pidx(int a) { return a + (a >> 4); }
__host__ __device__ constexpr int padded_len(int n) { return n + (n >> 4); }

// ---------------------------------------------------------------------------------------
// Register DFTs of size 2, 4, 8 and 16, natural order in and out.
// ---------------------------------------------------------------------------------------
template <typename T, bool INV> __device__ __forceinline__ void dft2(cplx<T>& a, cplx<T>& b) {
    cplx<T> t = a;
    a = cadd<T>(t, b);
    b = csub<T>(t, b);
}

template <typename T, bool INV> __device__ __forceinline__ void dft4(cplx<T>* v) {
    cplx<T> s02 = cadd<T>(v[0], v[2]), d02 = csub<T>(v[0], v[2]);
    cplx<T> s13 = cadd<T>(v[1], v[3]), d13 = rot4<T, INV>(csub<T>(v[1], v[3]));
    v[0] = cadd<T>(s02, s13);
    v[2] = csub<T>(s02, s13);
    v[1] = cadd<T>(d02, d13);
    v[3] = csub<T>(d02, d13);
}

template <typename T, bool INV> __device__ __forceinline__ void dft8(cplx<T>* v) {
    const T h = (T)0.70710678118654752440084436210484903928;  // sqrt(1/2)
    cplx<T> e[4] = {v[0], v[2], v[4], v[6]};
    cplx<T> o[4] = {v[1], v[3], v[5], v[7]};
    dft4<T, INV>(e);
    dft4<T, INV>(o);
    // o[k] *= exp(sign*i*pi*k/4)
    const T sg = INV ? (T)1 : (T)-1;
    o[1] = mk<T>(h * (o[1].x - sg * o[1].y), h * (o[1].y + sg * o[1].x));
    o[2] = rot4<T, INV>(o[2]);
    o[3] = mk<T>(-h * (o[3].x + sg * o[3].y), h * (sg * o[3].x - o[3].y));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = cadd<T>(e[k], o[k]);
        v[k + 4] = csub<T>(e[k], o[k]);
    }
}

template <typename T, bool INV> __device__ __forceinline__ void dft16(cplx<T>* v) {
    // 16 = 4 x 4: columns n2, inner index n1 (x[4*n1 + n2])
    const T c1 = (T)0.92387953251128675612818318939678828682;   // cos(pi/8)
    const T s1 = (T)0.38268343236508977172845998403039886676;   // sin(pi/8)
    const T h = (T)0.70710678118654752440084436210484903928;    // cos(pi/4)
    const T sg = INV ? (T)1 : (T)-1;
    cplx<T> y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
#pragma unroll
        for (int n1 = 0; n1 < 4; ++n1) y[n2][n1] = v[4 * n1 + n2];
        dft4<T, INV>(y[n2]);
    }
    // twiddle y[n2][k1] *= exp(sign*i*2*pi*n2*k1/16)
    // n2 = 1: angles pi/8 * k1; n2 = 2: pi/4 * k1; n2 = 3: 3pi/8 * k1
    const T cs[10] = {(T)1, c1, h, s1, (T)0, -s1, -h, -c1, (T)-1, -c1};
    const T sn[10] = {(T)0, s1, h, c1, (T)1, c1, h, s1, (T)0, -s1};
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2) {
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) {
            const int m = n2 * k1;  // 1..9
            cplx<T> w = mk<T>(cs[m], sg * sn[m]);
            y[n2][k1] = cmul<T>(y[n2][k1], w);
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        cplx<T> z[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
        dft4<T, INV>(z);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = z[k2];
    }
}

template <typename T, bool INV, int R> __device__ __forceinline__ void dftR(cplx<T>* v) {
    if constexpr (R == 2) dft2<T, INV>(v[0], v[1]);
    else if constexpr (R == 4) dft4<T, INV>(v);
    else if constexpr (R == 8) dft8<T, INV>(v);
    else dft16<T, INV>(v);
}

}  // namespace bastr
