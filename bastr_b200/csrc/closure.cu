// Learned subgrid closure for the coarse 3D solve: a small local network that maps the
// filtered velocity u (3 channels) to the subgrid term tau = filter(u.grad u) - u.grad u.
//
//   layer 1  3x3x3 periodic stencil, 3 -> 32 channels, GELU
//   layer 2  1x1x1, 32 -> 32, GELU
//   layer 3  1x1x1, 32 -> 32, GELU
//   layer 4  1x1x1, 32 -> 3
//
// Arithmetic: weights and every layer's inputs (the 81 taps, the activations h1..h3) are BF16
// (round to nearest even), every sum is accumulated in FP32, biases and GELU are FP32.  GELU is
// the tanh form 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), evaluated as z * sigmoid(2 y).  Parameter layout (NP = 4835
// floats): W1[32][81] (input tap i = c*27 + (dz+1)*9 + (dy+1)*3 + (dx+1)), b1[32], W2[32][32],
// b2[32], W3[32][32], b3[32], W4[3][32], b4[3].
//
// Inference (k_net_forward_tc) runs the four layers as tensor-core GEMMs: M = 128 points per
// tile, N = 32 channels (16 for the last layer, padded), K = 96 (81 taps padded) or 32, issued
// with tcgen05.mma by one thread, accumulated in TMEM and finished (bias, GELU, BF16 rounding)
// by the thread that owns the point's TMEM lane.
//
// Training: k_net_grad runs the same arithmetic per point on the FMA pipes for tiles of 64
// points, keeps every point's activations and back-propagated errors in shared memory, and
// accumulates the weight gradients of its tiles in registers (each thread owns fixed parameters
// and sums over points in a fixed order); the per-block partials are summed in fixed order by
// k_net_reduce, so a gradient is deterministic.  The rounding of layer inputs is passed through
// unchanged by back-propagation (its derivative is taken as 1).  k_net_adam updates the FP32
// master weights and their BF16 copy.
#pragma once
#include <cuda_bf16.h>
#include "solver.cuh"
#include "umma.cuh"

namespace bastr {

constexpr int kNetC = 32, kNetIn = 81;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kNetC * kNetIn, kOffW2 = kOffB1 + kNetC, kOffB2 = kOffW2 + kNetC * kNetC,
              kOffW3 = kOffB2 + kNetC, kOffB3 = kOffW3 + kNetC * kNetC, kOffW4 = kOffB3 + kNetC,
              kOffB4 = kOffW4 + 3 * kNetC, kNetNP = kOffB4 + 3;

// GELU, tanh form, evaluated as z * sigmoid(2y) (0.5 (1 + tanh y) = 1 / (1 + e^-2y), y = sqrt(2/pi)
// (z + 0.044715 z^3)) with the fast exponential and division intrinsics: a few instructions and
// about 1e-6 relative error, far below the BF16 rounding of the result.  dg = d gelu / dz
// = s + 2 z s (1 - s) sqrt(2/pi) (1 + 3 * 0.044715 z^2), s = sigmoid(2y).
__device__ __forceinline__ float gelu_s(float z) {
    // e^-2y = 2^(z (k1 + k3 z^2)), k1 = -2 sqrt(2/pi) log2(e), k3 = 0.044715 k1
    const float k1 = -2.302208198144325f, k3 = -0.10294324f;
    float e;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(z * fmaf(k3, z * z, k1)));
    return __fdividef(z, 1.0f + e);
}
__device__ __forceinline__ float gelu_t(float z, float& dg) {
    const float a = 0.7978845608028654f, c = 0.044715f;
    const float y = a * fmaf(c * z, z * z, z);
    const float sg = __fdividef(1.0f, 1.0f + __expf(-2.0f * y));
    dg = sg + 2.0f * z * sg * (1.0f - sg) * a * fmaf(3.0f * c, z * z, 1.0f);
    return z * sg;
}

// The BF16 value nearest x (ties to even), as FP32: the operand a tensor core would see.
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Weights from BF16 into shared memory as FP32 (every block, once).
__device__ __forceinline__ void load_weights(float* sw, const __nv_bfloat16* __restrict__ w) {
    for (int i = threadIdx.x; i < kNetNP; i += blockDim.x) sw[i] = __bfloat162float(w[i]);
}

// Input taps of point (x, y, z): 3 channels x 27 periodic neighbours, field [3][nz][ny][nx].
template <typename TI>
__device__ __forceinline__ float tap(const TI* __restrict__ u, int c, int x, int y, int z, int t, int nx, int ny,
                                     int nz, size_t n) {
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    const int xx = (x + dx + nx) % nx, yy = (y + dy + ny) % ny, zz = (z + dz + nz) % nz;
    return (float)u[c * n + ((size_t)zz * ny + yy) * nx + xx];
}

// Forward pass of one point -> out[3].  With GRAD it also records, for back-propagation, the
// 81 inputs X, the activations H1..H3 and the GELU slopes D1..D3 (kNetC each; shared memory).
template <typename TI, bool GRAD>
__device__ __forceinline__ void net_point(const float* sw, const TI* __restrict__ u, int x, int y, int z, int nx,
                                          int ny, int nz, size_t n, float* X, float* H1, float* H2, float* H3,
                                          float* D1, float* D2, float* D3, float out[3]) {
    float a[kNetC], b[kNetC];
#pragma unroll
    for (int o = 0; o < kNetC; ++o) a[o] = sw[kOffB1 + o];
    for (int i = 0; i < kNetIn; ++i) {
        const float xi = bf16r(tap(u, i / 27, x, y, z, i % 27, nx, ny, nz, n));
        if constexpr (GRAD) X[i] = xi;
#pragma unroll
        for (int o = 0; o < kNetC; ++o) a[o] = fmaf(sw[kOffW1 + o * kNetIn + i], xi, a[o]);
    }
#pragma unroll
    for (int o = 0; o < kNetC; ++o) {
        float d;
        a[o] = bf16r(gelu_t(a[o], d));
        if constexpr (GRAD) { H1[o] = a[o]; D1[o] = d; }
    }
#pragma unroll
    for (int o = 0; o < kNetC; ++o) {
        float s = sw[kOffB2 + o];
#pragma unroll
        for (int i = 0; i < kNetC; ++i) s = fmaf(sw[kOffW2 + o * kNetC + i], a[i], s);
        float d;
        b[o] = bf16r(gelu_t(s, d));
        if constexpr (GRAD) { H2[o] = b[o]; D2[o] = d; }
    }
#pragma unroll
    for (int o = 0; o < kNetC; ++o) {
        float s = sw[kOffB3 + o];
#pragma unroll
        for (int i = 0; i < kNetC; ++i) s = fmaf(sw[kOffW3 + o * kNetC + i], b[i], s);
        float d;
        a[o] = bf16r(gelu_t(s, d));
        if constexpr (GRAD) { H3[o] = a[o]; D3[o] = d; }
    }
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        float s = sw[kOffB4 + o];
#pragma unroll
        for (int i = 0; i < kNetC; ++i) s = fmaf(sw[kOffW4 + o * kNetC + i], a[i], s);
        out[o] = s;
    }
}

// ---------------------------------------------------------------------------------------
// Inference on the tensor cores.
// ---------------------------------------------------------------------------------------
constexpr int kFwdNT = 128;                 // threads per block = points per tile = MMA M
constexpr int kK1 = 96;                     // layer-1 K: 81 taps padded to a multiple of 16
constexpr int kN4 = 16;                     // layer-4 N: 3 outputs padded to the MMA minimum
constexpr uint32_t kFwdCols = 32;           // TMEM columns: one 128 x 32 FP32 accumulator
// dynamic shared memory: B operands (weights), biases, A operands (taps, activations)
constexpr uint32_t kSmW1 = 0, kSmW2 = kSmW1 + 32 * kK1 * 2, kSmW3 = kSmW2 + 32 * 32 * 2,
                   kSmW4 = kSmW3 + 32 * 32 * 2, kSmBias = kSmW4 + kN4 * 32 * 2, kSmX = kSmBias + 512,
                   kSmH = kSmX + kFwdNT * kK1 * 2, kFwdSmem = kSmH + kFwdNT * 32 * 2;

// Eight BF16 values as one 16-byte chunk.
__device__ __forceinline__ uint4 pack8_bf16(const float* v) {
    uint4 q;
    uint32_t* w = reinterpret_cast<uint32_t*>(&q);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        w[i] = *reinterpret_cast<const uint32_t*>(&h);
    }
    return q;
}

// Bias, GELU and BF16 rounding of one point's 32 accumulator columns into row r of the
// activation tile (the next layer's A operand).
__device__ __forceinline__ void act_row(unsigned char* smH, int r, const float (&acc)[32], const float* bias) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) h[i] = gelu_s(acc[8 * c + i] + bias[8 * c + i]);
        *reinterpret_cast<uint4*>(smH + umma_off(r, c, 32)) = pack8_bf16(h);
    }
}

// out[c][p] = scale * net(u)[c] at every point; persistent over tiles of 128 consecutive
// points.  Per tile: the block gathers the points' taps into the A tile, then for each layer one
// thread issues the K/16 MMAs and commits them to an mbarrier, every thread waits for it (bounded:
// on giving up it records TMA_ERR_TIMEOUT in *err, when given, writes NaN for its point and the
// block stops), reads its point's accumulator row from TMEM and writes the next A tile.
template <typename TI>
__global__ void __launch_bounds__(kFwdNT, 4) k_net_forward_tc(const TI* __restrict__ u, const __nv_bfloat16* __restrict__ w,
                                                           float* __restrict__ out, int nx, int ny, int nz, float scale,
                                                           unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smf[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int t = threadIdx.x, warp = t >> 5;
    // weights into the K-major B tiles (zero padding past 81 taps and past 3 outputs), biases
    for (int i = t; i < 32 * (kK1 / 8); i += kFwdNT) {
        const int r = i / (kK1 / 8), c = i % (kK1 / 8);
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int k = 8 * c + j;
            v[j] = k < kNetIn ? __bfloat162float(w[kOffW1 + r * kNetIn + k]) : 0.0f;
        }
        *reinterpret_cast<uint4*>(smf + kSmW1 + umma_off(r, c, kK1)) = pack8_bf16(v);
    }
    for (int i = t; i < (32 + 32 + kN4) * 4; i += kFwdNT) {
        const int m = i / (32 * 4), r = (i / 4) % 32, c = i % 4;   // m = 0: W2, 1: W3, 2: W4
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int k = 8 * c + j;
            v[j] = m == 0 ? __bfloat162float(w[kOffW2 + r * kNetC + k])
                 : m == 1 ? __bfloat162float(w[kOffW3 + r * kNetC + k])
                 : (r < 3 ? __bfloat162float(w[kOffW4 + r * kNetC + k]) : 0.0f);
        }
        const uint32_t base = m == 0 ? kSmW2 : m == 1 ? kSmW3 : kSmW4;
        *reinterpret_cast<uint4*>(smf + base + umma_off(r, c, 32)) = pack8_bf16(v);
    }
    float* sb = reinterpret_cast<float*>(smf + kSmBias);
    for (int i = t; i < 3 * kNetC + 3; i += kFwdNT)
        sb[i] = __bfloat162float(w[i < kNetC ? kOffB1 + i : i < 2 * kNetC ? kOffB2 + i - kNetC
                                 : i < 3 * kNetC ? kOffB3 + i - 2 * kNetC : kOffB4 + i - 3 * kNetC]);
    if (t == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(&tmem_base, kFwdCols);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t tmem_row = tmem + ((uint32_t)(warp * 32) << 16);   // this warp's 32 lanes
    const uint32_t sbase = smem_u32(smf);
    constexpr uint32_t kI32 = umma_idesc_bf16(kFwdNT, 32), kI16 = umma_idesc_bf16(kFwdNT, kN4);

    const size_t n = (size_t)nx * ny * nz;
    const size_t ntiles = (n + kFwdNT - 1) / kFwdNT;
    uint32_t phase = 0;
    bool lost = false;
    // one layer: K/16 MMAs from A (K values per row) and B, then the wait for their completion
    auto layer = [&](uint32_t a_off, uint32_t b_off, int K, uint32_t idesc) -> bool {
        if (t == 0) {
            tc_fence_after();
            for (int k = 0; k < K / 16; ++k)
                umma_bf16(tmem, umma_desc(sbase + a_off + 256u * k, kUmmaLBO, (uint32_t)(K / 8) * 128u),
                          umma_desc(sbase + b_off + 256u * k, kUmmaLBO, (uint32_t)(K / 8) * 128u), idesc, k > 0);
            umma_commit(&bar);
        }
        const bool mine = mbar_wait(&bar, phase, err);
        if (mine) phase ^= 1u;
        const bool ok = __syncthreads_and(mine);   // block-uniform, so every later barrier matches
        tc_fence_after();
        return ok;
    };
    for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const size_t p = tile * kFwdNT + t;
        const bool valid = p < n;
        // the point's 81 taps, BF16, as row t of the layer-1 A tile (each 16-byte chunk stored
        // as soon as its 8 values are gathered)
        {
            const int x = valid ? (int)(p % nx) : 0, y = valid ? (int)((p / nx) % ny) : 0;
            const int z = valid ? (int)(p / ((size_t)nx * ny)) : 0;
            // periodic neighbour offsets (n < 2^31 points: 32-bit offsets)
            const int xs[3] = {x == 0 ? nx - 1 : x - 1, x, x == nx - 1 ? 0 : x + 1};
            const int yo[3] = {(y == 0 ? ny - 1 : y - 1) * nx, y * nx, (y == ny - 1 ? 0 : y + 1) * nx};
            const int zo[3] = {(z == 0 ? nz - 1 : z - 1) * ny * nx, z * ny * nx, (z == nz - 1 ? 0 : z + 1) * ny * nx};
            float v[8];
#pragma unroll
            for (int i = 0; i < kK1; ++i) {
                float val = 0.0f;
                if (i < kNetIn && valid) {
                    const int c = i / 27, dz = (i / 9) % 3, dy = (i / 3) % 3, dx = i % 3;
                    val = (float)u[(unsigned)(c * (int)n + zo[dz] + yo[dy] + xs[dx])];
                }
                v[i % 8] = val;
                if (i % 8 == 7)
                    *reinterpret_cast<uint4*>(smf + kSmX + umma_off(t, i / 8, kK1)) = pack8_bf16(v);
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        float acc[32];
        bool ok = layer(kSmX, kSmW1, kK1, kI32);
        if (ok) {
            tmem_ld32(tmem_row, acc);
            act_row(smf + kSmH, t, acc, sb);
        }
        // layers 2 and 3: A = the activation tile, rewritten in place once its MMAs completed
#pragma unroll 1
        for (int l = 0; l < 2 && ok; ++l) {
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            ok = layer(kSmH, l == 0 ? kSmW2 : kSmW3, 32, kI32);
            if (ok) {
                tmem_ld32(tmem_row, acc);
                act_row(smf + kSmH, t, acc, sb + (l + 1) * kNetC);
            }
        }
        if (ok) {
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            ok = layer(kSmH, kSmW4, 32, kI16);
        }
        if (ok) {
            float o[16];
            tmem_ld16(tmem_row, o);
            if (valid) {
#pragma unroll
                for (int c = 0; c < 3; ++c) out[c * n + p] = scale * (o[c] + sb[3 * kNetC + c]);
            }
        } else if (valid) {
#pragma unroll
            for (int c = 0; c < 3; ++c) out[c * n + p] = __int_as_float(0x7fc00000);
        }
        // every thread's TMEM reads are done before the next tile's first MMA overwrites D
        tc_fence_before();
        if (__syncthreads_or(!ok)) {
            lost = true;
            break;
        }
    }
    if (lost && t == 0) mbar_wait(&bar, phase, nullptr);   // bounded drain of the MMAs in flight
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, kFwdCols);
}

constexpr int kGradTile = 64;    // points per tile
constexpr int kRow = kNetC + 1;  // padded row of a point's activations (no bank conflicts)
constexpr int kGradNT = 128;     // threads per block
constexpr int kGradPer = (kNetNP + kGradNT - 1) / kGradNT;   // parameters owned per thread

// Loss L = sum over points and channels of (net(u) - tau)^2 / (3 n) and its gradient: per-block
// partial sums part[block][kNetNP + 1] (the last entry: the block's sum of squared errors).
__global__ void __launch_bounds__(kGradNT) k_net_grad(const float* __restrict__ u, const float* __restrict__ tau,
                                                      const __nv_bfloat16* __restrict__ w, float* __restrict__ part,
                                                      int nx, int ny, int nz) {
    extern __shared__ __align__(16) float sm[];
    float* sw = sm;                                          // kNetNP
    float* sx = sw + ((kNetNP + 3) & ~3);                    // [tile][81] inputs
    float* sh = sx + kGradTile * kNetIn;                     // [3][tile][33] activations h1..h3
    float* sd = sh + 3 * kGradTile * kRow;                   // [3][tile][33] errors dz1..dz3
    float* so = sd + 3 * kGradTile * kRow;                   // [tile][3] output errors
    float* sr = so + kGradTile * 3;                          // reduction scratch [kGradNT]
    load_weights(sw, w);
    __syncthreads();
    const size_t n = (size_t)nx * ny * nz;
    const float inv = 1.0f / (3.0f * (float)n);
    float g[kGradPer];
#pragma unroll
    for (int k = 0; k < kGradPer; ++k) g[k] = 0.0f;
    float sse = 0.0f;
    const size_t ntiles = (n + kGradTile - 1) / kGradTile;
    for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const size_t p0 = tile * kGradTile;
        // forward + backward of the tile's points: threads 0..tile-1 take one point each
        const int j = threadIdx.x;
        if (j < kGradTile) {
            const size_t p = p0 + j;
            float* hx = sx + j * kNetIn;
            float* h1 = sh + (0 * kGradTile + j) * kRow;
            float* h2 = sh + (1 * kGradTile + j) * kRow;
            float* h3 = sh + (2 * kGradTile + j) * kRow;
            float* e1 = sd + (0 * kGradTile + j) * kRow;
            float* e2 = sd + (1 * kGradTile + j) * kRow;
            float* e3 = sd + (2 * kGradTile + j) * kRow;
            if (p < n) {
                const int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((size_t)nx * ny));
                float o[3];
                // forward, keeping inputs, activations and GELU slopes (slopes in the error rows)
                net_point<float, true>(sw, u, x, y, z, nx, ny, nz, n, hx, h1, h2, h3, e1, e2, e3, o);
                float eo[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float r = o[c] - tau[c * n + p];
                    sse = fmaf(r, r, sse);
                    eo[c] = 2.0f * r * inv;
                    so[j * 3 + c] = eo[c];
                }
                // dz3 = (W4^T eo) * gelu'(z3); dz2 = (W3^T dz3) * gelu'(z2); dz1 = (W2^T dz2) * gelu'(z1),
                // each overwriting the slopes in place
                for (int i = 0; i < kNetC; ++i) {
                    float s = 0.0f;
#pragma unroll
                    for (int c = 0; c < 3; ++c) s = fmaf(sw[kOffW4 + c * kNetC + i], eo[c], s);
                    e3[i] *= s;
                }
                for (int i = 0; i < kNetC; ++i) {
                    float s = 0.0f;
                    for (int o2 = 0; o2 < kNetC; ++o2) s = fmaf(sw[kOffW3 + o2 * kNetC + i], e3[o2], s);
                    e2[i] *= s;
                }
                for (int i = 0; i < kNetC; ++i) {
                    float s = 0.0f;
                    for (int o2 = 0; o2 < kNetC; ++o2) s = fmaf(sw[kOffW2 + o2 * kNetC + i], e2[o2], s);
                    e1[i] *= s;
                }
            } else {
                for (int i = 0; i < kNetIn; ++i) hx[i] = 0.0f;
                for (int i = 0; i < kNetC; ++i) h1[i] = h2[i] = h3[i] = e1[i] = e2[i] = e3[i] = 0.0f;
                for (int c = 0; c < 3; ++c) so[j * 3 + c] = 0.0f;
            }
        }
        __syncthreads();
        // weight gradients: thread t owns parameters q = t + k*kGradNT; sums over the tile in order
#pragma unroll
        for (int k = 0; k < kGradPer; ++k) {
            const int q = threadIdx.x + k * kGradNT;
            if (q >= kNetNP) break;
            float s = 0.0f;
            if (q < kOffB1) {
                const int o = q / kNetIn, i = q - o * kNetIn;
                for (int jj = 0; jj < kGradTile; ++jj) s = fmaf(sd[(0 * kGradTile + jj) * kRow + o], sx[jj * kNetIn + i], s);
            } else if (q < kOffW2) {
                const int o = q - kOffB1;
                for (int jj = 0; jj < kGradTile; ++jj) s += sd[(0 * kGradTile + jj) * kRow + o];
            } else if (q < kOffB2) {
                const int o = (q - kOffW2) / kNetC, i = (q - kOffW2) % kNetC;
                for (int jj = 0; jj < kGradTile; ++jj)
                    s = fmaf(sd[(1 * kGradTile + jj) * kRow + o], sh[(0 * kGradTile + jj) * kRow + i], s);
            } else if (q < kOffW3) {
                const int o = q - kOffB2;
                for (int jj = 0; jj < kGradTile; ++jj) s += sd[(1 * kGradTile + jj) * kRow + o];
            } else if (q < kOffB3) {
                const int o = (q - kOffW3) / kNetC, i = (q - kOffW3) % kNetC;
                for (int jj = 0; jj < kGradTile; ++jj)
                    s = fmaf(sd[(2 * kGradTile + jj) * kRow + o], sh[(1 * kGradTile + jj) * kRow + i], s);
            } else if (q < kOffW4) {
                const int o = q - kOffB3;
                for (int jj = 0; jj < kGradTile; ++jj) s += sd[(2 * kGradTile + jj) * kRow + o];
            } else if (q < kOffB4) {
                const int o = (q - kOffW4) / kNetC, i = (q - kOffW4) % kNetC;
                for (int jj = 0; jj < kGradTile; ++jj) s = fmaf(so[jj * 3 + o], sh[(2 * kGradTile + jj) * kRow + i], s);
            } else {
                const int o = q - kOffB4;
                for (int jj = 0; jj < kGradTile; ++jj) s += so[jj * 3 + o];
            }
            g[k] += s;
        }
        __syncthreads();
    }
    float* dst = part + (size_t)blockIdx.x * (kNetNP + 1);
#pragma unroll
    for (int k = 0; k < kGradPer; ++k) {
        const int q = threadIdx.x + k * kGradNT;
        if (q < kNetNP) dst[q] = g[k];
    }
    // block sum of squared errors (fixed order)
    sr[threadIdx.x] = sse;
    __syncthreads();
    for (int s = kGradNT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sr[threadIdx.x] += sr[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) dst[kNetNP] = sr[0];
}

constexpr size_t kGradSmem = (size_t)(((kNetNP + 3) & ~3) + kGradTile * kNetIn + 6 * kGradTile * kRow +
                                      kGradTile * 3 + kGradNT) * sizeof(float);

// grad[q] = sum over blocks of part[b][q] in block order; loss = sum of the squared errors / (3 n).
__global__ void k_net_reduce(const float* __restrict__ part, int nblk, float* __restrict__ grad,
                             double* __restrict__ loss, double inv_count) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q > kNetNP) return;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += (double)part[(size_t)b * (kNetNP + 1) + q];
    if (q < kNetNP) grad[q] = (float)s;
    else if (loss) *loss = s * inv_count;
}

// Adam step (Kingma & Ba 2015) on the FP32 master weights; writes their BF16 copy.
__global__ void k_net_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, float* __restrict__ m,
                           float* __restrict__ v, const float* __restrict__ g, int t, float lr, float b1, float b2,
                           float eps) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kNetNP) return;
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    const float mh = mq / (1.0f - powf(b1, (float)t)), vh = vq / (1.0f - powf(b2, (float)t));
    const float wq = w[q] - lr * mh / (sqrtf(vh) + eps);
    w[q] = wq;
    wb[q] = __float2bfloat16_rn(wq);
}

// u <- u - dt * tau_hat at every point (u: the handle's physical field [3][n], FP64).
__global__ void k_closure_update(double* __restrict__ u, const float* __restrict__ tau, size_t n3, double dt) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x)
        u[i] -= dt * (double)tau[i];
}

}  // namespace bastr
