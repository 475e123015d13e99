// Learned subgrid closure for the coarse 3D solve: a small local network that maps the
// filtered velocity u (3 channels) to the subgrid term tau = filter(u.grad u) - u.grad u.
//
//   layer 1  3x3x3 periodic stencil, 3 -> 32 channels, GELU
//   layer 2  1x1x1, 32 -> 32, GELU
//   layer 3  1x1x1, 32 -> 32, GELU
//   layer 4  1x1x1, 32 -> 3
//
// Weights are BF16 (rounded once from FP32 master weights by the optimizer), every sum is
// accumulated in FP32.  GELU is the tanh form 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))).
// Parameter layout (NP = 4835 floats): W1[32][81] (input tap i = c*27 + (dz+1)*9 + (dy+1)*3 +
// (dx+1)), b1[32], W2[32][32], b2[32], W3[32][32], b3[32], W4[3][32], b4[3].
//
// Training: k_net_grad runs the forward pass for tiles of 64 points, keeps every point's
// activations and back-propagated errors in shared memory, and accumulates the weight
// gradients of its tiles in registers (each thread owns fixed parameters and sums over points
// in a fixed order); the per-block partials are summed in fixed order by k_net_reduce, so a
// gradient is deterministic.  k_net_adam updates the FP32 master weights and their BF16 copy.
#pragma once
#include <cuda_bf16.h>
#include "solver.cuh"

namespace bastr {

constexpr int kNetC = 32, kNetIn = 81;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kNetC * kNetIn, kOffW2 = kOffB1 + kNetC, kOffB2 = kOffW2 + kNetC * kNetC,
              kOffW3 = kOffB2 + kNetC, kOffB3 = kOffW3 + kNetC * kNetC, kOffW4 = kOffB3 + kNetC,
              kOffB4 = kOffW4 + 3 * kNetC, kNetNP = kOffB4 + 3;

__device__ __forceinline__ float gelu_t(float z, float& dg) {
    const float a = 0.7978845608028654f, c = 0.044715f;
    const float t = tanhf(a * (z + c * z * z * z));
    dg = 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * a * (1.0f + 3.0f * c * z * z);
    return 0.5f * z * (1.0f + t);
}

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
        const float xi = tap(u, i / 27, x, y, z, i % 27, nx, ny, nz, n);
        if constexpr (GRAD) X[i] = xi;
#pragma unroll
        for (int o = 0; o < kNetC; ++o) a[o] = fmaf(sw[kOffW1 + o * kNetIn + i], xi, a[o]);
    }
#pragma unroll
    for (int o = 0; o < kNetC; ++o) {
        float d;
        a[o] = gelu_t(a[o], d);
        if constexpr (GRAD) { H1[o] = a[o]; D1[o] = d; }
    }
#pragma unroll
    for (int o = 0; o < kNetC; ++o) {
        float s = sw[kOffB2 + o];
#pragma unroll
        for (int i = 0; i < kNetC; ++i) s = fmaf(sw[kOffW2 + o * kNetC + i], a[i], s);
        float d;
        b[o] = gelu_t(s, d);
        if constexpr (GRAD) { H2[o] = b[o]; D2[o] = d; }
    }
#pragma unroll
    for (int o = 0; o < kNetC; ++o) {
        float s = sw[kOffB3 + o];
#pragma unroll
        for (int i = 0; i < kNetC; ++i) s = fmaf(sw[kOffW3 + o * kNetC + i], b[i], s);
        float d;
        a[o] = gelu_t(s, d);
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

// out[c][p] = scale * net(u)[c] at every point.
template <typename TI>
__global__ void __launch_bounds__(128) k_net_forward(const TI* __restrict__ u, const __nv_bfloat16* __restrict__ w,
                                                     float* __restrict__ out, int nx, int ny, int nz, float scale) {
    __shared__ float sw[kNetNP];
    load_weights(sw, w);
    __syncthreads();
    const size_t n = (size_t)nx * ny * nz;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((size_t)nx * ny));
        float o[3];
        net_point<TI, false>(sw, u, x, y, z, nx, ny, nz, n, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                             nullptr, o);
#pragma unroll
        for (int c = 0; c < 3; ++c) out[c * n + p] = scale * o[c];
    }
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
