// Learned closure: a stencil MLP that predicts the liquid closure's per-cell velocity
// correction from the red (post-redistribution) occupancy and mean-velocity fields.
//
//   features (75): a 5x5 stencil around the cell of N/gamma - 1, Ux, Uy of the red state
//                  (channel-major, dy outer, dx inner; wrapped on periodic axes, zero outside
//                  the walls)
//   target (2)   : the plain closure's kick, beta_applied * duRepair + duEOS
//                  (reference src/liquid_closure.cpp:380-389, :424-436), in velocity units
//   network      : 75 -> 64 -> 64 -> 2, GELU, weights rounded to BF16, FP32 accumulation;
//                  kick = output * scale
//
// Parameters live in one float array: W1[64][75], b1[64], W2[64][64], b2[64], W3[2][64], b3[2],
// scale. Training (k_mlp_grad + k_adam) keeps FP32 master weights and fits output = target /
// scale; every forward pass, in training and in the step, uses the weights' BF16 roundings.
// The scale is not trained (the trainer sets it to the targets' RMS).
#pragma once

#include <cuda_bf16.h>

#include "closure.cuh"
#include "common.cuh"

namespace mpcd_dev {

constexpr int kFeat = 75, kHid = 64, kOut = 2;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kFeat, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kOut * kHid, kOffScale = kOffB3 + kOut,
              kTrained = kOffScale, kParams = kOffScale + 1;  // 9154 trained + the output scale

__device__ __forceinline__ float bf16r(float w) { return __bfloat162float(__float2bfloat16_rn(w)); }
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// the stencil features of cell c
__device__ __forceinline__ void cell_features(const DevParams& P, const int* __restrict__ N, const double* __restrict__ Ux,
                                              const double* __restrict__ Uy, int c, float* f) {
    const int ix = c / P.Ny, iy = c - ix * P.Ny;
    int k = 0;
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx, ++k) {
            int jx = ix + dx, jy = iy + dy;
            bool in = true;
            if (P.perx) jx = wrap_index(jx, P.Nx);
            else in = in && jx >= 0 && jx < P.Nx;
            if (P.pery) jy = wrap_index(jy, P.Ny);
            else in = in && jy >= 0 && jy < P.Ny;
            float n = 0.0f, ux = 0.0f, uy = 0.0f;
            if (in) {
                const int q = jy + P.Ny * jx;
                n = (float)__dsub_rn(__ddiv_rn((double)N[q], P.gamma), 1.0);
                ux = (float)Ux[q];
                uy = (float)Uy[q];
            } else {
                n = -1.0f;
            }
            f[k] = n;
            f[25 + k] = ux;
            f[50 + k] = uy;
        }
}

// the network on one feature row (weights: BF16 in shared memory)
__device__ __forceinline__ void mlp_forward(const __nv_bfloat16* __restrict__ sw, const float* f, float& o0, float& o1) {
    float h1[kHid];
#pragma unroll 4
    for (int j = 0; j < kHid; ++j) {
        float z = __bfloat162float(sw[kOffB1 + j]);
#pragma unroll
        for (int k = 0; k < kFeat; ++k) z = fmaf(__bfloat162float(sw[kOffW1 + j * kFeat + k]), f[k], z);
        h1[j] = gelu(z);
    }
    o0 = __bfloat162float(sw[kOffB3]);
    o1 = __bfloat162float(sw[kOffB3 + 1]);
#pragma unroll 4
    for (int j = 0; j < kHid; ++j) {
        float z = __bfloat162float(sw[kOffB2 + j]);
#pragma unroll
        for (int k = 0; k < kHid; ++k) z = fmaf(__bfloat162float(sw[kOffW2 + j * kHid + k]), h1[k], z);
        const float a = gelu(z);
        o0 = fmaf(__bfloat162float(sw[kOffW3 + j]), a, o0);
        o1 = fmaf(__bfloat162float(sw[kOffW3 + kHid + j]), a, o1);
    }
}

__device__ __forceinline__ void stage_weights(const float* __restrict__ params, __nv_bfloat16* sw) {
    for (int i = threadIdx.x; i < kTrained; i += blockDim.x) sw[i] = __float2bfloat16_rn(params[i]);
}

// features and targets of every stride-th cell from offset (dataset collection)
__global__ void k_learned_samples(DevParams P, const int* __restrict__ N, const double* __restrict__ Ux,
                                  const double* __restrict__ Uy, const double* __restrict__ duRX,
                                  const double* __restrict__ duRY, const double* __restrict__ eosX,
                                  const double* __restrict__ eosY, const double* __restrict__ red, int stride, int offset,
                                  int count, float* __restrict__ X, float* __restrict__ Y) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const int c = offset + s * stride;
    if (c >= P.Nc) return;
    cell_features(P, N, Ux, Uy, c, X + (size_t)s * kFeat);
    const double beta = beta_applied(P, red[0], red[1]);
    Y[2 * (size_t)s] = (float)__dadd_rn(__dmul_rn(beta, duRX[c]), eosX[c]);
    Y[2 * (size_t)s + 1] = (float)__dadd_rn(__dmul_rn(beta, duRY[c]), eosY[c]);
}

// One block: forward and backward of kMlpTile samples (rows idx[blockIdx.x * kMlpTile ..] of
// X and Y), accumulating the gradient of the mean squared error of output - Y * yinv over the
// batch (batch rows, 2 outputs each) into grad (atomics) and the loss into loss[0].
constexpr int kMlpTile = 16, kMlpThreads = 256;
__global__ void __launch_bounds__(kMlpThreads) k_mlp_grad(const float* __restrict__ X, const float* __restrict__ Y,
                                                          const int* __restrict__ idx, int rows, int batch, float yinv,
                                                          const float* __restrict__ params, float* __restrict__ grad,
                                                          float* __restrict__ loss) {
    __shared__ __nv_bfloat16 sw[kTrained];
    __shared__ float x[kMlpTile][kFeat + 1];
    __shared__ float z1[kMlpTile][kHid], a1[kMlpTile][kHid], z2[kMlpTile][kHid], a2[kMlpTile][kHid];
    __shared__ float dout[kMlpTile][kOut];
    const int t = threadIdx.x;
    const int r0 = blockIdx.x * kMlpTile;
    const int nr = min(kMlpTile, rows - r0);
    stage_weights(params, sw);
    for (int i = t; i < kMlpTile * kFeat; i += blockDim.x) {
        const int r = i / kFeat, k = i - r * kFeat;
        x[r][k] = (r < nr) ? X[(size_t)idx[r0 + r] * kFeat + k] : 0.0f;
    }
    __syncthreads();
    for (int i = t; i < kMlpTile * kHid; i += blockDim.x) {
        const int r = i / kHid, j = i - r * kHid;
        float z = __bfloat162float(sw[kOffB1 + j]);
        for (int k = 0; k < kFeat; ++k) z = fmaf(__bfloat162float(sw[kOffW1 + j * kFeat + k]), x[r][k], z);
        z1[r][j] = z;
        a1[r][j] = gelu(z);
    }
    __syncthreads();
    for (int i = t; i < kMlpTile * kHid; i += blockDim.x) {
        const int r = i / kHid, j = i - r * kHid;
        float z = __bfloat162float(sw[kOffB2 + j]);
        for (int k = 0; k < kHid; ++k) z = fmaf(__bfloat162float(sw[kOffW2 + j * kHid + k]), a1[r][k], z);
        z2[r][j] = z;
        a2[r][j] = gelu(z);
    }
    __syncthreads();
    if (t < kMlpTile * kOut) {
        const int r = t / kOut, o = t - r * kOut;
        float z = __bfloat162float(sw[kOffB3 + o]);
        for (int k = 0; k < kHid; ++k) z = fmaf(__bfloat162float(sw[kOffW3 + o * kHid + k]), a2[r][k], z);
        float d = 0.0f;
        if (r < nr) {
            const float e = z - Y[(size_t)idx[r0 + r] * kOut + o] * yinv;
            d = 2.0f * e / (float)(batch * kOut);  // d(mean squared error)/d(output)
            atomicAdd(loss, e * e / (float)(batch * kOut));
        }
        dout[r][o] = d;
    }
    __syncthreads();
    // layer 3: dW3, db3; da2 -> dz2 (kept in z2)
    for (int i = t; i < kOut * kHid; i += blockDim.x) {
        const int o = i / kHid, k = i - o * kHid;
        float g = 0.0f;
        for (int r = 0; r < kMlpTile; ++r) g = fmaf(dout[r][o], a2[r][k], g);
        atomicAdd(grad + kOffW3 + i, g);
    }
    if (t < kOut) {
        float g = 0.0f;
        for (int r = 0; r < kMlpTile; ++r) g += dout[r][t];
        atomicAdd(grad + kOffB3 + t, g);
    }
    __syncthreads();
    for (int i = t; i < kMlpTile * kHid; i += blockDim.x) {
        const int r = i / kHid, k = i - r * kHid;
        float d = 0.0f;
        for (int o = 0; o < kOut; ++o) d = fmaf(dout[r][o], __bfloat162float(sw[kOffW3 + o * kHid + k]), d);
        z2[r][k] = d * gelu_d(z2[r][k]);
    }
    __syncthreads();
    // layer 2: dW2, db2; da1 -> dz1 (kept in z1)
    for (int i = t; i < kHid * kHid; i += blockDim.x) {
        const int j = i / kHid, k = i - j * kHid;
        float g = 0.0f;
        for (int r = 0; r < kMlpTile; ++r) g = fmaf(z2[r][j], a1[r][k], g);
        atomicAdd(grad + kOffW2 + i, g);
    }
    if (t < kHid) {
        float g = 0.0f;
        for (int r = 0; r < kMlpTile; ++r) g += z2[r][t];
        atomicAdd(grad + kOffB2 + t, g);
    }
    __syncthreads();
    for (int i = t; i < kMlpTile * kHid; i += blockDim.x) {
        const int r = i / kHid, k = i - r * kHid;
        float d = 0.0f;
        for (int j = 0; j < kHid; ++j) d = fmaf(z2[r][j], __bfloat162float(sw[kOffW2 + j * kHid + k]), d);
        z1[r][k] = d * gelu_d(z1[r][k]);
    }
    __syncthreads();
    // layer 1: dW1, db1
    for (int i = t; i < kHid * kFeat; i += blockDim.x) {
        const int j = i / kFeat, k = i - j * kFeat;
        float g = 0.0f;
        for (int r = 0; r < kMlpTile; ++r) g = fmaf(z1[r][j], x[r][k], g);
        atomicAdd(grad + kOffW1 + i, g);
    }
    if (t < kHid) {
        float g = 0.0f;
        for (int r = 0; r < kMlpTile; ++r) g += z1[r][t];
        atomicAdd(grad + kOffB1 + t, g);
    }
}

// Adam (Kingma & Ba) on the FP32 master weights; clears the gradient for the next batch.
__global__ void k_adam(float* __restrict__ params, float* __restrict__ grad, float* __restrict__ m, float* __restrict__ v,
                       int count, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    grad[i] = 0.0f;
}

// The learned kick of every cell of the red state, one thread per cell with the BF16-rounded
// weights in shared memory.
__global__ void __launch_bounds__(128) k_learned_cells(DevParams P, const int* __restrict__ N, const double* __restrict__ Ux,
                                                       const double* __restrict__ Uy, const float* __restrict__ params,
                                                       double* __restrict__ duX, double* __restrict__ duY,
                                                       const int* __restrict__ mode) {
    if (mode && *mode == 0) return;  // this step runs the plain closure
    __shared__ __nv_bfloat16 sw[kTrained];
    stage_weights(params, sw);
    __syncthreads();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.Nc) return;
    float f[kFeat];
    cell_features(P, N, Ux, Uy, c, f);
    float o0, o1;
    mlp_forward(sw, f, o0, o1);
    const float scale = params[kOffScale];
    duX[c] = (double)(o0 * scale);
    duY[c] = (double)(o1 * scale);
}

// The network on feature rows (inference check): out[r] = output * scale.
__global__ void __launch_bounds__(128) k_mlp_rows(const float* __restrict__ X, int rows, const float* __restrict__ params,
                                                  float* __restrict__ out) {
    __shared__ __nv_bfloat16 sw[kTrained];
    stage_weights(params, sw);
    __syncthreads();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float f[kFeat];
    for (int k = 0; k < kFeat; ++k) f[k] = X[(size_t)r * kFeat + k];
    float o0, o1;
    mlp_forward(sw, f, o0, o1);
    const float scale = params[kOffScale];
    out[2 * (size_t)r] = o0 * scale;
    out[2 * (size_t)r + 1] = o1 * scale;
}

// Mode of the next step from the occupancy spread of this step's red state: learned (1) while
// occStd <= limit (or no limit), plain (0) otherwise. sums: (sum N, sum N^2) over the cells.
// counters[mode of this step] += 1.
__global__ void k_learned_decide(const double* __restrict__ sums, int Nc, double gamma, double limit, int* mode,
                                 long long* counters) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    counters[*mode ? 1 : 0] += 1;
    const double N = (double)(Nc > 0 ? Nc : 1);
    const double mean = sums[0] / N;
    double var = sums[1] / N - mean * mean;
    if (var < 0.0) var = 0.0;
    const double occStd = sqrt(var) / (gamma > 1e-12 ? gamma : 1e-12);
    *mode = (limit <= 0.0 || occStd <= limit) ? 1 : 0;
}

}  // namespace mpcd_dev
