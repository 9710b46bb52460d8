// Learned closure: a stencil MLP that predicts the liquid closure's per-cell velocity
// correction from the red (post-redistribution) occupancy and mean-velocity fields.
//
//   features (75): a 5x5 stencil around the cell of N/gamma - 1, Ux - <Ux>, Uy - <Uy> of the
//                  red state, <.> the mean over the stencil's cells inside the walls
//                  (channel-major, dy outer, dx inner; wrapped on periodic axes; a point
//                  beyond a wall gives N term -1 and velocity terms 0). Velocities relative to
//                  the stencil mean make the network blind to a uniform flow, as the closure is.
//   kick         : the network's output per cell less its particle mean (sum of N du over the
//                  cells / n), so the learned kick conserves momentum
//   target (2)   : the plain closure's kick, beta_applied * duRepair + duEOS
//                  (reference src/liquid_closure.cpp:380-389, :424-436), in velocity units
//   network      : 75 -> 64 -> 64 -> 2, GELU (tanh form); kick = output * scale
//                  z1 = W1 bf(x) + b1, a1 = gelu(z1); z2 = W2 bf(a1) + b2, a2 = gelu(z2);
//                  output = W3 a2 + b3, with every weight and bias rounded to BF16 (bf) and
//                  FP32 accumulation: the operands of the two 64-wide layers are BF16 (they
//                  run on the tensor cores), the 64 -> 2 output layer takes a2 in FP32
//
// Parameters live in one float array: W1[64][75], b1[64], W2[64][64], b2[64], W3[2][64], b3[2],
// scale. Training (k_mlp_grad_tc on the tensor cores + k_adam) keeps FP32 master weights and fits output = target /
// scale (gradients pass straight through the BF16 roundings). The scale is not trained (the
// trainer sets it to the targets' RMS).
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
// GELU in the tanh form of Hendrycks and Gimpel, written as z * sigmoid(2u) with
// u = sqrt(2/pi) (z + 0.044715 z^3) (0.5 (1 + tanh u) = sigmoid(2u))
constexpr float kGeluC2 = 1.5957691216057308f;  // 2 sqrt(2/pi)
constexpr float kGeluA = 0.044715f;
__device__ __forceinline__ float gelu_sig(float z) {
    return __fdividef(1.0f, 1.0f + __expf(-kGeluC2 * fmaf(kGeluA * z, z * z, z)));
}
__device__ __forceinline__ float gelu(float z) { return z * gelu_sig(z); }
__device__ __forceinline__ float gelu_d(float z) {
    const float s = gelu_sig(z);
    return fmaf(z * s * (1.0f - s), kGeluC2 * fmaf(3.0f * kGeluA, z * z, 1.0f), s);
}

// Pairs of FP32 values in one 64-bit register, for the packed f32x2 arithmetic of sm_100a
// (per element the IEEE rounding of the scalar instruction, two elements per issue).
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
// GELU of a pair, the tanh form as z * sigmoid(2u) = z / (1 + 2^(-2u log2 e)): the power by
// ex2.approx, the quotient by rcp.approx (the special-function unit, one value per issue),
// the rest packed
constexpr float kGeluE = (float)(-1.5957691216057308 * 1.4426950408889634);  // -2 sqrt(2/pi) log2(e)
__device__ __forceinline__ f32x2 gelu2(f32x2 z) {
    const f32x2 t = f2_fma(f2_mul(z, f2_pack(kGeluA, kGeluA)), f2_mul(z, z), z);  // z + a z^3
    float e0, e1;
    f2_unpack(f2_mul(t, f2_pack(kGeluE, kGeluE)), e0, e1);
    asm("ex2.approx.ftz.f32 %0, %0;" : "+f"(e0));
    asm("ex2.approx.ftz.f32 %0, %0;" : "+f"(e1));
    float d0, d1;
    f2_unpack(f2_add(f2_pack(e0, e1), f2_pack(1.0f, 1.0f)), d0, d1);
    asm("rcp.approx.ftz.f32 %0, %0;" : "+f"(d0));
    asm("rcp.approx.ftz.f32 %0, %0;" : "+f"(d1));
    return f2_mul(z, f2_pack(d0, d1));
}

// Stencil of cell c: start of each column jx (-1 beyond a wall) and each row jy (-1), and the
// mean velocity over the points inside the walls.
struct Stencil {
    int col[5], row[5];
    float mx, my;
};

__device__ __forceinline__ Stencil stencil_of(const DevParams& P, const float4* __restrict__ feat, int c) {
    Stencil S;
    const int ix = c / P.Ny, iy = c - ix * P.Ny;
#pragma unroll
    for (int d = 0; d < 5; ++d) {
        int jx = ix + d - 2, jy = iy + d - 2;
        if (P.perx) jx = wrap_index(jx, P.Nx);
        S.col[d] = (jx >= 0 && jx < P.Nx) ? jx * P.Ny : -1;
        if (P.pery) jy = wrap_index(jy, P.Ny);
        S.row[d] = (jy >= 0 && jy < P.Ny) ? jy : -1;
    }
    float sx = 0.0f, sy = 0.0f;
    int cnt = 0;
#pragma unroll
    for (int dy = 0; dy < 5; ++dy)
#pragma unroll
        for (int dx = 0; dx < 5; ++dx)
            if (S.col[dx] >= 0 && S.row[dy] >= 0) {
                const float4 q = __ldg(feat + S.col[dx] + S.row[dy]);
                sx += q.y;
                sy += q.z;
                ++cnt;
            }
    S.mx = sx / (float)cnt;  // the cell itself is always inside
    S.my = sy / (float)cnt;
    return S;
}

// The layer-1 operands of cell c as BF16 pairs: operand column k is channel k % 3 of stencil
// point k / 3 (the values stencil_value gives, the stencil mean taken in the same order as
// stencil_of), column 75 the bias input 1, columns 76-79 zero. The 25 points are read twice
// (the mean, then the values), each as one float4.
template <int kCols>
__device__ __forceinline__ void stencil_operands(const DevParams& P, const float4* __restrict__ feat, int c,
                                                 uint32_t (&w)[kCols / 2]) {
    const int ix = c / P.Ny, iy = c - ix * P.Ny;
    int col[5], row[5];
#pragma unroll
    for (int d = 0; d < 5; ++d) {
        int jx = ix + d - 2, jy = iy + d - 2;
        if (P.perx) jx = wrap_index(jx, P.Nx);
        col[d] = (jx >= 0 && jx < P.Nx) ? jx * P.Ny : -1;
        if (P.pery) jy = wrap_index(jy, P.Ny);
        row[d] = (jy >= 0 && jy < P.Ny) ? jy : -1;
    }
    float sx = 0.0f, sy = 0.0f;
    int cnt = 0;
#pragma unroll
    for (int pnt = 0; pnt < 25; ++pnt) {
        const int dy = pnt / 5, dx = pnt % 5;
        if (col[dx] >= 0 && row[dy] >= 0) {
            const float4 q = __ldg(feat + col[dx] + row[dy]);
            sx += q.y;
            sy += q.z;
            ++cnt;
        }
    }
    const float mx = sx / (float)cnt, my = sy / (float)cnt;  // the cell itself is always inside
    float op[kCols];
#pragma unroll
    for (int pnt = 0; pnt < 25; ++pnt) {
        const int dy = pnt / 5, dx = pnt % 5;
        float a0 = -1.0f, a1 = 0.0f, a2 = 0.0f;
        if (col[dx] >= 0 && row[dy] >= 0) {
            const float4 q = __ldg(feat + col[dx] + row[dy]);
            a0 = q.x;
            a1 = q.y - mx;
            a2 = q.z - my;
        }
        op[3 * pnt] = a0;
        op[3 * pnt + 1] = a1;
        op[3 * pnt + 2] = a2;
    }
#pragma unroll
    for (int k = 75; k < kCols; ++k) op[k] = k == 75 ? 1.0f : 0.0f;
#pragma unroll
    for (int j = 0; j < kCols / 2; ++j) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(op[2 * j], op[2 * j + 1]);
        w[j] = *reinterpret_cast<const uint32_t*>(&h);
    }
}

// channel ch (0 N, 1 Ux, 2 Uy) of stencil point pnt (5 dy + dx)
__device__ __forceinline__ float stencil_value(const Stencil& S, const float4* __restrict__ feat, int pnt, int ch) {
    const int dy = pnt / 5, dx = pnt - 5 * dy;
    if (S.col[dx] < 0 || S.row[dy] < 0) return ch == 0 ? -1.0f : 0.0f;
    const float* q = reinterpret_cast<const float*>(feat + S.col[dx] + S.row[dy]);
    const float val = __ldg(q + ch);
    return ch == 0 ? val : val - (ch == 1 ? S.mx : S.my);
}

// the stencil features of cell c (channel-major)
__device__ __forceinline__ void cell_features(const DevParams& P, const float4* __restrict__ feat, int c, float* f) {
    const Stencil S = stencil_of(P, feat, c);
    for (int ch = 0; ch < 3; ++ch)
        for (int k = 0; k < 25; ++k) f[25 * ch + k] = stencil_value(S, feat, k, ch);
}

// training samples of the fast form's learned closure: the stencil features of every
// stride-th cell from offset (the collided state's occupancy, kinetic pressure and mean vx),
// and the plain closure's EOS kick there (the part the network replaces)
__global__ void k_fast_learned_samples(DevParams P, const float4* __restrict__ feat, const double* __restrict__ eosX,
                                       const double* __restrict__ eosY, int stride, int offset, int count,
                                       float* __restrict__ X, float* __restrict__ Y) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const int c = offset + s * stride;
    if (c >= P.Nc) return;
    cell_features(P, feat, c, X + (size_t)s * kFeat);
    Y[2 * (size_t)s] = (float)eosX[c];
    Y[2 * (size_t)s + 1] = (float)eosY[c];
}

// features and targets of every stride-th cell from offset (dataset collection)
__global__ void k_learned_samples(DevParams P, const float4* __restrict__ feat, const double* __restrict__ duRX,
                                  const double* __restrict__ duRY, const double* __restrict__ eosX,
                                  const double* __restrict__ eosY, const double* __restrict__ red, int stride, int offset,
                                  int count, float* __restrict__ X, float* __restrict__ Y) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const int c = offset + s * stride;
    if (c >= P.Nc) return;
    cell_features(P, feat, c, X + (size_t)s * kFeat);
    const double beta = beta_applied(P, red[0], red[1]);
    Y[2 * (size_t)s] = (float)__dadd_rn(__dmul_rn(beta, duRX[c]), eosX[c]);
    Y[2 * (size_t)s + 1] = (float)__dadd_rn(__dmul_rn(beta, duRY[c]), eosY[c]);
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

// ---------------------------------------------------------------- tensor-core inference
// One CTA of 128 threads runs tiles of 128 rows (cells, or feature rows): thread t owns row t,
// which is TMEM lane t of the accumulators. Per tile:
//   1. every thread writes its row's 80 layer-1 operands to shared memory as BF16: the 75
//      features point-major (operand column 3p + ch holds channel ch of stencil point p, so a
//      point's three values are written together), a constant 1 that carries b1, 4 zeros;
//   2. one thread issues 5 tcgen05.mma (M=128, N=64, K=16) into TMEM columns [0, 64);
//   3. every thread loads its 64 accumulators (tcgen05.ld), applies GELU and writes a1 as BF16;
//   4. one thread issues 4 tcgen05.mma into TMEM columns [64, 128);
//   5. every thread loads z2, adds b2, applies GELU and runs the 64 -> 2 layer in FP32.
// Operands use the canonical K-major layout without swizzle: 8x8 core matrices (8 rows of
// 16 bytes, stored contiguously), adjacent along K at 128 bytes (LBO), 8-row groups at
// K * 16 bytes (SBO).
constexpr int kTcRows = 128, kTcThreads = 128, kTcK1 = 80;
constexpr uint32_t kTcOffA = 0;                                  // [128][80] bf16
constexpr uint32_t kTcOffH = kTcOffA + kTcRows * kTcK1 * 2;       // [128][64] bf16
constexpr uint32_t kTcOffW1 = kTcOffH + kTcRows * kHid * 2;       // [64][80] bf16 (b1 in column 75)
constexpr uint32_t kTcOffW2 = kTcOffW1 + kHid * kTcK1 * 2;        // [64][64] bf16
constexpr uint32_t kTcOffB2 = kTcOffW2 + kHid * kHid * 2;         // [64] f32
constexpr uint32_t kTcOffW3 = kTcOffB2 + kHid * 4;                // [2][64] f32
constexpr uint32_t kTcOffB3 = kTcOffW3 + kOut * kHid * 4;         // b3[2], scale, pad: f32
constexpr uint32_t kTcOffBar = kTcOffB3 + 16;                     // mbarrier (8 bytes)
constexpr uint32_t kTcOffTmem = kTcOffBar + 8;                    // TMEM base address
constexpr uint32_t kTcSmem = kTcOffTmem + 8;
constexpr uint32_t kTcTmemCols = 128;
constexpr int kTcSpinLimit = 1 << 22;
// Shared memory bounds the CTAs per SM to 4, so their TMEM (4 x 128 columns) always fits.
static_assert(5 * (kTcSmem + 1024) > 228 * 1024, "more than 4 CTAs per SM would oversubscribe TMEM");

// instruction descriptor, kind::f16: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kHid >> 3) << 17) |
                              ((uint32_t)(kTcRows >> 4) << 24);

__host__ __device__ constexpr uint32_t kmajor_offset(int r, int k, int K) {
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start, LBO, SBO (all >> 4), version 1 (bit 46), no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool tc_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for the barrier phase; false when the limit ran out
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < kTcSpinLimit; ++i)
        if (tc_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 accumulator columns of this thread's lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}
// completes the loads; the registers are tied to it so no use is scheduled earlier
__device__ __forceinline__ void tc_ld_wait16(uint32_t* r) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]) :: "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Inference on tiles of 128 rows. kRows: rows of X (count rows), out[2 r] = kick; else the
// cells of the red state, features gathered from feat, kick written to duX, duY (and
// nothing when *mode == 0: the step runs the plain closure).
template <bool kRows>
__global__ void __launch_bounds__(kTcThreads, 4)
    k_mlp_tc(DevParams P, const float4* __restrict__ feat, const float* __restrict__ X, int rows, const float* __restrict__ params, double* __restrict__ duX,
             double* __restrict__ duY, float* __restrict__ out, const int* __restrict__ mode,
             unsigned long long* __restrict__ duSum, int bulkOnly, DevStatus* st) {
    if (!kRows && mode && *mode == 0) return;
    extern __shared__ __align__(128) unsigned char sm[];
    const int t = threadIdx.x, warp = t >> 5;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const uint32_t bar = sbase + kTcOffBar;
    float* sB2 = reinterpret_cast<float*>(sm + kTcOffB2);
    float* sW3 = reinterpret_cast<float*>(sm + kTcOffW3);
    float* sB3 = reinterpret_cast<float*>(sm + kTcOffB3);
    // weights once per CTA (W1's columns in the point-major operand order)
    for (int i = t; i < kHid * kTcK1; i += kTcThreads) {
        const int n = i / kTcK1, k = i - n * kTcK1;
        const int pk = (k % 3) * 25 + k / 3;  // parameter column of operand column k
        const float w = k < kFeat ? params[kOffW1 + n * kFeat + pk] : (k == kFeat ? params[kOffB1 + n] : 0.0f);
        *reinterpret_cast<__nv_bfloat16*>(sm + kTcOffW1 + kmajor_offset(n, k, kTcK1)) = __float2bfloat16_rn(w);
    }
    for (int i = t; i < kHid * kHid; i += kTcThreads) {
        const int n = i / kHid, k = i - n * kHid;
        *reinterpret_cast<__nv_bfloat16*>(sm + kTcOffW2 + kmajor_offset(n, k, kHid)) =
            __float2bfloat16_rn(params[kOffW2 + i]);
    }
    if (t < kHid) sB2[t] = bf16r(params[kOffB2 + t]);
    for (int i = t; i < kOut * kHid; i += kTcThreads) sW3[i] = bf16r(params[kOffW3 + i]);
    if (t < kOut) sB3[t] = bf16r(params[kOffB3 + t]);
    if (t == 0) {
        sB3[2] = params[kOffScale];
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + kTcOffTmem),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_smem_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kTcOffTmem);
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 TMEM lanes
    const float scale = sB3[2];
    const int total = kRows ? rows : P.Nc;
    const int tiles = (total + kTcRows - 1) / kTcRows;
    uint32_t phase = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int r = tile * kTcRows + t;
        const bool live = r < total;
        // 1. layer-1 operands of row t (operand column k: stencil point k / 3, channel k % 3)
        bool inside = true;  // the stencil stays inside the walls
        if (kRows) {
            auto operand = [&](int k) -> float {
                if (k >= kFeat) return k == kFeat ? 1.0f : 0.0f;
                if (!live) return 0.0f;
                const int pnt = k / 3, ch = k - 3 * pnt;
                return X[(size_t)r * kFeat + ch * 25 + pnt];
            };
#pragma unroll
            for (int j = 0; j < kTcK1 / 8; ++j) {
                uint32_t w[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) w[q] = pack_bf16(operand(8 * j + 2 * q), operand(8 * j + 2 * q + 1));
                *reinterpret_cast<uint4*>(sm + kTcOffA + kmajor_offset(t, 8 * j, kTcK1)) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        } else {
            uint32_t w[kTcK1 / 2];
            if (live) {
                stencil_operands<kTcK1>(P, feat, r, w);
                if (bulkOnly) {
                    const int ix = r / P.Ny, iy = r - ix * P.Ny;
                    inside = (P.perx || (ix >= 2 && ix < P.Nx - 2)) && (P.pery || (iy >= 2 && iy < P.Ny - 2));
                }
            } else {
#pragma unroll
                for (int j = 0; j < kTcK1 / 2; ++j)
                    w[j] = pack_bf16(2 * j == kFeat ? 1.0f : 0.0f, 2 * j + 1 == kFeat ? 1.0f : 0.0f);
            }
#pragma unroll
            for (int j = 0; j < kTcK1 / 8; ++j)
                *reinterpret_cast<uint4*>(sm + kTcOffA + kmajor_offset(t, 8 * j, kTcK1)) =
                    make_uint4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
        }
        tc_fence_smem_async();
        tc_fence_before();
        __syncthreads();
        // 2. layer 1 on the tensor cores
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int ks = 0; ks < kTcK1 / 16; ++ks)
                tc_mma(tmem, tc_desc(sbase + kTcOffA + ks * 256, 128, kTcK1 * 16),
                       tc_desc(sbase + kTcOffW1 + ks * 256, 128, kTcK1 * 16), ks > 0 ? 1u : 0u);
            tc_commit(bar);
        }
        ok = tc_wait(bar, phase);
        phase ^= 1;
        if (__syncthreads_and(ok) == 0) {
            if (t == 0) raise_error(st, kErrTensorWait, tile);
            ok = false;
            break;
        }
        tc_fence_after();
        // 3. a1 = gelu(z1) as BF16 operands of layer 2
#pragma unroll
        for (int h = 0; h < kHid / 16; ++h) {
            uint32_t z[16];
            tc_ld16(lane_base + 16 * h, z);
            tc_ld_wait16(z);
            uint32_t w[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                float g0, g1;
                f2_unpack(gelu2(f2_pack(__uint_as_float(z[2 * q]), __uint_as_float(z[2 * q + 1]))), g0, g1);
                w[q] = pack_bf16(g0, g1);
            }
            *reinterpret_cast<uint4*>(sm + kTcOffH + kmajor_offset(t, 16 * h, kHid)) = make_uint4(w[0], w[1], w[2], w[3]);
            *reinterpret_cast<uint4*>(sm + kTcOffH + kmajor_offset(t, 16 * h + 8, kHid)) = make_uint4(w[4], w[5], w[6], w[7]);
        }
        tc_fence_smem_async();
        tc_fence_before();
        __syncthreads();
        // 4. layer 2 on the tensor cores
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int ks = 0; ks < kHid / 16; ++ks)
                tc_mma(tmem + kHid, tc_desc(sbase + kTcOffH + ks * 256, 128, kHid * 16),
                       tc_desc(sbase + kTcOffW2 + ks * 256, 128, kHid * 16), ks > 0 ? 1u : 0u);
            tc_commit(bar);
        }
        ok = tc_wait(bar, phase);
        phase ^= 1;
        if (__syncthreads_and(ok) == 0) {
            if (t == 0) raise_error(st, kErrTensorWait, tile);
            ok = false;
            break;
        }
        tc_fence_after();
        // 5. output layer in FP32, over pairs of hidden units (even and odd partial sums)
        f32x2 p0 = f2_pack(0.0f, 0.0f), p1 = p0;
#pragma unroll
        for (int h = 0; h < kHid / 16; ++h) {
            uint32_t z[16];
            tc_ld16(lane_base + kHid + 16 * h, z);
            tc_ld_wait16(z);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int j = 16 * h + 2 * q;
                const f32x2 a = gelu2(f2_add(f2_pack(__uint_as_float(z[2 * q]), __uint_as_float(z[2 * q + 1])),
                                             *reinterpret_cast<const f32x2*>(sB2 + j)));
                p0 = f2_fma(a, *reinterpret_cast<const f32x2*>(sW3 + j), p0);
                p1 = f2_fma(a, *reinterpret_cast<const f32x2*>(sW3 + kHid + j), p1);
            }
        }
        float e0, e1, f0, f1;
        f2_unpack(p0, e0, e1);
        f2_unpack(p1, f0, f1);
        float o0 = sB3[0] + (e0 + e1), o1 = sB3[1] + (f0 + f1);
        tc_fence_before();  // the next tile's MMAs overwrite these columns after the barrier
        if (!kRows && bulkOnly) {  // no learned kick where the stencil crosses a wall
            // bulkOnly 2: a NaN marks the cell, whose kick the caller computes itself
            if (!inside) o0 = o1 = (bulkOnly == 2) ? __int_as_float(0x7fc00000) : 0.0f;
        }
        if (live) {
            if (kRows) {
                out[2 * (size_t)r] = o0 * scale;
                out[2 * (size_t)r + 1] = o1 * scale;
            } else {
                duX[r] = (double)(o0 * scale);
                duY[r] = (double)(o1 * scale);
            }
        }
        if (!kRows) {  // sum of N du over the cells, int64 at 2^-32 (exact and order-free), and
                       // the particles of the cells that take a learned kick
            long long qx = 0, qy = 0, qn = 0;
            if (live && !isnan(o0)) {
                // |N du| <= 2^8 per cell keeps the sum over up to 2^22 cells below 2^62 at 2^-32
                // (exact, no wrap); a larger kick is a diverged network: flagged, not summed
                const double nc = (double)__ldg(reinterpret_cast<const float*>(feat + r) + 3);
                const double px = nc * (double)(o0 * scale), py = nc * (double)(o1 * scale);
                if (fabs(px) <= 256.0 && fabs(py) <= 256.0) {
                    qx = __double2ll_rn(px * 0x1p32);
                    qy = __double2ll_rn(py * 0x1p32);
                    qn = (long long)nc;
                } else {
                    raise_error(st, kErrLearnedRange, r);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                qx += __shfl_xor_sync(0xffffffffu, qx, o);
                qy += __shfl_xor_sync(0xffffffffu, qy, o);
                qn += __shfl_xor_sync(0xffffffffu, qn, o);
            }
            if ((t & 31) == 0 && (qx != 0 || qy != 0 || qn != 0)) {
                atomicAdd(duSum, (unsigned long long)qx);
                atomicAdd(duSum + 1, (unsigned long long)qy);
                atomicAdd(duSum + 2, (unsigned long long)qn);
            }
        }
    }
    if (!ok) {  // an MMA did not complete in time: give it one more bounded wait before freeing TMEM
        tc_wait(bar, phase ^ 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols) : "memory");
    }
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

// ------------------------------------------------------------------ training on the tensor cores
// Forward and backward of 128-row tiles with tcgen05: one persistent CTA of 128 threads per SM,
// row t of a tile in thread t (TMEM lane t).
//   forward:  Z1 = X W1^T (b1 in operand column 75), a1 = bf16(gelu(Z1));
//             Z2 = A1 W2^T (b2 in operand column 64 of A1), a2 = gelu(Z2); out = W3 a2 + b3 (FP32)
//   backward: dout = 2 (out - y / scale) / (batch * 2); dW3, db3 in FP32 on the CUDA cores;
//             dz2 = bf16(dout W3 * gelu'(Z2)); dA1 = dz2 W2;  dz1 = bf16(dA1 * gelu'(Z1));
//             dW2^T += A1^T dz2 and dW1^T += X^T dz1, accumulated in TMEM over the CTA's tiles
//             (their rows 64 and 75, the constant columns, are db2 and db1)
// The transposed operands are written to shared memory beside the row-major ones, in the
// canonical no-swizzle K-major layout with K = 128 rows. Five MMAs (M = 128, N = 64) per tile.
// TMEM columns: Z1 [0, 64), Z2 [64, 128), dA1 [128, 192), dW2^T [192, 256), dW1^T [256, 320).
constexpr int kTgK1 = 80, kTgK2 = 80, kTgKR = 128;
constexpr uint32_t kTgOffX = 0;                                   // [128][80] bf16
constexpr uint32_t kTgOffXT = kTgOffX + 128 * kTgK1 * 2;          // [128][128] bf16 (rows: operand column)
constexpr uint32_t kTgOffA1 = kTgOffXT + 128 * kTgKR * 2;         // [128][80] bf16
constexpr uint32_t kTgOffA1T = kTgOffA1 + 128 * kTgK2 * 2;        // [128][128] bf16
constexpr uint32_t kTgOffD2 = kTgOffA1T + 128 * kTgKR * 2;        // [128][64] bf16
constexpr uint32_t kTgOffD2T = kTgOffD2 + 128 * kHid * 2;         // [64][128] bf16
constexpr uint32_t kTgOffD1T = kTgOffD2T + kHid * kTgKR * 2;      // [64][128] bf16
constexpr uint32_t kTgOffW1 = kTgOffD1T + kHid * kTgKR * 2;       // [64][80] bf16 (b1 in column 75)
constexpr uint32_t kTgOffW2 = kTgOffW1 + kHid * kTgK1 * 2;        // [64][80] bf16 (b2 in column 64)
constexpr uint32_t kTgOffW2T = kTgOffW2 + kHid * kTgK2 * 2;       // [64][64] bf16: W2^T
constexpr uint32_t kTgOffA2 = kTgOffW2T + kHid * kHid * 2;        // [128][64] f32
constexpr uint32_t kTgOffDO = kTgOffA2 + 128 * kHid * 4;          // [128][2] f32
constexpr uint32_t kTgOffW3 = kTgOffDO + 128 * kOut * 4;          // [2][64] f32, b3[2], pad
constexpr uint32_t kTgOffBar = kTgOffW3 + kOut * kHid * 4 + 16;   // mbarrier
constexpr uint32_t kTgOffTmem = kTgOffBar + 8;
constexpr uint32_t kTgSmem = kTgOffTmem + 8;
constexpr uint32_t kTgTmemCols = 512;
static_assert(kTgSmem <= 227 * 1024, "training tile exceeds shared memory");
static_assert(2 * (kTgSmem + 1024) > 228 * 1024, "one training CTA per SM (its TMEM takes all 512 columns)");
constexpr uint32_t kTgIdesc = kTcIdesc;  // D F32, A and B BF16 K-major, N = 64, M = 128

// the MMA of a K-major A [128 x K] and B [64 x K] at shared addresses a, b into TMEM column d
__device__ __forceinline__ void tg_mma(uint32_t d, uint32_t a, uint32_t b, int K, bool accumulate) {
    for (int ks = 0; ks < K / 16; ++ks)
        tc_mma(d, tc_desc(a + ks * 256, 128, K * 16), tc_desc(b + ks * 256, 128, K * 16),
               (accumulate || ks > 0) ? 1u : 0u);
}

__device__ __forceinline__ void tg_put(unsigned char* sm, uint32_t off, int r, int k, int K, float v) {
    *reinterpret_cast<__nv_bfloat16*>(sm + off + kmajor_offset(r, k, K)) = __float2bfloat16_rn(v);
}

__global__ void __launch_bounds__(128, 1)
    k_mlp_grad_tc(const float* __restrict__ X, const float* __restrict__ Y, const int* __restrict__ idx, int rows,
                  int batch, float yinv, const float* __restrict__ params, float* __restrict__ grad,
                  float* __restrict__ loss, DevStatus* st) {
    extern __shared__ __align__(128) unsigned char sm[];
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const uint32_t bar = sbase + kTgOffBar;
    float* sA2 = reinterpret_cast<float*>(sm + kTgOffA2);
    float* sDO = reinterpret_cast<float*>(sm + kTgOffDO);
    float* sW3 = reinterpret_cast<float*>(sm + kTgOffW3);
    // weights (W1 in the point-major operand order of the features), zero padding of the
    // transposed operands' unused rows
    for (int i = t; i < kHid * kTgK1; i += 128) {
        const int n = i / kTgK1, k = i - n * kTgK1;
        const int pk = (k % 3) * 25 + k / 3;
        const float w = k < kFeat ? params[kOffW1 + n * kFeat + pk] : (k == kFeat ? params[kOffB1 + n] : 0.0f);
        tg_put(sm, kTgOffW1, n, k, kTgK1, w);
    }
    for (int i = t; i < kHid * kTgK2; i += 128) {
        const int n = i / kTgK2, k = i - n * kTgK2;
        const float w = k < kHid ? params[kOffW2 + n * kHid + k] : (k == kHid ? params[kOffB2 + n] : 0.0f);
        tg_put(sm, kTgOffW2, n, k, kTgK2, w);
    }
    for (int i = t; i < kHid * kHid; i += 128) {
        const int n = i / kHid, k = i - n * kHid;  // W2^T[n][k] = W2[k][n]
        tg_put(sm, kTgOffW2T, n, k, kHid, params[kOffW2 + k * kHid + n]);
    }
    for (int i = t; i < kOut * kHid; i += 128) sW3[i] = bf16r(params[kOffW3 + i]);
    if (t < kOut) sW3[kOut * kHid + t] = bf16r(params[kOffB3 + t]);
    for (int i = t; i < 128 * kTgKR; i += 128) {
        const int r = i / kTgKR, k = i - r * kTgKR;
        if (r >= kTgK1 - 4) tg_put(sm, kTgOffXT, r, k, kTgKR, 0.0f);   // operand columns 76..127
        if (r > kHid) tg_put(sm, kTgOffA1T, r, k, kTgKR, 0.0f);       // columns 65..127
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + kTgOffTmem),
                     "r"(kTgTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_smem_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kTgOffTmem);
    const uint32_t lb = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 TMEM lanes
    const float b3a = sW3[kOut * kHid], b3b = sW3[kOut * kHid + 1];
    const float dscale = 2.0f / (float)(batch * kOut);
    const int tiles = (rows + 127) / 128;
    uint32_t phase = 0;
    bool ok = true, first = true;
    float accW3 = 0.0f, accB3 = 0.0f, lossAcc = 0.0f;
    auto sync_mma = [&](auto issue) {  // shared stores visible, one thread issues, all wait
        tc_fence_smem_async();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
            issue();
            tc_commit(bar);
        }
        ok = tc_wait(bar, phase);
        phase ^= 1;
        if (__syncthreads_and(ok) == 0) {
            if (t == 0) raise_error(st, kErrTensorWait, blockIdx.x);
            ok = false;
        }
        tc_fence_after();
        return ok;
    };
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int r = tile * 128 + t;
        const bool live = r < rows;
        const int src = live ? idx[r] : 0;
        // 1. the row's operands, row-major and transposed (point-major feature order)
        float y0 = 0.0f, y1 = 0.0f;
        if (live) {
            y0 = Y[(size_t)src * kOut] * yinv;
            y1 = Y[(size_t)src * kOut + 1] * yinv;
        }
        for (int k = 0; k < kTgK1; ++k) {
            float v = 0.0f;
            if (k < kFeat) v = live ? X[(size_t)src * kFeat + (k % 3) * 25 + k / 3] : 0.0f;
            else if (k == kFeat) v = 1.0f;
            tg_put(sm, kTgOffX, t, k, kTgK1, v);
            if (k <= kFeat) tg_put(sm, kTgOffXT, k, t, kTgKR, v);
        }
        // 2. Z1 = X W1^T
        if (!sync_mma([&] { tg_mma(tmem, sbase + kTgOffX, sbase + kTgOffW1, kTgK1, false); })) break;
        // 3. a1 = bf16(gelu(Z1)), row-major (column 64: the constant of b2) and transposed
#pragma unroll
        for (int h = 0; h < kHid / 16; ++h) {
            uint32_t z[16];
            tc_ld16(lb + 16 * h, z);
            tc_ld_wait16(z);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const float a = gelu(__uint_as_float(z[q]));
                tg_put(sm, kTgOffA1, t, 16 * h + q, kTgK2, a);
                tg_put(sm, kTgOffA1T, 16 * h + q, t, kTgKR, a);
            }
        }
        for (int k = kHid; k < kTgK2; ++k) tg_put(sm, kTgOffA1, t, k, kTgK2, k == kHid ? 1.0f : 0.0f);
        tg_put(sm, kTgOffA1T, kHid, t, kTgKR, 1.0f);
        // 4. Z2 = A1 W2^T
        if (!sync_mma([&] { tg_mma(tmem + kHid, sbase + kTgOffA1, sbase + kTgOffW2, kTgK2, false); })) break;
        // 5. a2, the output layer, dout; dz2 = bf16(dout W3 * gelu'(Z2)), row-major and transposed
        float o0 = b3a, o1 = b3b;
#pragma unroll
        for (int h = 0; h < kHid / 16; ++h) {
            uint32_t z[16];
            tc_ld16(lb + kHid + 16 * h, z);
            tc_ld_wait16(z);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int j = 16 * h + q;
                const float a = gelu(__uint_as_float(z[q]));
                sA2[t * kHid + j] = a;
                o0 = fmaf(sW3[j], a, o0);
                o1 = fmaf(sW3[kHid + j], a, o1);
            }
        }
        const float e0 = o0 - y0, e1 = o1 - y1;
        const float d0 = live ? dscale * e0 : 0.0f, d1 = live ? dscale * e1 : 0.0f;
        if (live) lossAcc += (e0 * e0 + e1 * e1) / (float)(batch * kOut);
        sDO[2 * t] = d0;
        sDO[2 * t + 1] = d1;
#pragma unroll
        for (int h = 0; h < kHid / 16; ++h) {
            uint32_t z[16];
            tc_ld16(lb + kHid + 16 * h, z);
            tc_ld_wait16(z);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int j = 16 * h + q;
                const float dz = (d0 * sW3[j] + d1 * sW3[kHid + j]) * gelu_d(__uint_as_float(z[q]));
                tg_put(sm, kTgOffD2, t, j, kHid, dz);
                tg_put(sm, kTgOffD2T, j, t, kTgKR, dz);
            }
        }
        // 6. dA1 = dz2 W2; dW2^T += A1^T dz2
        if (!sync_mma([&] {
                tg_mma(tmem + 2 * kHid, sbase + kTgOffD2, sbase + kTgOffW2T, kHid, false);
                tg_mma(tmem + 3 * kHid, sbase + kTgOffA1T, sbase + kTgOffD2T, kTgKR, !first);
            }))
            break;
        // dW3, db3 over the tile's rows (thread i: entry i of W3)
        {
            const int o = t / kHid, k = t - o * kHid;
            float g = 0.0f, gb = 0.0f;
            for (int rr = 0; rr < 128; ++rr) {
                const float d = sDO[2 * rr + o];
                g = fmaf(d, sA2[rr * kHid + k], g);
                gb += d;
            }
            accW3 += g;
            if (k == 0) accB3 += gb;
        }
        // 7. dz1 = bf16(dA1 * gelu'(Z1)), transposed
#pragma unroll
        for (int h = 0; h < kHid / 16; ++h) {
            uint32_t z[16], d[16];
            tc_ld16(lb + 16 * h, z);
            tc_ld16(lb + 2 * kHid + 16 * h, d);
            tc_ld_wait16(z);
            tc_ld_wait16(d);
#pragma unroll
            for (int q = 0; q < 16; ++q)
                tg_put(sm, kTgOffD1T, 16 * h + q, t, kTgKR, __uint_as_float(d[q]) * gelu_d(__uint_as_float(z[q])));
        }
        // 8. dW1^T += X^T dz1 (the wait also frees the operands for the next tile)
        if (!sync_mma([&] { tg_mma(tmem + 4 * kHid, sbase + kTgOffXT, sbase + kTgOffD1T, kTgKR, !first); })) break;
        first = false;
    }
    // the accumulated gradients: lane t of dW1^T is operand column t (feature, or b1 at 75),
    // lane t of dW2^T is A1 column t (or b2 at 64)
    if (ok && !first) {
        const int pk = t < kFeat ? (t % 3) * 25 + t / 3 : -1;
#pragma unroll
        for (int h = 0; h < kHid / 16; ++h) {
            uint32_t a[16], b[16];
            tc_ld16(lb + 4 * kHid + 16 * h, a);
            tc_ld16(lb + 3 * kHid + 16 * h, b);
            tc_ld_wait16(a);
            tc_ld_wait16(b);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int j = 16 * h + q;
                if (t < kFeat) atomicAdd(grad + kOffW1 + j * kFeat + pk, __uint_as_float(a[q]));
                else if (t == kFeat) atomicAdd(grad + kOffB1 + j, __uint_as_float(a[q]));
                if (t < kHid) atomicAdd(grad + kOffW2 + j * kHid + t, __uint_as_float(b[q]));
                else if (t == kHid) atomicAdd(grad + kOffB2 + j, __uint_as_float(b[q]));
            }
        }
        atomicAdd(grad + kOffW3 + t, accW3);
        if (t % kHid == 0) atomicAdd(grad + kOffB3 + t / kHid, accB3);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lossAcc += __shfl_xor_sync(0xffffffffu, lossAcc, o);
    if (lane == 0 && lossAcc != 0.0f) atomicAdd(loss, lossAcc);
    if (!ok) tc_wait(bar, phase ^ 1);  // an MMA did not complete in time: one more bounded wait
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTgTmemCols) : "memory");
    }
}

}  // namespace mpcd_dev
