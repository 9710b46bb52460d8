// Liquid closure (reference src/liquid_closure.cpp:329-444).
//
//   ref fields  : cell fields of the post-collision state (computed before the zone passes)
//   k_pdrive    : pdriveRaw = Pkin + Pvir of ref, blended with the 5-point cross smoothing on
//                 the static interzone mask (:401-419, local_cross_smooth :215-241)
//   k_eos       : boundary-aware central gradient and the EOS kick (:243-295, :424-430)
//   k_closure_cells : red-state momenta per cell, duRepair and the beta_opt terms (:343-360)
//   k_reduce_*  : fixed-order reductions (num, den and diagnostics)
//   k_kick      : v <- (v + beta*duRepair[c]) + duEOS[c] per particle (:380-389, :432-436),
//                 writing particles in (cell, particle id) order into the next buffer
#pragma once

#include "common.cuh"

namespace mpcd_dev {

// local_cross_smooth at one cell (acc = centre, then left, right, down, up)
__device__ __forceinline__ double cross_smooth(const double* raw, int ix, int iy, const DevParams& P) {
    double acc = raw[iy + P.Ny * ix];
    int cnt = 1;
    const int jj[4][2] = {{iy, ix - 1}, {iy, ix + 1}, {iy - 1, ix}, {iy + 1, ix}};
    for (int q = 0; q < 4; ++q) {
        int jy = jj[q][0], jx = jj[q][1];
        if (P.perx) jx = wrap_index(jx, P.Nx);
        else if (jx < 0 || jx >= P.Nx) continue;
        if (P.pery) jy = wrap_index(jy, P.Ny);
        else if (jy < 0 || jy >= P.Ny) continue;
        acc = __dadd_rn(acc, raw[jy + P.Ny * jx]);
        ++cnt;
    }
    return __ddiv_rn(acc, (double)cnt);
}

// skip (nullable): a device flag; when set, the step runs the learned closure and these
// kernels of the plain one do nothing
__global__ void k_pdrive(DevParams P, const double* __restrict__ pkin, const double* __restrict__ pvir, double* __restrict__ raw,
                         const int* skip) {
    if (skip && *skip) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.Nc) return;
    raw[c] = __dadd_rn(pkin[c], pvir[c]);
}

__device__ __forceinline__ void pdrive_blend_block(int bx, const DevParams& P, const double* __restrict__ raw,
                                                   const int* __restrict__ mask, int anyMask, double* __restrict__ pdrive,
                                                   const int* skip) {
    if (skip && *skip) return;
    const int c = bx * blockDim.x + threadIdx.x;
    if (c >= P.Nc) return;
    double v = raw[c];
    if (anyMask && mask[c] != 0) {
        const int ix = c / P.Ny, iy = c - ix * P.Ny;
        const double ps = cross_smooth(raw, ix, iy, P);
        v = __dadd_rn(__dmul_rn(__dsub_rn(1.0, P.smoothBlend), raw[c]), __dmul_rn(P.smoothBlend, ps));
    }
    pdrive[c] = v;
}

__global__ void k_pdrive_blend(DevParams P, const double* __restrict__ raw, const int* __restrict__ mask, int anyMask,
                               double* __restrict__ pdrive, const int* skip) {
    pdrive_blend_block((int)blockIdx.x, P, raw, mask, anyMask, pdrive, skip);
}

__global__ void k_eos(DevParams P, const double* __restrict__ pd, double* __restrict__ eosX, double* __restrict__ eosY,
                      const int* skip) {
    if (skip && *skip) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.Nc) return;
    const int ix = c / P.Ny, iy = c - ix * P.Ny;
    double gx, gy;
    if (P.perx) gx = __ddiv_rn(__dsub_rn(pd[iy + P.Ny * wrap_index(ix + 1, P.Nx)], pd[iy + P.Ny * wrap_index(ix - 1, P.Nx)]), __dmul_rn(2.0, P.dx));
    else if (ix == 0) gx = __ddiv_rn(__dsub_rn(pd[iy + P.Ny * (ix + 1)], pd[c]), P.dx);
    else if (ix == P.Nx - 1) gx = __ddiv_rn(__dsub_rn(pd[c], pd[iy + P.Ny * (ix - 1)]), P.dx);
    else gx = __ddiv_rn(__dsub_rn(pd[iy + P.Ny * (ix + 1)], pd[iy + P.Ny * (ix - 1)]), __dmul_rn(2.0, P.dx));
    if (P.pery) gy = __ddiv_rn(__dsub_rn(pd[wrap_index(iy + 1, P.Ny) + P.Ny * ix], pd[wrap_index(iy - 1, P.Ny) + P.Ny * ix]), __dmul_rn(2.0, P.dy));
    else if (iy == 0) gy = __ddiv_rn(__dsub_rn(pd[(iy + 1) + P.Ny * ix], pd[c]), P.dy);
    else if (iy == P.Ny - 1) gy = __ddiv_rn(__dsub_rn(pd[c], pd[(iy - 1) + P.Ny * ix]), P.dy);
    else gy = __ddiv_rn(__dsub_rn(pd[(iy + 1) + P.Ny * ix], pd[(iy - 1) + P.Ny * ix]), __dmul_rn(2.0, P.dy));
    const double k = -__ddiv_rn(P.dt, P.rhoTarget);
    eosX[c] = __dmul_rn(__dmul_rn(k, gx), P.betaEOS);
    eosY[c] = __dmul_rn(__dmul_rn(k, gy), P.betaEOS);
}

// Per cell of the red (post-redistribution) state: momenta in particle-id order, velocity,
// duRepair = (P_ref - P_red) / gamma and the beta_opt terms. cols: 2 doubles per cell
// (num term, den term) for the fixed-order reduction.
struct RedFields {
    int* N;
    double *Px, *Py, *Ux, *Uy;
    float4* feat;  // (N/gamma - 1, Ux, Uy, N) as FP32: the learned closure's stencil input
};
template <class V>
__global__ void k_closure_cells(DevParams P, const uint64_t* __restrict__ start, const int* __restrict__ slots, V S,
                                const double* __restrict__ refPx,
                                const double* __restrict__ refPy, const double* __restrict__ refUx,
                                const double* __restrict__ refUy, RedFields red, double* __restrict__ duRX,
                                double* __restrict__ duRY, double* __restrict__ cols, int* __restrict__ cellOf) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.Nc) return;
    const int a = (int)(uint32_t)start[c], b = (int)(uint32_t)start[c + 1];
    const int m = b - a;
    double px = 0.0, py = 0.0;
    for (int j = a; j < b; ++j) {
        const double2 w = S.vel(slots[j]);
        px = __dadd_rn(px, w.x);
        py = __dadd_rn(py, w.y);
        if (cellOf) cellOf[j] = c;
    }
    double ux = 0.0, uy = 0.0;
    if (m > 0) {
        ux = __ddiv_rn(px, (double)m);
        uy = __ddiv_rn(py, (double)m);
    }
    const double ax = __ddiv_rn(__dsub_rn(refPx[c], px), P.gamma);
    const double ay = __ddiv_rn(__dsub_rn(refPy[c], py), P.gamma);
    const double ex = __dsub_rn(ux, refUx[c]), ey = __dsub_rn(uy, refUy[c]);
    duRX[c] = ax;
    duRY[c] = ay;
    cols[2 * (size_t)c] = -__dadd_rn(__dmul_rn(ex, ax), __dmul_rn(ey, ay));
    cols[2 * (size_t)c + 1] = __dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay));
    if (red.N) red.N[c] = m;
    if (red.Px) red.Px[c] = px;
    if (red.Py) red.Py[c] = py;
    if (red.Ux) red.Ux[c] = ux;
    if (red.Uy) red.Uy[c] = uy;
    if (red.feat) red.feat[c] = make_float4((float)__dsub_rn(__ddiv_rn((double)m, P.gamma), 1.0), (float)ux, (float)uy, (float)m);
}

// ---------------------------------------------------------------- fixed-order reductions
// K interleaved columns over n rows; kind bit k set -> max instead of sum for column k.
constexpr int kRedThreads = 256;
constexpr int kRedMaxCols = 16;
__device__ __forceinline__ void reduce_partial_block(int bx, const double* __restrict__ in, int64_t n, int K,
                                                     unsigned maxMask, int rowsPerBlock, double* __restrict__ partial) {
    __shared__ double sh[kRedMaxCols][kRedThreads];
    const int t = threadIdx.x;
    const int64_t r0 = (int64_t)bx * rowsPerBlock;
    const int64_t r1 = min((int64_t)n, r0 + rowsPerBlock);
    for (int k = 0; k < K; ++k) {
        double a = 0.0;
        for (int64_t r = r0 + t; r < r1; r += kRedThreads) {
            const double x = in[r * K + k];
            a = ((maxMask >> k) & 1u) ? smax(a, x) : __dadd_rn(a, x);
        }
        sh[k][t] = a;
    }
    __syncthreads();
    for (int o = kRedThreads / 2; o > 0; o >>= 1) {
        if (t < o)
            for (int k = 0; k < K; ++k)
                sh[k][t] = ((maxMask >> k) & 1u) ? smax(sh[k][t], sh[k][t + o]) : __dadd_rn(sh[k][t], sh[k][t + o]);
        __syncthreads();
    }
    if (t < K) partial[(size_t)bx * K + t] = sh[t][0];
}

__global__ void __launch_bounds__(kRedThreads) k_reduce_partial(const double* __restrict__ in, int64_t n, int K,
                                                                unsigned maxMask, int rowsPerBlock,
                                                                double* __restrict__ partial) {
    reduce_partial_block((int)blockIdx.x, in, n, K, maxMask, rowsPerBlock, partial);
}

__device__ __forceinline__ void reduce_final_block(const double* __restrict__ partial, int nb, int K, unsigned maxMask,
                                                   double* __restrict__ out) {
    __shared__ double sh[kRedMaxCols][kRedThreads];
    const int t = threadIdx.x;
    for (int k = 0; k < K; ++k) {
        double a = 0.0;
        for (int b = t; b < nb; b += kRedThreads) {
            const double x = partial[(size_t)b * K + k];
            a = ((maxMask >> k) & 1u) ? smax(a, x) : __dadd_rn(a, x);
        }
        sh[k][t] = a;
    }
    __syncthreads();
    for (int o = kRedThreads / 2; o > 0; o >>= 1) {
        if (t < o)
            for (int k = 0; k < K; ++k)
                sh[k][t] = ((maxMask >> k) & 1u) ? smax(sh[k][t], sh[k][t + o]) : __dadd_rn(sh[k][t], sh[k][t + o]);
        __syncthreads();
    }
    if (t < K) out[t] = sh[t][0];
}

__global__ void __launch_bounds__(kRedThreads) k_reduce_final(const double* __restrict__ partial, int nb, int K,
                                                              unsigned maxMask, double* __restrict__ out) {
    reduce_final_block(partial, nb, K, maxMask, out);
}

// beta_applied from num/den (src/liquid_closure.cpp:364-377)
__device__ __forceinline__ double beta_applied(const DevParams& P, double num, double den) {
    double opt = 0.0;
    if (isfinite(num) && isfinite(den) && den > 0.0) opt = smax(__ddiv_rn(num, den), 0.0);
    if (!P.useOptimalBetaRepair) return P.betaRepair;
    if (!isfinite(opt) || !isfinite(den) || den < 1e-20) return P.betaRepair;
    return (opt < 0.0) ? 0.0 : ((2.0 < opt) ? 2.0 : opt);
}

// The two kicks, one cell per thread in particle-id order. If xo/vo/pido are given the
// particles are written in (cell, id) order starting at the cell's segment (the next
// step's layout); otherwise v is updated in place. vrep (optional, slot order) receives the
// repaired velocities. stats: 8 columns per cell for the diagnostics reduction:
// sum kn_rep^2, max kn_rep, hypot(beta*duR), sum kn_eos^2, max kn_eos, sum vin.x, sum vin.y,
// sum vout.x - not used (momentum delta from vout sums) -> see column list in k_kick.
constexpr int kKickCols = 9;
// S: the red state (kicked in place unless permute); T: the next step's layout (permute)
template <class V>
__global__ void k_kick(DevParams P, const uint64_t* __restrict__ start, const int* __restrict__ slots,
                       const double* __restrict__ numden, const double* __restrict__ duRX,
                       const double* __restrict__ duRY, const double* __restrict__ eosX,
                       const double* __restrict__ eosY, V S, const int* __restrict__ pid, int permute, V T,
                       int* __restrict__ pido, double2* __restrict__ vrep, double* __restrict__ stats) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.Nc) return;
    const double beta = beta_applied(P, numden[0], numden[1]);
    const double kx = __dmul_rn(beta, duRX[c]), ky = __dmul_rn(beta, duRY[c]);
    const double ex = eosX[c], ey = eosY[c];
    const int a = (int)(uint32_t)start[c], b = (int)(uint32_t)start[c + 1];
    double sinx = 0.0, siny = 0.0, soutx = 0.0, souty = 0.0;
    for (int j = a; j < b; ++j) {
        const int s = slots[j];
        const double2 w = S.vel(s);
        const double2 r = make_double2(__dadd_rn(w.x, kx), __dadd_rn(w.y, ky));
        const double2 o = make_double2(__dadd_rn(r.x, ex), __dadd_rn(r.y, ey));
        if (vrep) vrep[s] = r;
        if (permute) {
            T.copy_pos(j, S, s);
            T.set_vel(j, o);
            pido[j] = pid[s];
        } else {
            S.set_vel(s, o);
        }
        sinx = __dadd_rn(sinx, w.x);
        siny = __dadd_rn(siny, w.y);
        soutx = __dadd_rn(soutx, o.x);
        souty = __dadd_rn(souty, o.y);
    }
    if (stats) {
        const int m = b - a;
        const double knr = sqrt(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)));
        const double kne = sqrt(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)));
        double* s = stats + (size_t)c * kKickCols;
        s[0] = __dmul_rn((double)m, __dmul_rn(knr, knr));
        s[1] = (m > 0) ? knr : 0.0;
        s[2] = mpcd_dd::hypot_cr(kx, ky);
        s[3] = __dmul_rn((double)m, __dmul_rn(kne, kne));
        s[4] = (m > 0) ? kne : 0.0;
        s[5] = sinx;
        s[6] = siny;
        s[7] = soutx;
        s[8] = souty;
    }
}

// The two kicks for index positions j (flat, coalesced), writing the particle at position j
// of the next step's layout: (cell, particle id) order. Each thread takes kKickItems positions
// (independent gathers in flight); the launch-wide factors (beta, or the learned kick's
// particle mean) are computed once per block.
constexpr int kKickItems = 2;
template <class V>
__global__ void k_kick_flat(DevParams P, int n, const int* __restrict__ cellOf, const int* __restrict__ slots,
                            const double* __restrict__ numden, const double* __restrict__ duRX,
                            const double* __restrict__ duRY, const double* __restrict__ eosX,
                            const double* __restrict__ eosY, V S, const int* __restrict__ pid, V T,
                            int* __restrict__ pido, const int* learned,
                            const double* __restrict__ duLX, const double* __restrict__ duLY,
                            const long long* __restrict__ duLSum) {
    __shared__ double fac[2];  // beta, or the learned kick's particle mean (x, y)
    __shared__ int lrn;
    if (threadIdx.x == 0) {
        lrn = learned ? *learned : 0;
        if (lrn) {
            // the learned closure's kick less its particle mean (sum over cells of N du, int64
            // at 2^-32), so that it leaves the total momentum unchanged
            fac[0] = __ddiv_rn((double)duLSum[0] * 0x1p-32, (double)P.n);
            fac[1] = __ddiv_rn((double)duLSum[1] * 0x1p-32, (double)P.n);
        } else {
            fac[0] = beta_applied(P, numden[0], numden[1]);
        }
    }
    __syncthreads();
    const int j0 = blockIdx.x * (blockDim.x * kKickItems) + threadIdx.x;
    int c[kKickItems], s[kKickItems];
#pragma unroll
    for (int k = 0; k < kKickItems; ++k) {
        const int j = j0 + k * (int)blockDim.x;
        c[k] = j < n ? cellOf[j] : 0;
        s[k] = j < n ? slots[j] : 0;
    }
    double2 w[kKickItems];
    int q[kKickItems];
#pragma unroll
    for (int k = 0; k < kKickItems; ++k) {
        const bool in = j0 + k * (int)blockDim.x < n;
        w[k] = in ? S.vel(s[k]) : make_double2(0.0, 0.0);
        q[k] = in ? pid[s[k]] : 0;
    }
#pragma unroll
    for (int k = 0; k < kKickItems; ++k) {
        const int j = j0 + k * (int)blockDim.x;
        if (j >= n) continue;
        if (lrn) {
            T.set_vel(j, make_double2(__dadd_rn(w[k].x, __dsub_rn(duLX[c[k]], fac[0])),
                                      __dadd_rn(w[k].y, __dsub_rn(duLY[c[k]], fac[1]))));
        } else {
            const double kx = __dmul_rn(fac[0], duRX[c[k]]), ky = __dmul_rn(fac[0], duRY[c[k]]);
            const double2 r = make_double2(__dadd_rn(w[k].x, kx), __dadd_rn(w[k].y, ky));
            T.set_vel(j, make_double2(__dadd_rn(r.x, eosX[c[k]]), __dadd_rn(r.y, eosY[c[k]])));
        }
        T.copy_pos(j, S, s[k]);
        pido[j] = q[k];
    }
}

// identity cell index after a permuting kick: slots[j] = j
__global__ void k_iota(int* __restrict__ a, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// per-particle sums for the step metrics: 0.5|v|^2, vx, vy (slot order; fixed reduction)
template <class V>
__global__ void k_particle_cols(V S, int n, double* __restrict__ cols) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 w = S.vel(i);
    cols[3 * (size_t)i] = __dmul_rn(0.5, __dadd_rn(__dmul_rn(w.x, w.x), __dmul_rn(w.y, w.y)));
    cols[3 * (size_t)i + 1] = w.x;
    cols[3 * (size_t)i + 2] = w.y;
}

// Poiseuille profile of the slot state: per row iy, the momentum along x (int64 at 2^-32,
// each particle rounded once, so the sums are exact and independent of order) and the count,
// added over the steps. Lanes of one row are summed in the warp before the atomics.
template <class V>
__global__ void k_profile_slots(DevParams P, V S, int n, unsigned long long* __restrict__ rowP,
                                unsigned long long* __restrict__ rowN) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const unsigned act = __ballot_sync(0xffffffffu, live);
    if (!live) return;
    const int row = S.std_cell(i, P) % P.Ny;
    const long long q = llrint(S.vel(i).x * 0x1p32);
    const unsigned grp = __match_any_sync(act, row);
    const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    long long sum = 0;
    for (unsigned m = grp; m; m &= m - 1) {
        const long long t = __shfl_sync(grp, q, __ffs(m) - 1);
        sum += t;
    }
    if (lane == leader) {
        atomicAdd(rowP + row, (unsigned long long)sum);
        atomicAdd(rowN + row, (unsigned long long)__popc(grp));
    }
}

// per-cell columns for occStd / outBand from a cell index (counts), and mean Ux / Uy
__global__ void k_count_cols(const uint64_t* __restrict__ start, int Nc, double highThr, double lowThr,
                             double* __restrict__ cols) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Nc) return;
    const double n = (double)((uint32_t)start[c + 1] - (uint32_t)start[c]);
    cols[3 * (size_t)c] = n;
    cols[3 * (size_t)c + 1] = __dmul_rn(n, n);
    cols[3 * (size_t)c + 2] = ((n > highThr) || (n > 0.0 && n < lowThr)) ? 1.0 : 0.0;
}

}  // namespace mpcd_dev
