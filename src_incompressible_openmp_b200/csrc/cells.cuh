// Per-cell kernels over a cell index (slots of each cell in ascending particle id):
// the SRD rotation collision and compute_cell_fields.
#pragma once

#include "common.cuh"

namespace mpcd_dev {

// The collision's rotation-sign stream: draw r of mt19937_64(seed) belongs to the r-th cell
// (in cell order) holding >= 2 particles (src/srd_collision.cpp:77-83); sign[r] = 1 when
// U(0,1) < 0.5 (theta = -alpha). One block generates `count` draws, one twist at a time.
constexpr int kSignThreads = 320;
// seedDev (graph replay): the next step's seed and output buffer (sign, sign1 by its parity)
__global__ void __launch_bounds__(kSignThreads) k_srd_signs(uint64_t seed, int count, uint8_t* __restrict__ sign,
                                                           const uint64_t* seedDev, uint8_t* sign1) {
    if (seedDev) {
        seed = seedDev[kSeedSignsNext];
        if (seedDev[kSeedNextParity]) sign = sign1;
    }
    __shared__ uint64_t mt[kMtN];
    const int t = threadIdx.x;
    if (t == 0) {
        uint64_t w = seed;
        mt[0] = w;
        for (int i = 1; i < kMtN; ++i) {
            w = mt_seed_next(w, i);
            mt[i] = w;
        }
    }
    __syncthreads();
    for (int base = 0; base < count; base += kMtN) {
        uint64_t nv = 0;
        if (t < kMtN - kMtM) nv = mt[t + kMtM] ^ mt_mix(mt[t], mt[t + 1]);
        __syncthreads();
        if (t < kMtN - kMtM) mt[t] = nv;
        __syncthreads();
        if (t >= kMtN - kMtM && t < kMtN) {
            const uint64_t nxt = (t + 1 < kMtN) ? mt[t + 1] : mt[0];
            nv = mt[t - (kMtN - kMtM)] ^ mt_mix(mt[t], nxt);
        }
        __syncthreads();
        if (t >= kMtN - kMtM && t < kMtN) mt[t] = nv;
        __syncthreads();
        if (t < kMtN && base + t < count) sign[base + t] = (canon(mt_temper(mt[t])) < 0.5) ? 1 : 0;
        __syncthreads();
    }
}

// srd_collision_step (src/srd_collision.cpp:47-124) on one SRD cell whose m velocities are
// read by ld(j) and written by st(j, w), j in particle-id order: mean, a +-alpha rotation of
// the relative velocities (sign from the cell's rank among cells with >= 2 particles) and the
// thermostat rescaling. start0: packed (segment start | rank << 32). Returns false on error.
template <typename Ld, typename St>
__device__ __forceinline__ bool collide_cell(const DevParams& P, uint64_t start0, int m, const uint8_t* sign,
                                             int signCount, DevStatus* st, Ld ld, St stv) {
    double sx = 0.0, sy = 0.0;
    for (int j = 0; j < m; ++j) {
        const double2 w = ld(j);
        sx = __dadd_rn(sx, w.x);
        sy = __dadd_rn(sy, w.y);
    }
    const double ux = __ddiv_rn(sx, (double)m), uy = __ddiv_rn(sy, (double)m);
    int rot = 0;
    if (m >= 2) {
        const int r = (int)(start0 >> 32);
        if (r >= signCount) {
            raise_error(st, kErrRngCapacity, r);
            return false;
        }
        rot = sign[r] ? 2 : 1;
    }
    const double ct = P.rotCos[rot], sn = P.rotSin[rot];
    double lam = 1.0;
    if (P.useThermostat) {
        double sr = 0.0;
        for (int j = 0; j < m; ++j) {
            const double2 w = ld(j);
            const double xr = __dsub_rn(w.x, ux), yr = __dsub_rn(w.y, uy);
            const double x2 = __dsub_rn(__dmul_rn(ct, xr), __dmul_rn(sn, yr));
            const double y2 = __dadd_rn(__dmul_rn(sn, xr), __dmul_rn(ct, yr));
            sr = __dadd_rn(sr, __dadd_rn(__dmul_rn(x2, x2), __dmul_rn(y2, y2)));
        }
        if (m > 1 && sr > 0.0) lam = sqrt(__ddiv_rn(__dmul_rn((double)(2 * (m - 1)), P.kBT), sr));
    }
    for (int j = 0; j < m; ++j) {
        const double2 w = ld(j);
        const double xr = __dsub_rn(w.x, ux), yr = __dsub_rn(w.y, uy);
        double x2 = __dsub_rn(__dmul_rn(ct, xr), __dmul_rn(sn, yr));
        double y2 = __dadd_rn(__dmul_rn(sn, xr), __dmul_rn(ct, yr));
        if (P.useThermostat) {
            x2 = __dmul_rn(x2, lam);
            y2 = __dmul_rn(y2, lam);
        }
        stv(j, make_double2(__dadd_rn(ux, x2), __dadd_rn(uy, y2)));
    }
    return true;
}

// The collision over kCollideCells consecutive SRD cells per block. Their segments are
// contiguous in slots[]: the velocities are gathered once into shared memory by the whole
// block, each thread runs its cell there, and the block scatters them back. A block whose
// segments exceed the tile works on global memory instead. The tile shape (cells and threads
// per block) is a template argument; the context's autotuner picks one of kCollideShapes by
// timing them on its own state. Every shape gives the same result: a cell's collision does
// not depend on the tiling.
struct CollideShape {
    int cells, threads;
};
constexpr int kCollideShapes = 7;
constexpr CollideShape kCollideShape[kCollideShapes] = {{32, 128}, {64, 256}, {128, 256}, {256, 512},
                                                        {16, 128}, {32, 256},  {16, 64}};

template <class V, int kCollideCells, int kCollideThreads>
__global__ void __launch_bounds__(kCollideThreads) k_srd_collide(DevParams P, const uint64_t* __restrict__ start,
                                                                 const int* __restrict__ slots,
                                                                 const uint8_t* __restrict__ sign, int signCount,
                                                                 V S, DevStatus* st,
                                                                 const uint64_t* seedDev,
                                                                 const uint8_t* __restrict__ sign1, int tileCap) {
    extern __shared__ __align__(16) double2 tv[];
    int* ts = reinterpret_cast<int*>(tv + tileCap);
    if (seedDev && seedDev[kSeedParity]) sign = sign1;
    const int c0 = blockIdx.x * kCollideCells;
    const int nc = min(kCollideCells, P.Nc - c0);
    const int A = (int)(uint32_t)start[c0], B = (int)(uint32_t)start[c0 + nc];
    const int t = threadIdx.x;
    if (B - A > tileCap) {
        if (t < nc) {
            const uint64_t s0 = start[c0 + t];
            const int a = (int)(uint32_t)s0, m = (int)(uint32_t)start[c0 + t + 1] - a;
            if (m > 0)
                collide_cell(P, s0, m, sign, signCount, st, [&](int j) { return S.vel(slots[a + j]); },
                             [&](int j, double2 w) { S.set_vel(slots[a + j], w); });
        }
        return;
    }
#pragma unroll 4
    for (int i = t; i < B - A; i += blockDim.x) {
        const int sl = slots[A + i];
        ts[i] = sl;
        tv[i] = S.vel(sl);
    }
    __syncthreads();
    if (t < nc) {
        const uint64_t s0 = start[c0 + t];
        const int a = (int)(uint32_t)s0 - A, m = (int)(uint32_t)start[c0 + t + 1] - A - a;
        if (m > 0)
            collide_cell(P, s0, m, sign, signCount, st, [&](int j) { return tv[a + j]; },
                         [&](int j, double2 w) { tv[a + j] = w; });
    }
    __syncthreads();
    for (int i = t; i < B - A; i += blockDim.x) S.set_vel(ts[i], tv[i]);
}

struct FieldsOut {
    int* N;
    double *Ux, *Uy, *Px, *Py, *T, *rho, *Pkin, *Pvir, *P, *rhoTarget;
};

// compute_cell_fields (src/common_grid.cpp:32-100), one cell per thread.
template <class V>
__global__ void k_cell_fields(DevParams Pm, const uint64_t* __restrict__ start, const int* __restrict__ slots, V S,
                              double rhoTarget, FieldsOut o, const int* skip = nullptr) {
    if (skip && *skip) return;  // a learned-closure step needs no reference fields
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Pm.Nc) return;
    const int a = (int)(uint32_t)start[c], b = (int)(uint32_t)start[c + 1];
    const int m = b - a;
    double px = 0.0, py = 0.0;
    for (int j = a; j < b; ++j) {
        const double2 w = S.vel(slots[j]);
        px = __dadd_rn(px, w.x);
        py = __dadd_rn(py, w.y);
    }
    double ux = 0.0, uy = 0.0;
    if (m > 0) {
        ux = __ddiv_rn(px, (double)m);
        uy = __ddiv_rn(py, (double)m);
    }
    const double rho = __ddiv_rn((double)m, Pm.Vc);
    double T = 0.0, pk = 0.0;
    const int dof = 2 * max(m - 1, 0);
    if (dof > 0 && (o.T || o.Pkin || o.P)) {
        double s2 = 0.0;
        for (int j = a; j < b; ++j) {
            const double2 w = S.vel(slots[j]);
            const double ax = __dsub_rn(w.x, ux), ay = __dsub_rn(w.y, uy);
            s2 = __dadd_rn(s2, __dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)));
        }
        T = __ddiv_rn(s2, (double)dof);
        pk = __dmul_rn(rho, T);
    }
    const double pv = __dmul_rn(Pm.Kvirial, __dsub_rn(rho, rhoTarget));
    if (o.N) o.N[c] = m;
    if (o.Ux) o.Ux[c] = ux;
    if (o.Uy) o.Uy[c] = uy;
    if (o.Px) o.Px[c] = px;
    if (o.Py) o.Py[c] = py;
    if (o.T) o.T[c] = T;
    if (o.rho) o.rho[c] = rho;
    if (o.Pkin) o.Pkin[c] = pk;
    if (o.Pvir) o.Pvir[c] = pv;
    if (o.P) o.P[c] = __dadd_rn(pk, pv);
    if (o.rhoTarget) o.rhoTarget[c] = rhoTarget;
}

}  // namespace mpcd_dev
