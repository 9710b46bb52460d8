// Shared device definitions: the parameter block, error flags, MT19937-64 and the
// libstdc++-13 distributions restated for warp-uniform use on sm_100a.
//
// All FP64 arithmetic in this library is compiled with -fmad=false: every a*b+c rounds
// twice, exactly like the reference's x86-64 build (no FMA contraction).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ddmath.cuh"

namespace mpcd_dev {

constexpr int kWarp = 32;

// Device-side error codes (written to DevStatus::code with atomicCAS: first error wins).
enum DevError : int {
    kDevOk = 0,
    kErrUnsupportedBcLeft = 1,
    kErrUnsupportedBcRight = 2,
    kErrUnsupportedBcBottom = 3,
    kErrUnsupportedBcTop = 4,
    kErrZoneCapacity = 5,       // a zone list exceeded its provable bound
    kErrTableRange = 6,         // a minimal step outside the 5x5 tables
    kErrBcLateSweep = 7,        // a particle crossed a wall again after the first sweep
    kErrEventCapacity = 8,      // more wall events than the event buffer holds
    kErrCellId = 9,             // a caller-given cell id outside [0, Nc)
    kErrTargetIsSource = 10,    // a dense cell targeting itself (periodic axis shorter than 3)
    kErrRngCapacity = 11,       // the collision sign stream was shorter than needed
    kErrTensorWait = 12,        // a tensor-core MMA did not complete within the wait limit
    // 13, 14: the fast form's bin and record capacities (fast.cuh)
    kErrLearnedRange = 15       // a learned kick N du beyond the bound that keeps its int64 sum exact
};

struct DevStatus {
    int code;
    int detail;
    unsigned long long count;
};

__device__ __forceinline__ void raise_error(DevStatus* st, int code, int detail) {
    if (atomicCAS(&st->code, 0, code) == 0) st->detail = detail;
}

// Parameter block passed by value to every kernel. Derived constants are computed on the
// host once per context, with the host libm where the reference calls libm (cos, sin,
// atan2 and hypot of small integer steps).
struct DevParams {
    int Nx, Ny, Nc, n;
    double Lx, Ly, dt, a0, dx, dy, Vc;
    double invDx, invDy, invA0, invLx, invLy;  // correctly rounded reciprocals (floor_div)
    double alpha, kBT, g, bodyForceX;
    int useThermostat, keepMeanFlow;
    int bc[4];  // left, right, bottom, top (mpcd_bc_mode)
    int perx, pery;
    double Utop, Ubottom, wallSigma;
    int tileNx, tileNy, momCorr, maxPasses, useLFF, lowThrBulkInt, listBound, reserved0;
    double gamma, coef, highThr, lowThrBulk, lowFrac, highFrac, fluidFracGain, lowThrFloor, highThrFloor;
    int useLiquidClosure, useOptimalBetaRepair, smoothWidth, reserved1;
    double betaRepair, betaEOS, Kvirial, smoothBlend, rhoTarget;
    // rotation: index 0 -> theta = 0, 1 -> +alpha, 2 -> -alpha
    double rotCos[3], rotSin[3];
    // (ddx+2) + 5*(ddy+2) -> angular bin of atan2(ddy, ddx) and hypot(ddx, ddy)
    int atanBin[25];
    double hypotTab[25];
    // FP32 precision form: the largest FP32 offsets strictly inside a cell (x, y)
    float offMaxX, offMaxY;
};

// Device-side seed table of one step (CUDA-graph replay: the step number lives on the
// device and every seeded kernel reads its seed here instead of from its arguments).
// Seeds follow the benchmark schedule (src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:249-266).
enum StepSeed { kSeedBc = 0, kSeedSrdShift, kSeedSignsNext, kSeedBase, kSeedShifted, kSeedParity, kSeedNextParity,
                kStepSeeds };

__device__ __forceinline__ void step_begin(long long* __restrict__ step, uint64_t* __restrict__ seeds) {
    const long long s = *step + 1;
    *step = s;
    const uint64_t u = (uint64_t)s;
    seeds[kSeedBc] = 104729ULL + 10007ULL * u;
    seeds[kSeedSrdShift] = 130363ULL + 10007ULL * u;
    seeds[kSeedSignsNext] = 433494437ULL + 10007ULL * (u + 1ULL);
    seeds[kSeedBase] = 88172645463325252ULL + 10007ULL * u;
    seeds[kSeedShifted] = 88172645463325252ULL + 4099ULL + 10007ULL * u;
    seeds[kSeedParity] = u & 1ULL;
    seeds[kSeedNextParity] = (u + 1ULL) & 1ULL;
}

__device__ __forceinline__ int wrap_index(int i, int n) {
    int r = i % n;
    return (r < 0) ? r + n : r;
}

// std::max / std::min / std::clamp argument-order semantics (NaN-faithful)
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }

// reference src/common_grid.cpp:9-19
// floor(x / d) with the quotient correctly rounded, as floor(x / d) computes it, given
// invd = RN(1 / d). q = RN(x * invd) is within 2^-51 |q| of RN(x / d) (two roundings of
// 2^-53 each on the way to x / d, one more to RN(x / d)), so the two floors can differ only if
// an integer lies within 2^-51 |q| of q. Outside 2^-49 |q| of every integer floor(q) is
// returned; otherwise (cell boundaries hit exactly, |q| >= 2^52, NaN) the quotient is divided
// out. The multiply stands in for a division sequence of about twenty FP64 operations.
__device__ __forceinline__ double floor_div(double x, double d, double invd) {
    const double q = __dmul_rn(x, invd);
    const double f = floor(q);
    const double r = __dsub_rn(q, f);  // exact: q and floor(q) differ by less than one
    const double tol = __dmul_rn(fabs(q), 0x1p-49);
    if (r > tol && r < __dsub_rn(1.0, tol)) return f;
    return floor(__ddiv_rn(x, d));
}

__device__ __forceinline__ int cell_of(double x, double y, const DevParams& P) {
    int ix = (int)floor_div(x, P.dx, P.invDx), iy = (int)floor_div(y, P.dy, P.invDy);
    if (ix < 0) ix = 0;
    if (ix >= P.Nx) ix = P.Nx - 1;
    if (iy < 0) iy = 0;
    if (iy >= P.Ny) iy = P.Ny - 1;
    return iy + P.Ny * ix;
}

// ------------------------------------------------------------------ particle state views
// The step's kernels read and write the slot-ordered particle state through a view.
// View64, the plain form: FP64 positions and velocities (the reference's arithmetic, bit for
// bit). View32, the FP32 precision form: per slot the standard-grid cell (int32), the
// position inside that cell as FP32 offsets from the cell's lower corner, and FP32
// velocities (8 + 4 + 8 bytes instead of 32). Loads widen to FP64 and all arithmetic stays
// FP64; stores round to FP32 (positions relative to the cell, so to 2^-24 of a cell width).
struct View64 {
    double2* x;
    double2* v;
    static constexpr bool kF32 = false;
    __device__ __forceinline__ double2 pos(int s, const DevParams&) const { return x[s]; }
    // c: the standard-grid cell of X (cell_of), kept by the FP32 form
    __device__ __forceinline__ void set_pos(int s, double2 X, int, const DevParams&) const { x[s] = X; }
    __device__ __forceinline__ int std_cell(int s, const DevParams& P) const;
    __device__ __forceinline__ double2 vel(int s) const { return v[s]; }
    __device__ __forceinline__ void set_vel(int s, double2 V) const { v[s] = V; }
    // position of slot s of src into slot j (a permutation keeps the stored bits)
    __device__ __forceinline__ void copy_pos(int j, const View64& src, int s) const { x[j] = src.x[s]; }
};

struct View32 {
    float2* off;
    int* cell;
    float2* v;
    static constexpr bool kF32 = true;
    __device__ __forceinline__ double2 pos(int s, const DevParams& P) const {
        const int c = cell[s];
        const int ix = c / P.Ny, iy = c - ix * P.Ny;
        const float2 o = off[s];
        return make_double2(__dadd_rn(__dmul_rn((double)ix, P.dx), (double)o.x),
                            __dadd_rn(__dmul_rn((double)iy, P.dy), (double)o.y));
    }
    __device__ __forceinline__ void set_pos(int s, double2 X, int c, const DevParams& P) const {
        const int ix = c / P.Ny, iy = c - ix * P.Ny;
        const float ox = __double2float_rn(__dsub_rn(X.x, __dmul_rn((double)ix, P.dx)));
        const float oy = __double2float_rn(__dsub_rn(X.y, __dmul_rn((double)iy, P.dy)));
        off[s] = make_float2(fminf(fmaxf(ox, 0.0f), P.offMaxX), fminf(fmaxf(oy, 0.0f), P.offMaxY));
        cell[s] = c;
    }
    __device__ __forceinline__ int std_cell(int s, const DevParams&) const { return cell[s]; }
    __device__ __forceinline__ double2 vel(int s) const {
        const float2 w = v[s];
        return make_double2((double)w.x, (double)w.y);
    }
    __device__ __forceinline__ void set_vel(int s, double2 V) const {
        v[s] = make_float2(__double2float_rn(V.x), __double2float_rn(V.y));
    }
    __device__ __forceinline__ void copy_pos(int j, const View32& src, int s) const {
        off[j] = src.off[s];
        cell[j] = src.cell[s];
    }
};

__device__ __forceinline__ int View64::std_cell(int s, const DevParams& P) const { return cell_of(x[s].x, x[s].y, P); }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ------------------------------------------------------------------ MT19937-64
constexpr int kMtN = 312;
constexpr int kMtM = 156;
constexpr uint64_t kMtUM = 0xFFFFFFFF80000000ULL;
constexpr uint64_t kMtLM = 0x7FFFFFFFULL;
constexpr uint64_t kMtA = 0xB5026F5AA96619E9ULL;

__host__ __device__ __forceinline__ uint64_t mt_temper(uint64_t z) {
    z ^= (z >> 29) & 0x5555555555555555ULL;
    z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
    z ^= (z << 37) & 0xFFF7EEE000000000ULL;
    z ^= z >> 43;
    return z;
}

__host__ __device__ __forceinline__ uint64_t mt_mix(uint64_t a, uint64_t b) {
    const uint64_t y = (a & kMtUM) | (b & kMtLM);
    return (y >> 1) ^ ((y & 1ULL) ? kMtA : 0ULL);
}

// Sequential seeding recurrence (one thread).
__host__ __device__ __forceinline__ uint64_t mt_seed_next(uint64_t prev, int i) {
    return 6364136223846793005ULL * (prev ^ (prev >> 62)) + (uint64_t)i;
}

// Out-of-place twist of a 312-word state A into B by one warp (A is left intact). Not
// inlined: it is reached from every RNG call site and would otherwise bloat the zone kernel.
__device__ __noinline__ void mt_twist_warp(const uint64_t* A, uint64_t* B, int lane) {
    for (int i = lane; i < kMtN - kMtM; i += kWarp) B[i] = A[i + kMtM] ^ mt_mix(A[i], A[i + 1]);
    __syncwarp();
    for (int i = kMtN - kMtM + lane; i < kMtN - 1; i += kWarp) B[i] = B[i - (kMtN - kMtM)] ^ mt_mix(A[i], A[i + 1]);
    if (lane == 0) B[kMtN - 1] = B[kMtM - 1] ^ mt_mix(A[kMtN - 1], B[0]);
    __syncwarp();
}

// generate_canonical<double, 53> of one 64-bit draw
__device__ __forceinline__ double canon(uint64_t u) {
    double c = __dmul_rn(__ull2double_rn(u), 0x1p-64);  // exact scaling
    if (c >= 1.0) c = 0x1.fffffffffffffp-1;  // nextafter(1, 0)
    return c;
}

// Warp-uniform MT19937-64 stream over a double-buffered state in shared memory. Every lane
// of the warp must call the member functions with identical arguments (uniform control
// flow); the buffers are only written inside mt_twist_warp.
struct WarpMt {
    uint64_t* buf;  // 2 * 312 words: buffers 0 and 1
    int cur;        // buffer holding draws pos..311 of the current block
    int pos;        // next draw within the current block
    int nextReady;  // buffer cur^1 holds the following block
    int lane;

    __device__ __forceinline__ void init_from_seeded(int lane_) {
        lane = lane_;
        cur = 0;
        pos = kMtN;
        nextReady = 0;
    }
    // make draws pos .. pos+k-1 available (k <= 312)
    __device__ __forceinline__ void ensure(int k) {
        if (pos + k > kMtN && !nextReady) {
            mt_twist_warp(buf + cur * kMtN, buf + (cur ^ 1) * kMtN, lane);
            nextReady = 1;
        }
    }
    // draw i (0-based) past the current position; requires ensure(i+1) first
    __device__ __forceinline__ uint64_t peek(int i) const {
        const int j = pos + i;
        return mt_temper((j < kMtN) ? buf[cur * kMtN + j] : buf[(cur ^ 1) * kMtN + (j - kMtN)]);
    }
    // pos == 312 means the block is exhausted; a swap happens only once a draw past the
    // block end was taken (ensure() produced the next block before it was peeked)
    __device__ __forceinline__ void consume(int k) {
        pos += k;
        if (pos > kMtN) {
            cur ^= 1;
            pos -= kMtN;
            nextReady = 0;
        }
    }
    __device__ __forceinline__ uint64_t next() {
        ensure(1);
        const uint64_t u = peek(0);
        consume(1);
        return u;
    }
    __device__ __forceinline__ double u01() { return canon(next()); }
    // uniform_int_distribution on [lo, hi] (Lemire downscaling with 128-bit products)
    __device__ __forceinline__ uint64_t uint_in(uint64_t lo, uint64_t hi) {
        const uint64_t range = hi - lo + 1ULL;
        uint64_t u = next();
        uint64_t low = u * range;
        uint64_t high = __umul64hi(u, range);
        if (low < range) {
            const uint64_t thr = (0ULL - range) % range;
            while (low < thr) {
                u = next();
                low = u * range;
                high = __umul64hi(u, range);
            }
        }
        return high + lo;
    }
};

// log_cr as an out-of-line device function (shared by all call sites)
__device__ __noinline__ double log_cr_dev(double x) { return mpcd_dd::log_cr(x); }

// normal_distribution<double>(0, 1): Marsaglia polar method with one cached deviate
struct PolarNormal {
    double saved;
    int has;
    __device__ __forceinline__ void reset() { has = 0; saved = 0.0; }
    __device__ __forceinline__ double next(WarpMt& r) {
        if (has) {
            has = 0;
            return saved;
        }
        double x, y, r2;
        do {
            x = __dsub_rn(__dmul_rn(2.0, r.u01()), 1.0);
            y = __dsub_rn(__dmul_rn(2.0, r.u01()), 1.0);
            r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
        } while (r2 > 1.0 || r2 == 0.0);
        const double mult = sqrt(__ddiv_rn(__dmul_rn(-2.0, log_cr_dev(r2)), r2));
        saved = __dmul_rn(x, mult);
        has = 1;
        return __dmul_rn(y, mult);
    }
};

// std::shuffle of m entries at a (warp-uniform; lane 0 performs the swaps)
template <typename T>
__device__ __forceinline__ void warp_shuffle(T* a, int m, WarpMt& r, int lane) {
    if (m <= 0) return;
    int i = 1;
    if ((m % 2) == 0) {
        const int j = (int)r.uint_in(0, 1);
        if (lane == 0) {
            const T t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
        ++i;
    }
    while (i != m) {
        const uint64_t sr = (uint64_t)i + 1ULL;
        const uint64_t x = r.uint_in(0, sr * (sr + 1ULL) - 1ULL);
        const int p1 = (int)(x / (sr + 1ULL)), p2 = (int)(x % (sr + 1ULL));
        if (lane == 0) {
            T t = a[i];
            a[i] = a[p1];
            a[p1] = t;
            t = a[i + 1];
            a[i + 1] = a[p2];
            a[p2] = t;
        }
        i += 2;
    }
    __syncwarp();
}

// Block-wide exclusive scan of one u64 per thread (blockDim a multiple of 32, <= 1024).
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* sh, uint64_t* total) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    uint64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        uint64_t s = (lane < nw) ? sh[lane] : 0ULL;
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    const uint64_t warpPrefix = (wid > 0) ? sh[wid - 1] : 0ULL;
    if (total) *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warpPrefix + x - v;
}

}  // namespace mpcd_dev
