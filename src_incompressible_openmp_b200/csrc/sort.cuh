// Cell index: for every cell, the slots of its particles in ascending particle id.
//
// The reference walks particles in id order whenever it accumulates per-cell sums
// (src/common_grid.cpp:62-67, src/srd_collision.cpp:61-66) or builds per-cell lists
// (src/zone_pass.cpp:112-118). Ordering each cell's slots by particle id makes every
// per-cell FP64 sum on the device run in exactly that order, so sums are bit-identical.
//
// Build: warp-aggregated histogram with atomics (one atomic per run of equal cell ids in a
// warp), exclusive scan of the counts, scatter of slots, then an insertion sort of each
// cell's short segment by particle id.
#pragma once

#include "common.cuh"

namespace mpcd_dev {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// ------------------------------------------------------------------ exclusive scan (u64)
__global__ void k_scan_reduce(const uint64_t* __restrict__ in, int64_t n, uint64_t* __restrict__ blockSums) {
    __shared__ uint64_t sh[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint64_t s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint64_t tot;
    block_exclusive_scan(s, sh, &tot);
    if (threadIdx.x == 0) blockSums[blockIdx.x] = tot;
}

// single block: exclusive scan of nb block sums in place
__global__ void k_scan_blocks(uint64_t* __restrict__ blockSums, int nb) {
    __shared__ uint64_t sh[32];
    uint64_t carry = 0;
    for (int base = 0; base < nb; base += kScanThreads) {
        const int i = base + threadIdx.x;
        const uint64_t v = (i < nb) ? blockSums[i] : 0ULL;
        uint64_t tot;
        const uint64_t ex = block_exclusive_scan(v, sh, &tot);
        if (i < nb) blockSums[i] = carry + ex;
        carry += tot;
        __syncthreads();
    }
}

// out[i] = exclusive prefix of in; out[n] = total (out has n+1 entries)
__global__ void k_scan_apply(const uint64_t* __restrict__ in, int64_t n, const uint64_t* __restrict__ blockSums,
                             uint64_t* __restrict__ out) {
    __shared__ uint64_t sh[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint64_t v[kScanItems];
    uint64_t s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0ULL;
        s += v[k];
    }
    uint64_t tot;
    uint64_t ex = block_exclusive_scan(s, sh, &tot) + blockSums[blockIdx.x];
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = ex;
        ex += v[k];
    }
    if (base + kScanItems >= n && base < n) out[n] = ex;  // the thread holding the last element
}

// Arrays of at most kSmallScan entries are scanned by one block in one launch (a step of a
// small replica launches many short kernels, so their number counts).
constexpr int kSmallScan = 65536;

// one block: out[i] = exclusive prefix of in, out[n] = total (n <= kSmallScan)
__global__ void __launch_bounds__(kScanThreads) k_scan_small(const uint64_t* __restrict__ in, int n,
                                                              uint64_t* __restrict__ out) {
    __shared__ uint64_t sh[32];
    const int per = (n + kScanThreads - 1) / kScanThreads;
    const int a = min(n, (int)threadIdx.x * per), b = min(n, a + per);
    uint64_t sum = 0;
    for (int i = a; i < b; ++i) sum += in[i];
    uint64_t tot;
    uint64_t ex = block_exclusive_scan(sum, sh, &tot);
    for (int i = a; i < b; ++i) {
        const uint64_t v = in[i];
        out[i] = ex;
        ex += v;
    }
    if (threadIdx.x == 0) out[n] = tot;
}

// ------------------------------------------------------------------ cell index
// pack (count, count >= 2) so one scan yields both the segment starts and the rank of each
// cell among cells holding at least two particles (the SRD sign stream index). Each count is
// cleared once read, ready for the next build's histogram.
__global__ void k_pack_counts(int* __restrict__ count, int Nc, uint64_t* __restrict__ packed) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < Nc) {
        const int k = count[c];
        count[c] = 0;
        packed[c] = (uint64_t)(uint32_t)k | ((uint64_t)(k >= 2) << 32);
    }
}

// one block: the packed counts' exclusive scan into start (Nc <= kSmallScan), clearing the counts
__global__ void __launch_bounds__(kScanThreads) k_scan_counts_small(int* __restrict__ count, int Nc,
                                                                     uint64_t* __restrict__ start) {
    __shared__ uint64_t sh[32];
    const int per = (Nc + kScanThreads - 1) / kScanThreads;
    const int a = min(Nc, (int)threadIdx.x * per), b = min(Nc, a + per);
    uint64_t sum = 0;
    for (int i = a; i < b; ++i) {
        const int k = count[i];
        sum += (uint64_t)(uint32_t)k | ((uint64_t)(k >= 2) << 32);
    }
    uint64_t tot;
    uint64_t ex = block_exclusive_scan(sum, sh, &tot);
    for (int i = a; i < b; ++i) {
        const int k = count[i];
        count[i] = 0;
        start[i] = ex;
        ex += (uint64_t)(uint32_t)k | ((uint64_t)(k >= 2) << 32);
    }
    if (threadIdx.x == 0) start[Nc] = tot;
}

// pos[s] = arrival order of slot s within its cell (any order; fixed later by k_cell_sort).
// One atomic per run of equal cell ids among consecutive lanes: after the end-of-step
// re-sort, slots are ordered by cell, so a warp's lanes form a few long runs.
__global__ void k_histogram(const int* __restrict__ cid, int n, int* __restrict__ count, int* __restrict__ pos) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int c = (s < n) ? cid[s] : -1;
    const int prev = __shfl_up_sync(0xffffffffu, c, 1);
    const bool headOfRun = (lane == 0) || (prev != c);
    const unsigned heads = __ballot_sync(0xffffffffu, headOfRun);
    // run start = highest head lane <= lane; run end = next head lane
    const unsigned upTo = heads & (0xffffffffu >> (31 - lane));
    const int runStart = 31 - __clz(upTo);
    const unsigned after = heads & ~(0xffffffffu >> (31 - lane));
    const int runEnd = after ? (__ffs(after) - 1) : 32;
    int base = 0;
    if (headOfRun && c >= 0) base = atomicAdd(&count[c], runEnd - runStart);
    base = __shfl_sync(0xffffffffu, base, runStart);
    if (s < n) pos[s] = base + (lane - runStart);
}

__global__ void k_scatter(const int* __restrict__ cid, const int* __restrict__ pos, int n,
                          const uint64_t* __restrict__ start, int* __restrict__ slots) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) slots[(uint32_t)start[cid[s]] + pos[s]] = s;
}

// Bitonic sort of 16 or 32 keys held in registers (fully unrolled, no local memory).
template <int N>
__device__ __forceinline__ void bitonic_regs(uint64_t (&k)[N]) {
#pragma unroll
    for (int size = 2; size <= N; size <<= 1)
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1)
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = ((i & size) == 0);
                    const uint64_t a = k[i], b = k[j];
                    const bool sw = up ? (a > b) : (a < b);
                    k[i] = sw ? b : a;
                    k[j] = sw ? a : b;
                }
            }
}

template <int N>
__device__ __forceinline__ void sort_segment_regs(int a, int m, const int* __restrict__ pid, int* __restrict__ slots) {
    uint64_t k[N];
    int sl[N];
#pragma unroll
    for (int i = 0; i < N; ++i) sl[i] = (i < m) ? slots[a + i] : 0;
#pragma unroll
    for (int i = 0; i < N; ++i) k[i] = (i < m) ? (((uint64_t)(uint32_t)pid[sl[i]] << 32) | (uint32_t)sl[i]) : ~0ULL;
    bitonic_regs<N>(k);
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (i < m) slots[a + i] = (int)(uint32_t)k[i];
}

// sort each cell's slots by particle id (segments are short: ~ particles per cell)
__global__ void k_cell_sort(const uint64_t* __restrict__ start, int Nc, const int* __restrict__ pid,
                            int* __restrict__ slots) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Nc) return;
    const int a = (int)(uint32_t)start[c], b = (int)(uint32_t)start[c + 1];
    const int m = b - a;
    if (m <= 1) return;
    if (m <= 16) {
        sort_segment_regs<16>(a, m, pid, slots);
    } else if (m <= 32) {
        sort_segment_regs<32>(a, m, pid, slots);
    } else {
        // long segment: insertion sort in place in global memory
        for (int i = a + 1; i < b; ++i) {
            const int v = slots[i];
            const int pv = pid[v];
            int j = i;
            while (j > a && pid[slots[j - 1]] > pv) {
                slots[j] = slots[j - 1];
                --j;
            }
            slots[j] = v;
        }
    }
}

}  // namespace mpcd_dev
