// Cell index: for every cell, the slots of its particles in ascending particle id.
//
// The reference walks particles in id order whenever it accumulates per-cell sums
// (src/common_grid.cpp:62-67, src/srd_collision.cpp:61-66) or builds per-cell lists
// (src/zone_pass.cpp:112-118). Ordering each cell's slots by particle id makes every
// per-cell FP64 sum on the device run in exactly that order, so sums are bit-identical.
//
// Build: warp-aggregated histogram with atomics (one atomic per run of equal cell ids in a
// warp), exclusive scan of the counts, scatter of (particle id, slot) keys into the cells'
// segments, then a rank sort of each tile of cells in shared memory: an entry's place in its
// cell is the number of the cell's keys below its own.
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
// A cell's count is scanned packed as (count, count >= 2), so one scan yields both the segment
// starts and the rank of each cell among cells holding at least two particles (the SRD sign
// stream index). Each count is cleared once read, ready for the next build's histogram.
__device__ __forceinline__ uint64_t pack_count(int k) { return (uint64_t)(uint32_t)k | ((uint64_t)(k >= 2) << 32); }

// k_scan_reduce over the packed counts
__global__ void k_count_scan_reduce(const int* __restrict__ count, int64_t n, uint64_t* __restrict__ blockSums) {
    __shared__ uint64_t sh[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint64_t s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += pack_count(count[i]);
    }
    uint64_t tot;
    block_exclusive_scan(s, sh, &tot);
    if (threadIdx.x == 0) blockSums[blockIdx.x] = tot;
}

// k_scan_apply over the packed counts, clearing them
__global__ void k_count_scan_apply(int* __restrict__ count, int64_t n, const uint64_t* __restrict__ blockSums,
                                   uint64_t* __restrict__ out) {
    __shared__ uint64_t sh[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint64_t v[kScanItems];
    uint64_t s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = 0ULL;
        if (base + k < n) {
            v[k] = pack_count(count[base + k]);
            count[base + k] = 0;
        }
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

// one block: the packed counts' exclusive scan into start (Nc <= kSmallScan), clearing the counts
__device__ __forceinline__ void scan_counts_small_block(int* __restrict__ count, int Nc, uint64_t* __restrict__ start) {
    __shared__ uint64_t sh[32];
    const int per = (Nc + kScanThreads - 1) / kScanThreads;
    const int a = min(Nc, (int)threadIdx.x * per), b = min(Nc, a + per);
    uint64_t sum = 0;
    for (int i = a; i < b; ++i) {
        sum += pack_count(count[i]);
    }
    uint64_t tot;
    uint64_t ex = block_exclusive_scan(sum, sh, &tot);
    for (int i = a; i < b; ++i) {
        const int k = count[i];
        count[i] = 0;
        start[i] = ex;
        ex += pack_count(k);
    }
    if (threadIdx.x == 0) start[Nc] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_counts_small(int* __restrict__ count, int Nc,
                                                                     uint64_t* __restrict__ start) {
    scan_counts_small_block(count, Nc, start);
}

// pos[s] = arrival order of slot s within its cell (any order; fixed by k_cell_rank).
// One atomic per run of equal cell ids among consecutive lanes: after the end-of-step
// re-sort, slots are ordered by cell, so a warp's lanes form a few long runs. Each warp
// covers kIndexItems runs of 32 consecutive slots, whose atomics are in flight together.
constexpr int kIndexItems = 4;

__device__ __forceinline__ void histogram_block(int blk, const int* __restrict__ cid, int n, int* __restrict__ count,
                                                int* __restrict__ pos) {
    const int lane = threadIdx.x & 31;
    const int base = ((blk * (int)blockDim.x + (int)threadIdx.x) >> 5) * (32 * kIndexItems) + lane;
    int c[kIndexItems], got[kIndexItems], runStart[kIndexItems];
#pragma unroll
    for (int k = 0; k < kIndexItems; ++k) c[k] = (base + 32 * k < n) ? cid[base + 32 * k] : -1;
#pragma unroll
    for (int k = 0; k < kIndexItems; ++k) {
        const int prev = __shfl_up_sync(0xffffffffu, c[k], 1);
        const bool headOfRun = (lane == 0) || (prev != c[k]);
        const unsigned heads = __ballot_sync(0xffffffffu, headOfRun);
        // run start = highest head lane <= lane; run end = next head lane
        runStart[k] = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
        const unsigned after = heads & ~(0xffffffffu >> (31 - lane));
        const int runEnd = after ? (__ffs(after) - 1) : 32;
        got[k] = (headOfRun && c[k] >= 0) ? atomicAdd(&count[c[k]], runEnd - runStart[k]) : 0;
    }
#pragma unroll
    for (int k = 0; k < kIndexItems; ++k) {
        const int b = __shfl_sync(0xffffffffu, got[k], runStart[k]);
        if (base + 32 * k < n) pos[base + 32 * k] = b + (lane - runStart[k]);
    }
}

__global__ void k_histogram(const int* __restrict__ cid, int n, int* __restrict__ count, int* __restrict__ pos) {
    histogram_block((int)blockIdx.x, cid, n, count, pos);
}

// keys[start[cid[s]] + pos[s]] = (pid[s] << 32) | s: each cell's segment holds its
// particles' keys in arrival order (same slot coverage as k_histogram)
__device__ __forceinline__ void scatter_keys_block(int blk, const int* __restrict__ cid, const int* __restrict__ pos,
                                                   const int* __restrict__ pid, int n,
                                                   const uint64_t* __restrict__ start, uint64_t* __restrict__ keys) {
    const int lane = threadIdx.x & 31;
    const int base = ((blk * (int)blockDim.x + (int)threadIdx.x) >> 5) * (32 * kIndexItems) + lane;
    int c[kIndexItems], p[kIndexItems], q[kIndexItems];
#pragma unroll
    for (int k = 0; k < kIndexItems; ++k) {
        const int s = base + 32 * k;
        c[k] = s < n ? cid[s] : 0;
        p[k] = s < n ? pos[s] : 0;
        q[k] = s < n ? pid[s] : 0;
    }
    uint32_t at[kIndexItems];
#pragma unroll
    for (int k = 0; k < kIndexItems; ++k) at[k] = (uint32_t)start[c[k]];
#pragma unroll
    for (int k = 0; k < kIndexItems; ++k) {
        const int s = base + 32 * k;
        if (s < n) keys[at[k] + p[k]] = ((uint64_t)(uint32_t)q[k] << 32) | (uint32_t)s;
    }
}

__global__ void k_scatter_keys(const int* __restrict__ cid, const int* __restrict__ pos, const int* __restrict__ pid,
                               int n, const uint64_t* __restrict__ start, uint64_t* __restrict__ keys) {
    scatter_keys_block((int)blockIdx.x, cid, pos, pid, n, start, keys);
}

constexpr int kRankThreads = 128;
constexpr int kRankCap = 2048;  // keys of one shared-memory tile (24 KB with their segment words)

// cells per block of k_cell_rank: a power of two giving about 1,280 keys per block at the
// mean occupancy (so a tile rarely needs splitting)
inline int rank_cells_per_block(int64_t n, int Nc) {
    const double mean = Nc > 0 ? (double)n / (double)Nc : 1.0;
    int cells = 1;
    while (cells < 4096 && (double)(2 * cells) * mean <= 1280.0) cells *= 2;
    return cells;
}

__device__ __forceinline__ int seg_lo(uint64_t s) { return (int)(uint32_t)s; }

// slots[start[c] + rank] = slot of the key of that rank among cell c's keys (ascending
// particle id; ids are unique, so they alone rank a cell's keys). A block takes cellsPerBlock
// consecutive cells, stages their ids and slots in shared memory (splitting the run of cells
// where it exceeds kRankCap keys) and ranks each key against its own cell's ids. A cell above
// kRankCap keys on its own is ranked from global memory.
__device__ __forceinline__ void cell_rank_block(int blk, const uint64_t* __restrict__ start, int Nc, int cellsPerBlock,
                                                const uint64_t* __restrict__ keys, int* __restrict__ slots) {
    __shared__ uint32_t kid[kRankCap];   // particle id
    __shared__ int ksl[kRankCap];        // slot
    __shared__ uint32_t seg[kRankCap];   // per key: its cell's segment [a, b) in the tile, a | b << 16
    const int t = threadIdx.x;
    const int c0 = (int)min((int64_t)blk * cellsPerBlock, (int64_t)Nc);
    const int c1 = min(Nc, c0 + cellsPerBlock);
    int cs = c0;
    while (cs < c1) {  // block-uniform
        const int A = seg_lo(start[cs]);
        int ce = c1;
        if (seg_lo(start[c1]) - A > kRankCap) {
            int lo = cs, hi = c1 - 1;  // the last ce with start[ce] - A <= kRankCap
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (seg_lo(start[mid]) - A <= kRankCap)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            ce = lo;
        }
        if (ce == cs) {
            const int b = seg_lo(start[cs + 1]);
            for (int i = A + t; i < b; i += kRankThreads) {
                const uint64_t k = keys[i];
                const uint32_t id = (uint32_t)(k >> 32);
                int r = 0;
                for (int j = A; j < b; ++j) r += (uint32_t)(keys[j] >> 32) < id;
                slots[A + r] = (int)(uint32_t)k;
            }
            ++cs;
            continue;
        }
        const int m = seg_lo(start[ce]) - A;
#pragma unroll 4
        for (int i = t; i < m; i += kRankThreads) {
            const uint64_t k = keys[A + i];
            kid[i] = (uint32_t)(k >> 32);
            ksl[i] = (int)(uint32_t)k;
        }
        for (int c = cs + t; c < ce; c += kRankThreads) {
            const int a = seg_lo(start[c]) - A, b = seg_lo(start[c + 1]) - A;
            for (int j = a; j < b; ++j) seg[j] = (uint32_t)a | ((uint32_t)b << 16);
        }
        __syncthreads();
        for (int i = t; i < m; i += kRankThreads) {
            const uint32_t sg = seg[i];
            const int a = (int)(sg & 0xffffu), b = (int)(sg >> 16);
            const uint32_t id = kid[i];
            int r = 0;
#pragma unroll 4
            for (int j = a; j < b; ++j) r += kid[j] < id;
            slots[A + a + r] = ksl[i];
        }
        __syncthreads();
        cs = ce;
    }
}

__global__ void __launch_bounds__(kRankThreads) k_cell_rank(const uint64_t* __restrict__ start, int Nc,
                                                            int cellsPerBlock, const uint64_t* __restrict__ keys,
                                                            int* __restrict__ slots) {
    cell_rank_block((int)blockIdx.x, start, Nc, cellsPerBlock, keys, slots);
}

// ------------------------------------------------------------------ batched index builds
// The index builds of many contexts (the replicas of a batch) as one launch per kernel: job r
// is one context's build; blocks [offs[r], offs[r + 1]) of a launch are its blocks.
struct IndexJob {
    const int* cid;
    int* count;
    int* pos;
    uint64_t* start;
    int* slots;
    const int* pid;
    uint64_t* keys;
    int n, Nc, rankCells;
};

// the job r with offs[r] <= b < offs[r + 1] (offs ascending, offs[0] = 0)
__device__ __forceinline__ int job_of(const int* __restrict__ offs, int nJobs, int b) {
    int lo = 0, hi = nJobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (offs[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// offs: blocks of kThreads threads covering each job's slots (kIndexItems per thread)
__global__ void k_histogram_batch(const IndexJob* __restrict__ jobs, const int* __restrict__ offs, int nJobs) {
    const int b = (int)blockIdx.x;
    if (nJobs <= 0 || b >= offs[nJobs]) return;
    const int r = job_of(offs, nJobs, b);
    const IndexJob J = jobs[r];
    histogram_block(b - offs[r], J.cid, J.n, J.count, J.pos);
}

// one block per job (every job has Nc <= kSmallScan)
__global__ void __launch_bounds__(kScanThreads) k_scan_counts_small_batch(const IndexJob* __restrict__ jobs) {
    const IndexJob J = jobs[blockIdx.x];
    scan_counts_small_block(J.count, J.Nc, J.start);
}

__global__ void k_scatter_keys_batch(const IndexJob* __restrict__ jobs, const int* __restrict__ offs, int nJobs) {
    const int b = (int)blockIdx.x;
    if (nJobs <= 0 || b >= offs[nJobs]) return;
    const int r = job_of(offs, nJobs, b);
    const IndexJob J = jobs[r];
    scatter_keys_block(b - offs[r], J.cid, J.pos, J.pid, J.n, J.start, J.keys);
}

// offs: blocks of each job's rank sort (ceil(Nc / rankCells))
__global__ void __launch_bounds__(kRankThreads) k_cell_rank_batch(const IndexJob* __restrict__ jobs,
                                                                  const int* __restrict__ offs, int nJobs) {
    const int b = (int)blockIdx.x;
    if (nJobs <= 0 || b >= offs[nJobs]) return;
    const int r = job_of(offs, nJobs, b);
    const IndexJob J = jobs[r];
    cell_rank_block(b - offs[r], J.start, J.Nc, J.rankCells, J.keys, J.slots);
}

}  // namespace mpcd_dev
