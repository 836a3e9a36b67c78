// Deterministic, stable LSD radix sort of 32-bit cell keys with 32-bit payload
// indices, and the tile-list compaction.  No global atomics: each pass builds
// per-block digit counts (shared-memory counters), scans them digit-major into
// global offsets (row totals, then per-digit row scans) and scatters every key
// to offset + its stable rank inside the block, ranked with warp match masks.
#pragma once

#include "mpm_common.cuh"

namespace mpm {

constexpr int RADIX_BITS = 9;
constexpr int RADIX = 1 << RADIX_BITS;
constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 16;                       // keys per thread per block
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS; // keys per block

// Per-block digit histogram.  hist is digit-major: hist[d * nblk + b].
__global__ void __launch_bounds__(SORT_THREADS)
radix_hist_kernel(const unsigned* __restrict__ keys, long long n, int shift, unsigned* __restrict__ hist, int nblk) {
    __shared__ unsigned cnt[RADIX];
    for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) cnt[d] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * SORT_TILE;
#pragma unroll 4
    for (int r = 0; r < SORT_ITEMS; ++r) {
        long long q = base + (long long)r * SORT_THREADS + threadIdx.x;
        if (q < n) atomicAdd(&cnt[(keys[q] >> shift) & (RADIX - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) hist[(long long)d * nblk + blockIdx.x] = cnt[d];
}

// totals[d] = sum_b hist[d][b]   (one block per digit, fixed-order tree)
__global__ void __launch_bounds__(256)
radix_rowsum_kernel(const unsigned* __restrict__ hist, int nblk, unsigned* __restrict__ totals) {
    __shared__ unsigned red[256];
    int d = blockIdx.x;
    unsigned s = 0;
    for (int b = threadIdx.x; b < nblk; b += 256) s += hist[(long long)d * nblk + b];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) totals[d] = red[0];
}

// hist[d][b] <- sum_{d'<d} totals[d'] + sum_{b'<b} hist[d][b']   (one block per digit)
__global__ void __launch_bounds__(256)
radix_rowscan_kernel(unsigned* __restrict__ hist, int nblk, const unsigned* __restrict__ totals) {
    __shared__ unsigned sh[256];
    __shared__ unsigned carry;
    int d = blockIdx.x;
    // digit offset: sum of the totals of the smaller digits
    unsigned part = 0;
    for (int e = threadIdx.x; e < d; e += 256) part += totals[e];
    sh[threadIdx.x] = part;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) carry = sh[0];
    __syncthreads();
    for (int b0 = 0; b0 < nblk; b0 += 256) {
        int b = b0 + threadIdx.x;
        unsigned v = (b < nblk) ? hist[(long long)d * nblk + b] : 0u;
        sh[threadIdx.x] = v;
        __syncthreads();
        // Hillis-Steele inclusive scan
        for (int o = 1; o < 256; o <<= 1) {
            unsigned t = (threadIdx.x >= (unsigned)o) ? sh[threadIdx.x - o] : 0u;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        unsigned incl = sh[threadIdx.x];
        unsigned c = carry;
        if (b < nblk) hist[(long long)d * nblk + b] = c + incl - v;
        __syncthreads();
        if (threadIdx.x == 255) carry = c + incl;
        __syncthreads();
    }
}

// Stable scatter.  vals_in == nullptr means the identity payload (slot index).
// Warp w of a block owns the contiguous chunk [w*PER_WARP, (w+1)*PER_WARP) of
// the block's tile, so the order (warp, round, lane) is the input order.
// Pass 1 counts each warp's digits, one block-wide prefix turns the counts
// into the warps' output offsets per digit, pass 2 scatters: a key's
// position is its warp's running offset for its digit plus its rank among the
// lanes of its round with the same digit (warp match masks).
__global__ void __launch_bounds__(SORT_THREADS)
radix_scatter_kernel(const unsigned* __restrict__ keys_in, const unsigned* __restrict__ vals_in, long long n,
                     int shift, const unsigned* __restrict__ offs, int nblk,
                     unsigned* __restrict__ keys_out, unsigned* __restrict__ vals_out) {
    constexpr int NW = SORT_THREADS / 32;
    constexpr int PER_WARP = SORT_TILE / NW;   // SORT_ITEMS rounds of 32 keys
    __shared__ unsigned wcnt[NW][RADIX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int i = threadIdx.x; i < NW * RADIX; i += SORT_THREADS) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const long long wbase = (long long)blockIdx.x * SORT_TILE + (long long)warp * PER_WARP;
    unsigned key[SORT_ITEMS], val[SORT_ITEMS];
    // pass 1: digit counts of this warp's chunk
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        const long long q = wbase + (long long)r * 32 + lane;
        const bool valid = q < n;
        key[r] = valid ? keys_in[q] : 0u;
        val[r] = valid ? (vals_in ? vals_in[q] : (unsigned)q) : 0u;
        const unsigned dig = (key[r] >> shift) & (RADIX - 1);
        const unsigned vmask = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const unsigned peers = __match_any_sync(vmask, dig);
            if ((peers & lt_mask) == 0) wcnt[warp][dig] += __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over the warps, from the block's offset
    for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) {
        unsigned run = offs[(long long)d * nblk + blockIdx.x];
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const unsigned c = wcnt[w][d];
            wcnt[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
    // pass 2: scatter
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        const long long q = wbase + (long long)r * 32 + lane;
        const bool valid = q < n;
        const unsigned dig = (key[r] >> shift) & (RADIX - 1);
        const unsigned vmask = __ballot_sync(0xffffffffu, valid);
        unsigned peers = 0, rank = 0, base = 0;
        int leader = lane;
        if (valid) {
            peers = __match_any_sync(vmask, dig);
            rank = __popc(peers & lt_mask);
            leader = __ffs(peers) - 1;
            if (rank == 0) base = wcnt[warp][dig];
        }
        base = __shfl_sync(0xffffffffu, base, leader);
        if (valid && MPM_INB((long long)base + rank, n, 10)) {
            keys_out[base + rank] = key[r];
            vals_out[base + rank] = val[r];
        }
        __syncwarp();
        if (valid && rank == 0) wcnt[warp][dig] = base + __popc(peers);
        __syncwarp();
    }
}

}  // namespace mpm
