// Deterministic, stable LSD radix sort of 32-bit cell keys with 32-bit payload
// indices, and the incremental re-sort of a chained step.  No global atomics: each pass builds
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

// Blocks of a sort over *n_dev keys (a count on the device; the grid and the
// histogram stride are sized for nblk blocks of TILE keys), or nblk.
__device__ __forceinline__ int active_blocks(int nblk, int tile, const int* __restrict__ n_dev) {
    if (!n_dev) return nblk;
    const long long a = ((long long)*n_dev + tile - 1) / tile;
    return (int)(a < nblk ? a : nblk);
}

// Per-tile digit histogram.  hist is digit-major: hist[d * nblk + b] for tile
// b of TILE = 256 * ITEMS keys.  n_dev (may be null): sort the first *n_dev
// keys.  Blocks stride over the active tiles, so a grid smaller than nblk
// serves a device-side count without launching a block per possible tile.
template <int ITEMS>
__global__ void __launch_bounds__(SORT_THREADS)
radix_hist_kernel(const unsigned* __restrict__ keys, long long n, int shift, unsigned* __restrict__ hist, int nblk,
                  const int* __restrict__ n_dev) {
    constexpr int TILE = SORT_THREADS * ITEMS;
    if (n_dev) n = *n_dev;
    const long long tiles = (n + TILE - 1) / TILE;      // active tiles (a device-side count may leave some idle)
    __shared__ unsigned cnt[RADIX];
    for (long long b = blockIdx.x; b < tiles; b += gridDim.x) {
        for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) cnt[d] = 0;
        __syncthreads();
        const long long base = b * TILE;
#pragma unroll 4
        for (int r = 0; r < ITEMS; ++r) {
            const long long q = base + (long long)r * SORT_THREADS + threadIdx.x;
            if (q < n) atomicAdd(&cnt[(keys[q] >> shift) & (RADIX - 1)], 1u);
        }
        __syncthreads();
        for (int d = threadIdx.x; d < RADIX; d += SORT_THREADS) hist[(long long)d * nblk + b] = cnt[d];
        __syncthreads();
    }
}

// totals[d] = sum_b hist[d][b]   (one block per digit, fixed-order tree)
__global__ void __launch_bounds__(256)
radix_rowsum_kernel(const unsigned* __restrict__ hist, int nblk, unsigned* __restrict__ totals, int tile,
                    const int* __restrict__ n_dev) {
    const int nact = active_blocks(nblk, tile, n_dev);
    __shared__ unsigned red[256];
    int d = blockIdx.x;
    unsigned s = 0;
    for (int b = threadIdx.x; b < nact; b += 256) s += hist[(long long)d * nblk + b];
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
radix_rowscan_kernel(unsigned* __restrict__ hist, int nblk, const unsigned* __restrict__ totals, int tile,
                     const int* __restrict__ n_dev) {
    const int nact = active_blocks(nblk, tile, n_dev);
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
    for (int b0 = 0; b0 < nact; b0 += 256) {
        int b = b0 + threadIdx.x;
        unsigned v = (b < nact) ? hist[(long long)d * nblk + b] : 0u;
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
        if (b < nact) hist[(long long)d * nblk + b] = c + incl - v;
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
template <int ITEMS>
__global__ void __launch_bounds__(SORT_THREADS)
radix_scatter_kernel(const unsigned* __restrict__ keys_in, const unsigned* __restrict__ vals_in, long long n,
                     int shift, const unsigned* __restrict__ offs, int nblk,
                     unsigned* __restrict__ keys_out, unsigned* __restrict__ vals_out, const int* __restrict__ n_dev) {
    constexpr int TILE = SORT_THREADS * ITEMS;
    if (n_dev) n = *n_dev;
    const long long tiles = (n + TILE - 1) / TILE;
    constexpr int NW = SORT_THREADS / 32;
    constexpr int PER_WARP = TILE / NW;   // ITEMS rounds of 32 keys
    __shared__ unsigned wcnt[NW][RADIX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (long long b = blockIdx.x; b < tiles; b += gridDim.x) {
        for (int i = threadIdx.x; i < NW * RADIX; i += SORT_THREADS) (&wcnt[0][0])[i] = 0;
        __syncthreads();
        const long long wbase = b * TILE + (long long)warp * PER_WARP;
        unsigned key[ITEMS], val[ITEMS];
        // pass 1: digit counts of this warp's chunk
#pragma unroll
        for (int r = 0; r < ITEMS; ++r) {
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
            unsigned run = offs[(long long)d * nblk + b];
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
        for (int r = 0; r < ITEMS; ++r) {
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
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Incremental re-sort of a chained step.  The sorted order is by (cell key,
// particle index), the order of the stable radix sort of keys in particle
// order.  Between two steps few particles change cell: the emitting G2P of
// the previous step flags, per slot of the previous order and per particle,
// whether the particle's new key differs from its old one (a "mover").  The
// slots that keep their key ("stayers") are still in (key, particle) order.
// The movers are gathered in particle order and stable-sorted by key with the
// radix kernels on their device-side count (tiles of 256 keys, so that the few
// thousand movers spread over many blocks), which puts them in (key, particle)
// order; then the two sorted sequences are merged: the stayer at old slot q
// goes to q - (movers before q) + (movers ordered before it), mover i to
// i + (stayers ordered before it).  The result is exactly the full sort's.
// ---------------------------------------------------------------------------
constexpr int RESORT_THREADS = 256;        // threads per block; one 32-slot mask word per thread

// 32 flag bytes from index 32 w -> one mask word (bits of indices >= n clear)
__device__ __forceinline__ unsigned pack_flags(const unsigned char* __restrict__ flag, long long w, long long n) {
    const uint4* f = reinterpret_cast<const uint4*>(flag + (w << 5));
    const uint4 a = f[0], b = f[1];
    const unsigned wd[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    unsigned m = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if ((wd[i] >> (8 * j)) & 0xffu) m |= 1u << (4 * i + j);
    const long long rem = n - (w << 5);
    if (rem < 32) m &= (1u << rem) - 1u;
    return m;
}

__device__ __forceinline__ unsigned block_sum(unsigned c, unsigned* red) {
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    unsigned t = 0;
    for (int i = 0; i < RESORT_THREADS / 32; ++i) t += red[i];
    return t;
}

// Mover flags -> mask words, per slot (old order) and per particle, and each
// block's count of both.
__global__ void __launch_bounds__(RESORT_THREADS)
resort_count_kernel(const unsigned char* __restrict__ slot_flag, const unsigned char* __restrict__ part_flag,
                    long long n, unsigned* __restrict__ slot_mask, unsigned* __restrict__ part_mask,
                    unsigned* __restrict__ slot_blk, unsigned* __restrict__ part_blk) {
    __shared__ unsigned red[2][RESORT_THREADS / 32];
    const long long nw = (n + 31) >> 5;
    const long long w = (long long)blockIdx.x * RESORT_THREADS + threadIdx.x;
    unsigned ms = 0, mp = 0;
    if (w < nw) {
        ms = pack_flags(slot_flag, w, n);
        mp = pack_flags(part_flag, w, n);
        slot_mask[w] = ms;
        part_mask[w] = mp;
    }
    const unsigned cs = block_sum(__popc(ms), red[0]);
    const unsigned cp = block_sum(__popc(mp), red[1]);
    if (threadIdx.x == 0) {
        slot_blk[blockIdx.x] = cs;
        part_blk[blockIdx.x] = cp;
    }
}

// exclusive prefix of c over the block, from base
__device__ __forceinline__ unsigned block_prefix(unsigned c, unsigned* sh) {
    sh[threadIdx.x] = c;
    __syncthreads();
    for (int o = 1; o < RESORT_THREADS; o <<= 1) {
        const unsigned t = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0u;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    const unsigned r = sh[threadIdx.x] - c;
    __syncthreads();
    return r;
}

// After the block offsets are scanned: the movers before each slot mask word
// (wpre), and the movers' new keys and particle indices in particle order.
__global__ void __launch_bounds__(RESORT_THREADS)
resort_compact_kernel(const unsigned* __restrict__ slot_mask, const unsigned* __restrict__ part_mask, long long n,
                      const unsigned* __restrict__ slot_blk, const unsigned* __restrict__ part_blk,
                      const unsigned* __restrict__ keys, unsigned* __restrict__ wpre,
                      unsigned* __restrict__ mkey, unsigned* __restrict__ mpart) {
    __shared__ unsigned sh[RESORT_THREADS];
    const long long nw = (n + 31) >> 5;
    const long long w = (long long)blockIdx.x * RESORT_THREADS + threadIdx.x;
    const unsigned ms = w < nw ? slot_mask[w] : 0u, mp = w < nw ? part_mask[w] : 0u;
    const unsigned ps = block_prefix(__popc(ms), sh);
    const unsigned pp = block_prefix(__popc(mp), sh);
    if (w >= nw) return;
    wpre[w] = slot_blk[blockIdx.x] + ps;
    unsigned rest = mp, idx = part_blk[blockIdx.x] + pp;
    while (rest) {
        const int b = __ffs(rest) - 1;
        rest &= rest - 1u;
        const long long p = (w << 5) + b;
        if (MPM_INB(idx, n, 10)) {
            mkey[idx] = keys[p];
            mpart[idx] = (unsigned)p;
        }
        ++idx;
    }
}

// movers before slot q of the old order
__device__ __forceinline__ unsigned resort_movers_before(const unsigned* __restrict__ mask,
                                                         const unsigned* __restrict__ wpre, long long q,
                                                         long long n, unsigned total) {
    if (q >= n) return total;
    const long long w = q >> 5;
    const int b = (int)(q & 31);
    return wpre[w] + __popc(mask[w] & ((1u << b) - 1u));
}

__device__ __forceinline__ unsigned long long pair_key(unsigned k, unsigned p) {
    return ((unsigned long long)k << 32) | p;
}

// first sorted mover not ordered before v, in [lo, hi)
__device__ __forceinline__ int mover_bound(const unsigned* __restrict__ mk, const unsigned* __restrict__ mp,
                                           unsigned long long v, int lo, int hi) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (pair_key(mk[mid], mp[mid]) < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// First index in [lo, hi) whose pair (keys[i], vals[i]) is not ordered before
// v, or hi: a 32-ary search by the whole warp (v, lo, hi warp-uniform).  Each
// step probes 32 evenly spaced indices and keeps the interval between the last
// probe ordered before v and the first one not, so about log_33 of the range
// dependent loads instead of log_2.
__device__ __forceinline__ long long warp_pair_bound(const unsigned* __restrict__ keys,
                                                     const unsigned* __restrict__ vals, unsigned long long v,
                                                     long long lo, long long hi) {
    const int lane = threadIdx.x & 31;
    while (hi - lo > 32) {
        const long long span = hi - lo;
        const long long idx = lo + ((long long)(lane + 1) * span) / 33;      // in [lo, hi) since span >= 33
        const bool before = pair_key(keys[idx], vals[idx]) < v;
        const int c = __popc(__ballot_sync(0xffffffffu, before));           // a prefix of the lanes
        const long long nlo = c > 0 ? lo + ((long long)c * span) / 33 + 1 : lo;
        const long long nhi = c < 32 ? lo + ((long long)(c + 1) * span) / 33 : hi;
        lo = nlo;
        hi = nhi;
    }
    const long long idx = lo + lane;
    const bool before = idx < hi && pair_key(keys[idx], vals[idx]) < v;
    return lo + __popc(__ballot_sync(0xffffffffu, before));
}

// Stayers to their new slots, one warp per STAY_ROUNDS x 32 consecutive old
// slots.  A stayer's new slot is its old slot, minus the movers before it in
// the old order, plus the sorted movers ordered before it.  The latter are
// bracketed once per warp (the warp's first and last slot; the old order is
// sorted, so every stayer of the warp lies between); inside the bracket, a few
// movers on average, each stayer finds its own count by a short search.
constexpr int STAY_ROUNDS = 8;
__global__ void __launch_bounds__(RESORT_THREADS)
resort_place_stayers_kernel(const unsigned* __restrict__ mask, const unsigned* __restrict__ wpre, long long n,
                            const unsigned* __restrict__ old_keys, const unsigned* __restrict__ old_perm,
                            const unsigned* __restrict__ mk, const unsigned* __restrict__ mp,
                            const int* __restrict__ n_movers, unsigned* __restrict__ keys_out,
                            unsigned* __restrict__ perm_out) {
    const int lane = threadIdx.x & 31;
    const long long c0 = ((long long)blockIdx.x * (RESORT_THREADS / 32) + (threadIdx.x >> 5)) * (32 * STAY_ROUNDS);
    if (c0 >= n) return;                                      // warp-uniform
    const long long cl = (c0 + 32 * STAY_ROUNDS < n ? c0 + 32 * STAY_ROUNDS : n) - 1;   // last slot of the warp
    const int nm = *n_movers;
    unsigned k[STAY_ROUNDS], pv[STAY_ROUNDS], mw[STAY_ROUNDS], wp[STAY_ROUNDS];
#pragma unroll
    for (int r = 0; r < STAY_ROUNDS; ++r) {
        const long long q = c0 + r * 32 + lane;
        const bool valid = q < n;
        k[r] = valid ? old_keys[q] : 0u;
        pv[r] = valid ? old_perm[q] : 0u;
        const long long w = (c0 >> 5) + r;                  // the round's mask word (c0 is a multiple of 32)
        const bool wv = (w << 5) < n;
        mw[r] = wv ? mask[w] : 0xffffffffu;
        wp[r] = wv ? wpre[w] : 0u;
    }
    const unsigned long long v_first = pair_key(__shfl_sync(0xffffffffu, k[0], 0), __shfl_sync(0xffffffffu, pv[0], 0));
    const unsigned long long v_last = pair_key(old_keys[cl], old_perm[cl]);
    const int j_lo = (int)warp_pair_bound(mk, mp, v_first, 0, nm);
    const int j_hi = (int)warp_pair_bound(mk, mp, v_last, j_lo, nm);
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < STAY_ROUNDS; ++r) {
        const long long q = c0 + r * 32 + lane;
        if (q >= n || ((mw[r] >> lane) & 1u)) continue;
        const int j = mover_bound(mk, mp, pair_key(k[r], pv[r]), j_lo, j_hi);
        const long long pos = q - (long long)(wp[r] + __popc(mw[r] & lt)) + j;
        if (MPM_INB(pos, n, 10)) {
            keys_out[pos] = k[r];
            perm_out[pos] = pv[r];
        }
    }
}

// Movers to their new slots: one mover per warp at a time, its count of old
// slots ordered before it by the warp's 32-ary search.
__global__ void __launch_bounds__(RESORT_THREADS)
resort_place_movers_kernel(const unsigned* __restrict__ mask, const unsigned* __restrict__ wpre, long long n,
                           const unsigned* __restrict__ old_keys, const unsigned* __restrict__ old_perm,
                           const unsigned* __restrict__ mk, const unsigned* __restrict__ mp,
                           const int* __restrict__ n_movers, unsigned* __restrict__ keys_out,
                           unsigned* __restrict__ perm_out) {
    const int nm = *n_movers;
    const long long warps = (long long)gridDim.x * (RESORT_THREADS / 32);
    for (long long i = (long long)blockIdx.x * (RESORT_THREADS / 32) + (threadIdx.x >> 5); i < nm; i += warps) {
        const unsigned k = mk[i], p = mp[i];
        const long long lo = warp_pair_bound(old_keys, old_perm, pair_key(k, p), 0, n);
        if ((threadIdx.x & 31) == 0) {
            const long long pos = i + lo - (long long)resort_movers_before(mask, wpre, lo, n, (unsigned)nm);
            if (MPM_INB(pos, n, 10)) {
                keys_out[pos] = k;
                perm_out[pos] = p;
            }
        }
    }
}

}  // namespace mpm