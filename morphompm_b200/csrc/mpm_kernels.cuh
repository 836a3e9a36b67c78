// Kernels of one MLS-MPM growth step and of its reverse.
//
// Forward (python/morphompm/transfer.py:33-79):
//   bin_kernel        cell key of every particle (stencil base, exact rounding)
//   radix sort        (sort.cuh) cell-sorted particle order, deterministic
//   seg_* kernels     segment table of the occupied cells + active tile flags
//   compact_tiles     active node tiles -> compact grid slots
//   prepass_kernel    stress and the P2G record of every particle (particle order);
//                     in a chain of steps the previous G2P forms them instead
//   cell_sums_kernel  P2G phase 1: per occupied cell, its 27 stencil sums
//   node_sums_kernel  P2G phase 2: per node, the sums of its 27 source cells
//                     in a fixed order, + grid update with boundary conditions
//   g2p_kernel        gather, advect, F update; clears the cell marks; in a
//                     chain also bins the new state and forms its P2G records
// Reverse (python/morphompm/transfer.py:82-158):
//   cell_sums_adj     gv_b scatter phase 1 (nv_b, Cn_b' formed per particle)
//   node_sums<1>      gv_b gather + grid adjoint (gmom_b, gm_b)
//   bwd_particle_kernel  P2G adjoint, constitutive VJP, volume path, x_b terms
//
// P2G determinism: particles are sorted by cell, every occupied cell's sums
// are formed by one thread in sorted particle order, and every node adds its
// source cells in the fixed order of the stencil offsets.  No atomics, no
// shared-memory races: the result does not depend on scheduling.
#pragma once

#include "mpm_common.cuh"
#include "constitutive.cuh"

namespace mpm {

constexpr int PAYLOAD = 16;   // fx[3], m, a[3], B[9]

template <typename R> struct Vec4;
template <> struct Vec4<float> { using T = float4; };
template <> struct Vec4<double> { using T = double2; };

template <typename R>
__device__ __forceinline__ void load_record(const R* __restrict__ base, long long q, R r[PAYLOAD]) {
    using V = typename Vec4<R>::T;
    const V* p = reinterpret_cast<const V*>(base + q * PAYLOAD);
    constexpr int per = sizeof(V) / sizeof(R);
#pragma unroll
    for (int i = 0; i < PAYLOAD / per; ++i) {
        V v = __ldg(p + i);
        const R* e = reinterpret_cast<const R*>(&v);
#pragma unroll
        for (int k = 0; k < per; ++k) r[i * per + k] = e[k];
    }
}
template <typename R>
__device__ __forceinline__ void store_record(R* __restrict__ base, long long q, const R r[PAYLOAD]) {
    using V = typename Vec4<R>::T;
    V* p = reinterpret_cast<V*>(base + q * PAYLOAD);
    constexpr int per = sizeof(V) / sizeof(R);
#pragma unroll
    for (int i = 0; i < PAYLOAD / per; ++i) {
        V v;
        R* e = reinterpret_cast<R*>(&v);
#pragma unroll
        for (int k = 0; k < per; ++k) e[k] = r[i * per + k];
        p[i] = v;
    }
}
template <typename R>
__device__ __forceinline__ void load_node(const R* __restrict__ g, long long idx, R o[4]) {
    if constexpr (sizeof(R) == 4) {
        float4 v = __ldg(reinterpret_cast<const float4*>(g) + idx);
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    } else {
        const double2* p = reinterpret_cast<const double2*>(g) + 2 * idx;
        double2 a = __ldg(p), b = __ldg(p + 1);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
}
template <typename R>
__device__ __forceinline__ void store_node(R* __restrict__ g, long long idx, const R o[4]) {
    if constexpr (sizeof(R) == 4) {
        reinterpret_cast<float4*>(g)[idx] = make_float4(o[0], o[1], o[2], o[3]);
    } else {
        double2* p = reinterpret_cast<double2*>(g) + 2 * idx;
        p[0] = make_double2(o[0], o[1]);
        p[1] = make_double2(o[2], o[3]);
    }
}

__device__ __forceinline__ bool node_free(const MpmScene& sc, int i, int j, int k) {
    if (sc.wall > 0) {
        int w = sc.wall;
        if (i < w || j < w || k < w || i >= sc.shape[0] - w || j >= sc.shape[1] - w || k >= sc.shape[2] - w)
            return false;
    }
    if (sc.clamp_lo[0] < sc.clamp_hi[0] && sc.clamp_lo[1] < sc.clamp_hi[1] && sc.clamp_lo[2] < sc.clamp_hi[2]) {
        if (i >= sc.clamp_lo[0] && i < sc.clamp_hi[0] && j >= sc.clamp_lo[1] && j < sc.clamp_hi[1] &&
            k >= sc.clamp_lo[2] && k < sc.clamp_hi[2])
            return false;
    }
    return true;
}

// Fg of particle p (read, or the growth law)
template <typename R>
__device__ __forceinline__ void load_Fg(const Ctx& ctx, const MpmScene& sc, const MpmParticles& P, long long p,
                                        int t, R Fg[9], R* gphi) {
    if (sc.growth_mode == 1) {
        R phi = ctx.phi ? static_cast<const R*>(ctx.phi)[p] : R(1);
        R g = R(1) + (R)(sc.growth_A * growth_ramp(sc, t)) * phi;
#pragma unroll
        for (int i = 0; i < 9; ++i) Fg[i] = (i % 4 == 0) ? g : R(0);
        if (gphi) *gphi = (R)growth_ramp(sc, t) * phi;
    } else {
        ld9<R>(P.Fg, p, P.sp9, P.sc9, Fg);
        if (gphi) *gphi = R(0);
    }
}

// ---------------------------------------------------------------------------
// binning
// ---------------------------------------------------------------------------
// cell key of a particle at x (its padded stencil-base cell, or the scene's
// "outside" key) and its fractional position fx in the stencil
// Active tiles of the next step: the node tiles that the stencil of a particle
// inside the grid touches (nodes base..base+2 clipped to the grid), flagged
// where its cell key is formed.  Every particle of an occupied cell flags the
// same tiles; the flags are plain stores of 1.
__device__ __forceinline__ void flag_stencil_tiles(const Ctx& ctx, const MpmScene& sc, const SceneAux& ax,
                                                   const int base[3]) {
    int tlo[3], thi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int sh = d == 2 ? ctx.tile_z_shift : ctx.tile_xy_shift;
        const int lo = base[d] < 0 ? 0 : base[d];
        const int hi = base[d] + 2 > sc.shape[d] - 1 ? sc.shape[d] - 1 : base[d] + 2;
        tlo[d] = lo >> sh;
        thi[d] = hi >> sh;
    }
    for (int a = tlo[0]; a <= thi[0]; ++a)
        for (int b = tlo[1]; b <= thi[1]; ++b)
            for (int e = tlo[2]; e <= thi[2]; ++e) {
                const long long ti = ax.tile_begin + ((long long)a * ax.ntile[1] + b) * ax.ntile[2] + e;
                if (MPM_INB(ti, ctx.n_tiles, 1)) ctx.tile_flag[ti] = 1;
            }
}

template <typename R>
__device__ __forceinline__ unsigned particle_key(const Ctx& ctx, const MpmScene& sc, const SceneAux& ax,
                                                 const R x[3], R fx[3]) {
    int base[3];
    const bool inside = bin_particle(x, (R)(1.0 / sc.dx), sc.shape, base, fx);
    // the lanes of a warp in the same cell flag the same tiles: one of them does
    const long long cell = ((long long)(base[0] + 2) * (sc.shape[1] + 2) + (base[1] + 2)) * (sc.shape[2] + 2) +
                           (base[2] + 2);
    const unsigned tag = inside ? (unsigned)(ax.cell_begin + cell) : 0xffffffffu;
    const unsigned peers = __match_any_sync(__activemask(), tag);
    const bool leader = (peers & ((1u << (threadIdx.x & 31)) - 1u)) == 0u;
    if (inside) {
        if (leader) flag_stencil_tiles(ctx, sc, ax, base);
        return tag;
    }
    raise_status(ctx.status, MPM_WARN_OUTSIDE);
    return (unsigned)(ax.cell_begin + ax.ncells);
}

template <typename R>
__global__ void __launch_bounds__(256)
bin_kernel(Ctx ctx, MpmParticles P, unsigned* __restrict__ keys) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ctx.n) return;
    int s = ctx.scene_of[p];
    R x[3], fx[3];
    ld3<R>(P.x, p, P.sp3, P.sc3, x);
    keys[p] = particle_key<R>(ctx, ctx.scenes[s], ctx.aux[s], x, fx);
}

// keys of a single scene (C ABI mpm_bin_keys); local keys, no plan
template <typename R>
__global__ void bin_keys_single(MpmScene sc, long long n, const R* __restrict__ x, int* __restrict__ keys) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    R xp[3] = {x[3 * p], x[3 * p + 1], x[3 * p + 2]};
    int base[3];
    R fx[3];
    bool inside = bin_particle(xp, (R)(1.0 / sc.dx), sc.shape, base, fx);
    long long P0 = sc.shape[0] + 2, P1 = sc.shape[1] + 2, P2 = sc.shape[2] + 2;
    keys[p] = inside ? (int)(((base[0] + 2) * P1 + (base[1] + 2)) * P2 + (base[2] + 2)) : (int)(P0 * P1 * P2);
}

// ---------------------------------------------------------------------------
// segment tables: one segment per occupied cell (a run of equal sorted keys).
// Three kernels: per-block counts of segment starts, a
// single-block scan of the counts, and the writes of seg_first / seg_last /
// cell_seg with each slot's segment id from the scan.  "Outside" keys (stencil
// entirely off the grid) form no segment.
// ---------------------------------------------------------------------------
constexpr int SEG_THREADS = 256;

// Segment kernels: SEGK_ITEMS warp-striped rounds of slots per block (slot =
// block base + round*256 + thread, every key load coalesced), all their loads
// issued before any is used, few registers: a block waits on one chain of
// memory latencies (key, then its scene), not one per round.
#ifndef MPM_SEGK_ITEMS          // slots per thread (build-time; 4 measured fastest of 1, 2, 4, 8)
#define MPM_SEGK_ITEMS 4
#endif
constexpr int SEGK_ITEMS = MPM_SEGK_ITEMS;
constexpr int SEGK_TILE = SEG_THREADS * SEGK_ITEMS;

// Bit r of start / last: slot base + r*256 + thread starts / ends an inside
// segment (a run of equal keys whose cell lies in its scene's grid).
__device__ __forceinline__ void seg_flags(const Ctx& ctx, const unsigned* __restrict__ skeys, long long base,
                                          unsigned key[SEGK_ITEMS], unsigned& start, unsigned& last) {
    const int lane = threadIdx.x & 31;
    const long long n = ctx.n;
    unsigned edge[SEGK_ITEMS];
    int sid[SEGK_ITEMS];
#pragma unroll
    for (int r = 0; r < SEGK_ITEMS; ++r) {
        const long long s = base + (long long)r * SEG_THREADS + threadIdx.x;
        const bool valid = s < n;
        key[r] = valid ? skeys[s] : 0u;
        sid[r] = valid ? ctx.scene_of[s] : 0;
        // lane 0 needs the key before it, lane 31 the key after it
        const long long e = lane == 0 ? s - 1 : s + 1;
        edge[r] = ((lane == 0 || lane == 31) && e >= 0 && e < n) ? skeys[e] : 0u;
    }
    start = 0;
    last = 0;
#pragma unroll
    for (int r = 0; r < SEGK_ITEMS; ++r) {
        const long long s = base + (long long)r * SEG_THREADS + threadIdx.x;
        unsigned prv = __shfl_up_sync(0xffffffffu, key[r], 1);
        unsigned nxt = __shfl_down_sync(0xffffffffu, key[r], 1);
        if (lane == 0) prv = edge[r];
        if (lane == 31) nxt = edge[r];
        const bool valid = s < n;
        const bool a = valid && (s == 0 || prv != key[r]);
        const bool b = valid && (s == n - 1 || nxt != key[r]);
        if (a || b) {
            const SceneAux& ax = ctx.aux[sid[r]];
            if ((long long)key[r] - ax.cell_begin < ax.ncells) {
                start |= (a ? 1u : 0u) << r;
                last |= (b ? 1u : 0u) << r;
            }
        }
    }
}

__global__ void __launch_bounds__(SEG_THREADS)
seg_count_kernel(Ctx ctx, const unsigned* __restrict__ skeys) {
    __shared__ unsigned red[SEG_THREADS / 32];
    unsigned key[SEGK_ITEMS], start, last;
    seg_flags(ctx, skeys, (long long)blockIdx.x * SEGK_TILE, key, start, last);
    unsigned cnt = __popc(start);
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        for (int w = 0; w < SEG_THREADS / 32; ++w) t += red[w];
        ctx.blk_count[blockIdx.x] = t;
    }
}

// exclusive scan of per-block counts in place (single block of 1024 threads);
// the total, clamped to cap, goes to *total (a total above cap raises
// MPM_ERR_ARG).  Each thread sums a run of consecutive counts, the runs are
// scanned by warp shuffles and one pass over the 32 warp sums.
__global__ void __launch_bounds__(1024)
scan_counts_kernel(unsigned* __restrict__ cnt, int nblk, int* __restrict__ total, int cap, int* __restrict__ status) {
    __shared__ unsigned wsum[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int per = (nblk + 1023) / 1024;
    const long long b0 = (long long)threadIdx.x * per;
    unsigned loc = 0;
    for (int j = 0; j < per; ++j)
        if (b0 + j < nblk) loc += cnt[b0 + j];
    unsigned inc = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const unsigned w = wsum[lane];
        unsigned wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        wsum[lane] = wi - w;
    }
    __syncthreads();
    unsigned run = wsum[warp] + inc - loc;
    for (int j = 0; j < per; ++j) {
        if (b0 + j < nblk) {
            const unsigned v = cnt[b0 + j];
            cnt[b0 + j] = run;
            run += v;
        }
    }
    if (threadIdx.x == 1023) {       // its run ends at the grand total
        unsigned c = run;
        if (c > (unsigned)cap) {
            raise_status(status, MPM_ERR_ARG);
            c = (unsigned)cap;
        }
        *total = (int)c;
    }
}

// Reverse step: the segment table is the one the forward step recorded in the
// tape; only the dense cell marks (cleared by the forward G2P) are restored.
__global__ void __launch_bounds__(256)
remark_cells_kernel(Ctx ctx, const unsigned* __restrict__ skeys) {
    const int nseg = *ctx.n_seg;
    // NB segments per thread and pass, their loads issued together
    constexpr int NB = 4;
    const int stride = gridDim.x * blockDim.x;
    for (int id0 = blockIdx.x * blockDim.x + threadIdx.x; id0 < nseg; id0 += NB * stride) {
        int f[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int id = id0 + b * stride;
            f[b] = id < nseg ? ctx.seg_first[id] : -1;
        }
        unsigned k[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) k[b] = (f[b] >= 0 && MPM_INB(f[b], ctx.n, 11)) ? skeys[f[b]] : 0xffffffffu;
#pragma unroll
        for (int b = 0; b < NB; ++b)
            if (f[b] >= 0 && k[b] != 0xffffffffu && MPM_INB(k[b], ctx.n_keys, 2)) ctx.cell_seg[k[b]] = id0 + b * stride + 1;
    }
}

// exclusive scan, in place, of a block's E (round, warp) counts (round-major;
// warp 0, E / 32 per lane, or one per lane for E <= 32); call from all threads
template <int E>
__device__ __forceinline__ void scan_round_warp_counts(unsigned* pre) {
    static_assert(E <= 32 || E % 32 == 0, "E <= 32 or a multiple of 32");
    constexpr int PER = E <= 32 ? 1 : E / 32;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    if ((threadIdx.x >> 5) == 0) {
        unsigned v[PER], tot = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            v[j] = PER * lane + j < E ? pre[PER * lane + j] : 0u;
            tot += v[j];
        }
        unsigned inc = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        unsigned ex = inc - tot;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            if (PER * lane + j < E) pre[PER * lane + j] = ex;
            ex += v[j];
        }
    }
    __syncthreads();
}

// Active-tile list: the flagged tiles, in tile order.  Per-block counts, the
// block scan above, then ranks from warp ballots; the flags are reset for the
// next step.  A block covers TILEK_ITEMS warp-striped rounds of tiles (every
// load coalesced), and all its flag loads are issued before any is used; one
// scan of the (round, warp) counts replaces a barrier pair per round.
#ifndef MPM_TILEK_ITEMS         // tiles per thread (build-time; 4 measured faster than 16)
#define MPM_TILEK_ITEMS 4
#endif
constexpr int TILEK_ITEMS = MPM_TILEK_ITEMS;
constexpr int TILEK_TILE = SEG_THREADS * TILEK_ITEMS;
// Bit r: tile base + r*256 + thread is flagged.
__device__ __forceinline__ unsigned tile_flags(const int* __restrict__ flag, long long n_tiles, long long base) {
    unsigned on = 0;
    int f[TILEK_ITEMS];
#pragma unroll
    for (int r = 0; r < TILEK_ITEMS; ++r) {
        const long long t = base + (long long)r * SEG_THREADS + threadIdx.x;
        f[r] = t < n_tiles ? flag[t] : 0;
    }
#pragma unroll
    for (int r = 0; r < TILEK_ITEMS; ++r) on |= (f[r] != 0 ? 1u : 0u) << r;
    return on;
}

__global__ void __launch_bounds__(SEG_THREADS)
tile_count_kernel(const int* __restrict__ flag, long long n_tiles, unsigned* __restrict__ blk) {
    __shared__ unsigned red[SEG_THREADS / 32];
    unsigned cnt = __popc(tile_flags(flag, n_tiles, (long long)blockIdx.x * TILEK_TILE));
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        for (int w = 0; w < SEG_THREADS / 32; ++w) t += red[w];
        blk[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(SEG_THREADS)
tile_write_kernel(int* __restrict__ flag, long long n_tiles, const unsigned* __restrict__ blk,
                  int* __restrict__ active, int cap) {
    constexpr int NW = SEG_THREADS / 32;
    __shared__ unsigned pre[TILEK_ITEMS * NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const long long base = (long long)blockIdx.x * TILEK_TILE;
    const unsigned on = tile_flags(flag, n_tiles, base);
#pragma unroll
    for (int r = 0; r < TILEK_ITEMS; ++r) {
        const unsigned ball = __ballot_sync(0xffffffffu, (on >> r) & 1u);
        if (lane == 0) pre[r * NW + warp] = __popc(ball);
    }
    scan_round_warp_counts<TILEK_ITEMS * NW>(pre);
    const unsigned run = blk[blockIdx.x];
#pragma unroll
    for (int r = 0; r < TILEK_ITEMS; ++r) {
        const long long t = base + (long long)r * SEG_THREADS + threadIdx.x;
        const bool a = (on >> r) & 1u;
        const unsigned ball = __ballot_sync(0xffffffffu, a);
        if (a) {
            const unsigned before = run + pre[r * NW + warp] + __popc(ball & lt);
            if (before < (unsigned)cap) active[before] = (int)t;
            flag[t] = 0;
        }
    }
}

// Writes seg_first / seg_last / cell_seg.  A slot's segment id is the number of
// segment starts up to and including it: the block's count from the scan, the
// starts of the earlier (round, warp) pairs of the block (one exclusive scan
// of the SEGK_ITEMS x 8 warp counts) and the lanes before it.
__global__ void __launch_bounds__(SEG_THREADS)
seg_write_kernel(Ctx ctx, const unsigned* __restrict__ skeys) {
    constexpr int NW = SEG_THREADS / 32;
    constexpr int E = SEGK_ITEMS * NW;
    __shared__ unsigned pre[SEGK_ITEMS * NW];      // round-major
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const long long base = (long long)blockIdx.x * SEGK_TILE;
    unsigned key[SEGK_ITEMS], start, last;
    seg_flags(ctx, skeys, base, key, start, last);
#pragma unroll
    for (int r = 0; r < SEGK_ITEMS; ++r) {
        const unsigned ball = __ballot_sync(0xffffffffu, (start >> r) & 1u);
        if (lane == 0) pre[r * NW + warp] = __popc(ball);
    }
    scan_round_warp_counts<E>(pre);
    const unsigned run = ctx.blk_count[blockIdx.x];     // segments started before this block
#pragma unroll
    for (int r = 0; r < SEGK_ITEMS; ++r) {
        const long long s = base + (long long)r * SEG_THREADS + threadIdx.x;
        const bool st = (start >> r) & 1u;
        const unsigned ball = __ballot_sync(0xffffffffu, st);
        const unsigned id = run + pre[r * NW + warp] + __popc(ball & lt) + (st ? 1u : 0u);
        if (st && MPM_INB(id - 1, ctx.n, 3)) {
            ctx.seg_first[id - 1] = (int)s;
            if (MPM_INB(key[r], ctx.n_keys, 2)) ctx.cell_seg[key[r]] = (int)id;
        }
        if (((last >> r) & 1u) && id > 0 && MPM_INB(id - 1, ctx.n, 3)) ctx.seg_last[id - 1] = (int)(s + 1);
    }
}

// ---------------------------------------------------------------------------
// forward prepass: stress -> P2G record, stored in particle order
// record: fx[0..2], pmass, a = pmass v, B = (pmass C + dt sk) dx
// ---------------------------------------------------------------------------
template <typename R, int KIND = -1>
__device__ __forceinline__ void p2g_record(const Ctx& ctx, const MpmScene& sc, long long p, const R fx[3],
                                           const R v[3], const R C[9], const R F[9], const R Fg[9],
                                           R rec[PAYLOAD]) {
    ModelParams<R> M;
    M.load(sc);
    if constexpr (KIND >= 0) M.kind = KIND;     // a launch over scenes of one model
    const R dx = (R)sc.dx, dt = (R)sc.dt, inv_dx = (R)(1.0 / sc.dx);
    const R k4 = R(4) * inv_dx * inv_dx;
    R tau[9];
    bool fb = false;
    if (M.kind == MPM_MODEL_EXTERNAL)
        ld9<R>(ctx.ext_tau, p, 9, 1, tau);      // the caller's stress
    else
        fb = model_stress(M, ctx.gap_thresh, F, Fg, C, tau);
    if (fb) atomicAdd(ctx.fallbacks, 1ull);
    R pm, vol0;
    particle_mass<R>(ctx, sc, p, pm, vol0);
    R c = -k4 * vol0 * det3(Fg);
    rec[0] = fx[0]; rec[1] = fx[1]; rec[2] = fx[2]; rec[3] = pm;
#pragma unroll
    for (int i = 0; i < 3; ++i) rec[4 + i] = pm * v[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) rec[7 + i] = (pm * C[i] + dt * (c * tau[i])) * dx;
    if (!finite9(tau)) raise_status(ctx.status, MPM_ERR_NONFINITE);
}

template <typename R>
__global__ void __launch_bounds__(256, 3)
prepass_kernel(Ctx ctx, MpmParticles P, R* __restrict__ payload, int t) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ctx.n) return;
    const MpmScene& sc = ctx.scenes[ctx.scene_of[p]];
    R x[3], v[3], C[9], F[9], Fg[9];
    ld3<R>(P.x, p, P.sp3, P.sc3, x);
    ld3<R>(P.v, p, P.sp3, P.sc3, v);
    ld9<R>(P.C, p, P.sp9, P.sc9, C);
    ld9<R>(P.F, p, P.sp9, P.sc9, F);
    load_Fg<R>(ctx, sc, P, p, t, Fg, nullptr);
    int base[3];
    R fx[3];
    bin_particle(x, (R)(1.0 / sc.dx), sc.shape, base, fx);
    R rec[PAYLOAD];
    p2g_record<R>(ctx, sc, p, fx, v, C, F, Fg, rec);
    store_record(payload, p, rec);
}

// ---------------------------------------------------------------------------
// P2G, phase 1: per-cell sums.  One thread per segment (occupied cell) adds
// its particles' contributions to the 27 stencil nodes, in sorted order, in
// registers, and stores them as sums[o][segment] (o = 9 ox + 3 oy + oz).
// MODE 0: channels (m, mom[3]);  MODE 1: channels (gv_b[3], unused).
// OXB: stencil x-offsets accumulated per pass over the cell's particles.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void store_sum(R* __restrict__ S, long long idx, const R v[4]) {
    if constexpr (sizeof(R) == 4) {
        reinterpret_cast<float4*>(S)[idx] = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        double2* p = reinterpret_cast<double2*>(S) + 2 * idx;
        p[0] = make_double2(v[0], v[1]);
        p[1] = make_double2(v[2], v[3]);
    }
}

// Adds one particle record's contributions to the stencil sums of the x-offsets
// ox0 .. ox0+OXB-1: w(o) (a + B dp(o)) (and w(o) m in channel 0 for MODE 0),
// dp = o - fx in cell units (B carries the dx factor).
template <typename R, int MODE, int OXB>
__device__ __forceinline__ void accumulate_record(const R r[PAYLOAD], int ox0, R acc[OXB][3][3][4]) {
    R w[3][3];
    bspline(r, w);
    R dz[3] = {R(0) - r[2], R(1) - r[2], R(2) - r[2]};
    R dy[3] = {R(0) - r[1], R(1) - r[1], R(2) - r[1]};
#pragma unroll
    for (int a = 0; a < OXB; ++a) {
        const int ox = ox0 + a;
        const R dpx = R(ox) - r[0];
        R wx;
        if constexpr (OXB == 3) wx = w[a][0];
        else wx = ox == 0 ? w[0][0] : (ox == 1 ? w[1][0] : w[2][0]);
        // a + B dp with dp = (dpx, dy, dz), x part hoisted
        const R ax0 = r[4] + r[7] * dpx, ax1 = r[5] + r[10] * dpx, ax2 = r[6] + r[13] * dpx;
#pragma unroll
        for (int oy = 0; oy < 3; ++oy) {
            const R wxy = wx * w[oy][1];
            const R ay0 = ax0 + r[8] * dy[oy], ay1 = ax1 + r[11] * dy[oy], ay2 = ax2 + r[14] * dy[oy];
#pragma unroll
            for (int oz = 0; oz < 3; ++oz) {
                const R wt = wxy * w[oz][2];
                const R q0 = ay0 + r[9] * dz[oz];
                const R q1 = ay1 + r[12] * dz[oz];
                const R q2 = ay2 + r[15] * dz[oz];
                if constexpr (MODE == 0) {
                    acc[a][oy][oz][0] += wt * r[3];
                    acc[a][oy][oz][1] += wt * q0;
                    acc[a][oy][oz][2] += wt * q1;
                    acc[a][oy][oz][3] += wt * q2;
                } else {
                    acc[a][oy][oz][0] += wt * q0;
                    acc[a][oy][oz][1] += wt * q1;
                    acc[a][oy][oz][2] += wt * q2;
                }
            }
        }
    }
}

template <typename R, int OXB>
__device__ __forceinline__ void zero_acc(R acc[OXB][3][3][4]) {
#pragma unroll
    for (int a = 0; a < OXB; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int h = 0; h < 4; ++h) acc[a][b][c][h] = R(0);
}

template <typename R, int OXB>
__device__ __forceinline__ void store_acc(R* __restrict__ S, long long cap, int id, int ox0,
                                          R acc[OXB][3][3][4]) {
#pragma unroll
    for (int a = 0; a < OXB; ++a)
#pragma unroll
        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
            for (int oz = 0; oz < 3; ++oz) {
                const int o = 9 * (ox0 + a) + 3 * oy + oz;
                if (MPM_INB((long long)o * cap + id, 27 * cap, 4)) store_sum(S, (long long)o * cap + id, acc[a][oy][oz]);
            }
}

// OXB: stencil x-offsets accumulated per pass over a cell's particles (3 or 1).
template <typename R, int MODE, int OXB>
__global__ void __launch_bounds__(128)
cell_sums_kernel(Ctx ctx, const unsigned* __restrict__ perm, const R* __restrict__ payload, R* __restrict__ S,
                 long long cap) {
    const int nseg = *ctx.n_seg;
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < nseg; id += gridDim.x * blockDim.x) {
        const int first = ctx.seg_first[id], last = ctx.seg_last[id];
        if (!(MPM_INB(first, ctx.n + 1, 11) && MPM_INB(last, ctx.n + 1, 11))) continue;
#pragma unroll 1
        for (int ox0 = 0; ox0 < 3; ox0 += OXB) {
            R acc[OXB][3][3][4];
            zero_acc<R, OXB>(acc);
            for (int q = first; q < last; ++q) {
                R r[PAYLOAD];
                if (!MPM_INB(perm[q], ctx.n, 9)) continue;
                load_record(payload, perm[q], r);
                accumulate_record<R, MODE, OXB>(r, ox0, acc);
            }
            store_acc<R, OXB>(S, cap, id, ox0, acc);
        }
    }
}

// ---------------------------------------------------------------------------
// Reverse P2G, phase 1 (transfer.py:99-119 scatter of gv_b): per occupied cell
// the 27 stencil sums of w (nv_b + k4 Cn_b' dp), with nv_b = vn_b + dt xn_b
// (advect) and Cn_b' = Cn_b + dt Fn_b F^T formed here from the cotangents of
// the step's output, so no payload record is written for the reverse.
// ---------------------------------------------------------------------------
// the x-offsets ox_lo .. ox_lo + 3 - 1 of one occupied cell (OXB at a time)
template <typename R, int OXB>
__device__ __forceinline__ void adj_cell(const Ctx& ctx, const unsigned* __restrict__ perm, const MpmParticles& in,
                                         const MpmCotangents& ob, R* __restrict__ S, long long cap, int advect,
                                         int id, int ox_lo, int ox_hi) {
    const int first = ctx.seg_first[id], last = ctx.seg_last[id];
    if (!(MPM_INB(first, ctx.n, 11) && MPM_INB(last, ctx.n + 1, 11))) return;
    const MpmScene& sc = ctx.scenes[ctx.scene_of[first]];
    const R dx = (R)sc.dx, dt = (R)sc.dt, inv_dx = (R)(1.0 / sc.dx);
    const R kdx = R(4) * inv_dx * inv_dx * dx;
#pragma unroll 1
    for (int ox0 = ox_lo; ox0 < ox_hi; ox0 += OXB) {
        R acc[OXB][3][3][3];
#pragma unroll
        for (int a = 0; a < OXB; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int h = 0; h < 3; ++h) acc[a][b][c][h] = R(0);
        for (int q = first; q < last; ++q) {
            const long long p = perm[q];
            if (!MPM_INB(p, ctx.n, 9)) continue;
            R x[3], nv[3], B[9];
            ld3<R>(in.x, p, in.sp3, in.sc3, x);
            {
                R F[9], Fb[9], Cb[9], xb[3];
                ld9<R>(in.F, p, in.sp9, in.sc9, F);
                ld9<R>(ob.F, p, ob.sp9, ob.sc9, Fb);
                ld9<R>(ob.C, p, ob.sp9, ob.sc9, Cb);
                ld3<R>(ob.v, p, ob.sp3, ob.sc3, nv);
                if (advect) {
                    ld3<R>(ob.x, p, ob.sp3, ob.sc3, xb);
#pragma unroll
                    for (int i = 0; i < 3; ++i) nv[i] += dt * xb[i];
                }
                R FbFt[9];
                mmT(Fb, F, FbFt);
#pragma unroll
                for (int i = 0; i < 9; ++i) B[i] = kdx * (Cb[i] + dt * FbFt[i]);
            }
            int base[3];
            R fx[3];
            bin_particle(x, inv_dx, sc.shape, base, fx);
            R w[3][3];
            bspline(fx, w);
            const R dz[3] = {R(0) - fx[2], R(1) - fx[2], R(2) - fx[2]};
            const R dy[3] = {R(0) - fx[1], R(1) - fx[1], R(2) - fx[1]};
#pragma unroll
            for (int a = 0; a < OXB; ++a) {
                const int ox = ox0 + a;
                const R dpx = R(ox) - fx[0];
                R wx;
                if constexpr (OXB == 3) wx = w[a][0];
                else wx = ox == 0 ? w[0][0] : (ox == 1 ? w[1][0] : w[2][0]);
                const R ax0 = nv[0] + B[0] * dpx, ax1 = nv[1] + B[3] * dpx, ax2 = nv[2] + B[6] * dpx;
#pragma unroll
                for (int oy = 0; oy < 3; ++oy) {
                    const R wxy = wx * w[oy][1];
                    const R ay0 = ax0 + B[1] * dy[oy], ay1 = ax1 + B[4] * dy[oy], ay2 = ax2 + B[7] * dy[oy];
#pragma unroll
                    for (int oz = 0; oz < 3; ++oz) {
                        const R wt = wxy * w[oz][2];
                        acc[a][oy][oz][0] += wt * (ay0 + B[2] * dz[oz]);
                        acc[a][oy][oz][1] += wt * (ay1 + B[5] * dz[oz]);
                        acc[a][oy][oz][2] += wt * (ay2 + B[8] * dz[oz]);
                    }
                }
            }
        }
#pragma unroll
        for (int a = 0; a < OXB; ++a)
#pragma unroll
            for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                for (int oz = 0; oz < 3; ++oz) {
                    const int o = 9 * (ox0 + a) + 3 * oy + oz;
                    const R v4[4] = {acc[a][oy][oz][0], acc[a][oy][oz][1], acc[a][oy][oz][2], R(0)};
                    if (MPM_INB((long long)o * cap + id, 27 * cap, 4)) store_sum(S, (long long)o * cap + id, v4);
                }
    }
}

// OXB: stencil x-offsets per pass over a cell's particles (3 or 1).
template <typename R, int OXB>
__global__ void __launch_bounds__(128, 4)
cell_sums_adj_kernel(Ctx ctx, const unsigned* __restrict__ perm, MpmParticles in, MpmCotangents ob,
                     R* __restrict__ S, long long cap, int advect) {
    const int nseg = *ctx.n_seg;
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < nseg; id += gridDim.x * blockDim.x)
        adj_cell<R, OXB>(ctx, perm, in, ob, S, cap, advect, id, 0, 3);
}

// ---------------------------------------------------------------------------
// P2G, phase 2: node gather + grid update.  One thread per node of the
// active node tiles (persistent grid over the active list); every node adds
// the sums of its 27 source cells in the fixed order o = 0..26, then
// MODE 0: grid update -> (m, v[3]) with v = s mom/m + s dt g on free nodes;
// MODE 1: grid adjoint -> (gm_b, gmom_b[3]) from gv_b and the forward record.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void load_sum(const R* __restrict__ S, long long idx, R o[4]) {
    if constexpr (sizeof(R) == 4) {
        float4 v = __ldg(reinterpret_cast<const float4*>(S) + idx);
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    } else {
        const double2* p = reinterpret_cast<const double2*>(S) + 2 * idx;
        double2 a = __ldg(p), b = __ldg(p + 1);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
}

// Grid adjoint of one node (the reverse node gather's epilogue): gmom_b and
// gm_b from the gathered gv_b sums acc and the forward record, which is also
// restored into the dense scratch for the reverse particle kernel.
template <typename R>
__device__ __forceinline__ void node_adjoint(const Ctx& ctx, const MpmScene& sc, const SceneAux& ax, int i, int j,
                                             int k, long long gidx, const R acc[4], const R* __restrict__ grid_fwd,
                                             int advect) {
    const R s_damp = (R)(1.0 - sc.damping);
    const R dt = (R)sc.dt;
    const R eps = (R)sc.mass_eps;
    const R g0 = (R)sc.gravity[0], g1 = (R)sc.gravity[1], g2 = (R)sc.gravity[2];
    const long long didx = ax.node_begin + ((long long)i * sc.shape[1] + j) * sc.shape[2] + k;
    if (!(MPM_INB(didx, ctx.n_nodes, 7) && MPM_INB(gidx, ctx.grid_nodes, 8))) return;
    R rec[4] = {R(0), R(0), R(0), R(0)};
    R f[4];
    load_node(grid_fwd, gidx, f);
    store_node(static_cast<R*>(ctx.dense_f), didx, f);
    const R m = f[0];
    if (m > eps && node_free(sc, i, j, k)) {
        rec[1] = (s_damp * acc[0]) / m;
        rec[2] = (s_damp * acc[1]) / m;
        rec[3] = (s_damp * acc[2]) / m;
        if (advect) {
            const R sd = s_damp * dt;
            rec[0] = -(acc[0] * (f[1] - sd * g0) + acc[1] * (f[2] - sd * g1) + acc[2] * (f[3] - sd * g2)) / m;
        }
    }
    store_node(static_cast<R*>(ctx.dense_b), didx, rec);
}

// tile t of a scene -> its first node (L0, L1, L2)
__device__ __forceinline__ void tile_origin(const SceneAux& ax, long long lt, int T, int TZ, int L[3]) {
    const int tz = (int)(lt % ax.ntile[2]);
    const int ty = (int)((lt / ax.ntile[2]) % ax.ntile[1]);
    const int tx = (int)(lt / ((long long)ax.ntile[2] * ax.ntile[1]));
    L[0] = tx * T;
    L[1] = ty * T;
    L[2] = tz * TZ;
}

template <typename R, int T, int TZ, int MODE>
__global__ void __launch_bounds__(1024)
node_sums_kernel(Ctx ctx, const R* __restrict__ S, long long cap, const int* __restrict__ active,
                 const int* __restrict__ n_active, R* __restrict__ grid_out, const R* __restrict__ grid_fwd,
                 int advect) {
    // Both modes walk the nodes in CTA-uniform rounds of blockDim nodes (the
    // per-thread grid-stride form measured slower: forward 62.3 vs 65.8 ms,
    // reverse 80.8 vs 86.7 ms per config-4 trajectory); the forward keeps its
    // epilogue inline and the reverse calls node_adjoint, each the faster of
    // the two measured for its mode.  The sums and their order are the same.
    if constexpr (MODE == 0) {
        constexpr int TN = T * T * TZ;
        // one thread per node of the active tiles (tile-major, z fastest), grid-strided
        const long long total = (long long)(*n_active) * TN;
        for (long long r0 = (long long)blockIdx.x * blockDim.x; r0 < total; r0 += (long long)gridDim.x * blockDim.x) {
            const long long gidx = r0 + threadIdx.x;
            if (gidx >= total) continue;
            const int it = (int)(gidx / TN), node = (int)(gidx % TN);
            const int tile = active[it];
            const int s = ctx.tile_scene[tile];
            const MpmScene& sc = ctx.scenes[s];
            const SceneAux& ax = ctx.aux[s];
            long long lt = tile - ax.tile_begin;
            const int tz = (int)(lt % ax.ntile[2]);
            const int ty = (int)((lt / ax.ntile[2]) % ax.ntile[1]);
            const int tx = (int)(lt / ((long long)ax.ntile[2] * ax.ntile[1]));
            const int L0 = tx * T, L1 = ty * T, L2 = tz * TZ;
            const long long P1 = sc.shape[1] + 2, P2 = sc.shape[2] + 2;
            const R s_damp = (R)(1.0 - sc.damping);
            const R dt = (R)sc.dt;
            const R eps = (R)sc.mass_eps;
            const R g0 = (R)sc.gravity[0], g1 = (R)sc.gravity[1], g2 = (R)sc.gravity[2];
            {
                const int nz = node % TZ, ny = (node / TZ) % T, nx = node / (TZ * T);
                const int i = L0 + nx, j = L1 + ny, k = L2 + nz;
                if (i >= sc.shape[0] || j >= sc.shape[1] || k >= sc.shape[2]) continue;
                R acc[4] = {R(0), R(0), R(0), R(0)};
                const long long cbase = ax.cell_begin + ((long long)(i + 2) * P1 + (j + 2)) * P2 + (k + 2);
    #pragma unroll
                for (int ox = 0; ox < 3; ++ox)
    #pragma unroll
                    for (int oy = 0; oy < 3; ++oy)
    #pragma unroll
                        for (int oz = 0; oz < 3; ++oz) {
                            const long long ci = cbase - ((long long)ox * P1 + oy) * P2 - oz;
                            const int id1 = MPM_INB(ci, ctx.n_keys, 6) ? ctx.cell_seg[ci] : 0;
                            const long long si = (long long)(9 * ox + 3 * oy + oz) * cap + (id1 - 1);
                            if (id1 && MPM_INB(si, 27 * cap, 5)) {
                                R v[4];
                                load_sum(S, si, v);
                                acc[0] += v[0]; acc[1] += v[1]; acc[2] += v[2]; acc[3] += v[3];
                            }
                        }
                const long long didx = ax.node_begin + ((long long)i * sc.shape[1] + j) * sc.shape[2] + k;
                if (!(MPM_INB(didx, ctx.n_nodes, 7) && MPM_INB(gidx, ctx.grid_nodes, 8))) continue;
                R rec[4] = {R(0), R(0), R(0), R(0)};
                if constexpr (MODE == 0) {
                    const R m = acc[0];
                    rec[0] = m;
                    if (m > eps && node_free(sc, i, j, k)) {
                        rec[1] = (s_damp * acc[1]) / m + s_damp * dt * g0;
                        rec[2] = (s_damp * acc[2]) / m + s_damp * dt * g1;
                        rec[3] = (s_damp * acc[3]) / m + s_damp * dt * g2;
                    }
                } else {
                    R f[4];
                    load_node(grid_fwd, gidx, f);
                    store_node(static_cast<R*>(ctx.dense_f), didx, f);
                    const R m = f[0];
                    if (m > eps && node_free(sc, i, j, k)) {
                        rec[1] = (s_damp * acc[0]) / m;
                        rec[2] = (s_damp * acc[1]) / m;
                        rec[3] = (s_damp * acc[2]) / m;
                        if (advect) {
                            const R sd = s_damp * dt;
                            rec[0] = -(acc[0] * (f[1] - sd * g0) + acc[1] * (f[2] - sd * g1) + acc[2] * (f[3] - sd * g2)) / m;
                        }
                    }
                }
                if constexpr (MODE == 0) {
                    store_node(grid_out, gidx, rec);
                    store_node(static_cast<R*>(ctx.dense_f), didx, rec);
                } else {
                    store_node(static_cast<R*>(ctx.dense_b), didx, rec);
                }
            }
        }
    } else {
        constexpr int TN = T * T * TZ;
        // one thread per node of the active tiles (tile-major, z fastest), grid-strided
        const int nact = *n_active;
        const long long total = (long long)nact * TN;
        const long long stride = (long long)gridDim.x * blockDim.x;
        // (a CTA-uniform loop over rounds of blockDim nodes: 80.8 ms per config-4
        // trajectory against 86.7 for the per-thread grid-stride form)
        for (long long r0 = (long long)blockIdx.x * blockDim.x; r0 < total; r0 += stride) {
            const long long gidx = r0 + threadIdx.x;
            if (gidx >= total) continue;
            const int it = (int)(gidx / TN), node = (int)(gidx % TN);
            const int tile = active[it];
            const int s = ctx.tile_scene[tile];
            const MpmScene& sc = ctx.scenes[s];
            const SceneAux& ax = ctx.aux[s];
            int L[3];
            tile_origin(ax, tile - ax.tile_begin, T, TZ, L);
            const long long P1 = sc.shape[1] + 2, P2 = sc.shape[2] + 2;
            const int nz = node % TZ, ny = (node / TZ) % T, nx = node / (TZ * T);
            const int i = L[0] + nx, j = L[1] + ny, k = L[2] + nz;
            if (i >= sc.shape[0] || j >= sc.shape[1] || k >= sc.shape[2]) continue;
            R acc[4] = {R(0), R(0), R(0), R(0)};
            const long long cbase = ax.cell_begin + ((long long)(i + 2) * P1 + (j + 2)) * P2 + (k + 2);
#pragma unroll
            for (int ox = 0; ox < 3; ++ox)
#pragma unroll
                for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                    for (int oz = 0; oz < 3; ++oz) {
                        const long long ci = cbase - ((long long)ox * P1 + oy) * P2 - oz;
                        const int id1 = MPM_INB(ci, ctx.n_keys, 6) ? ctx.cell_seg[ci] : 0;
                        const long long si = (long long)(9 * ox + 3 * oy + oz) * cap + (id1 - 1);
                        if (id1 && MPM_INB(si, 27 * cap, 5)) {
                            R v[4];
                            load_sum(S, si, v);
                            acc[0] += v[0]; acc[1] += v[1]; acc[2] += v[2]; acc[3] += v[3];
                        }
                    }
            node_adjoint<R>(ctx, sc, ax, i, j, k, gidx, acc, grid_fwd, advect);
        }
    }
}

// ---------------------------------------------------------------------------
// stencil addressing into the dense node scratch: node (i,j,k) of a scene is
// node_begin + (i ny + j) nz + k; per particle the three axis offsets are
// formed once and a node costs two adds.
// ---------------------------------------------------------------------------
struct DenseStencil {
    long long ox[3], oy[3];
    int oz[3];
    bool vx[3], vy[3], vz[3];
    __device__ __forceinline__ void init(const MpmScene& sc, const SceneAux& ax, const int base[3]) {
        const long long ny = sc.shape[1], nz = sc.shape[2];
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            const int i = base[0] + o, j = base[1] + o, k = base[2] + o;
            vx[o] = i >= 0 && i < sc.shape[0];
            vy[o] = j >= 0 && j < sc.shape[1];
            vz[o] = k >= 0 && k < sc.shape[2];
            ox[o] = ax.node_begin + (long long)i * ny * nz;
            oy[o] = (long long)j * nz;
            oz[o] = k;
        }
    }
};

__device__ __forceinline__ void unmark_cell(const Ctx& ctx, const SceneAux& ax, const unsigned* __restrict__ skeys,
                                            long long sidx) {
    unsigned k = skeys[sidx];
    if ((sidx == 0 || skeys[sidx - 1] != k) && (long long)k - ax.cell_begin < ax.ncells && MPM_INB(k, ctx.n_keys, 2))
        ctx.cell_seg[k] = 0;
}

// ---------------------------------------------------------------------------
// G2P + advection + F update (transfer.py:61-79); writes the output state in
// the input's particle order and clears the cell marks of this step.
// ---------------------------------------------------------------------------
// Sorted slots [s_begin, s_end).  KIND >= 0: every scene of these slots uses
// material model KIND, so the kernel carries that model's code only.
template <typename R, bool EMIT, int KIND>
__global__ void __launch_bounds__(256, EMIT ? (sizeof(R) == 4 ? 3 : 1) : (sizeof(R) == 4 ? 4 : 2))
g2p_kernel(Ctx ctx, Tape<R> tp, MpmParticles in, MpmParticles out, int advect, unsigned* __restrict__ keys,
           R* __restrict__ payload, int t, long long s_begin, long long s_end) {
    long long sidx = s_begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= s_end) return;
    long long p = tp.perm[sidx];
    if (!MPM_INB(p, ctx.n, 9)) return;
    const int s = ctx.scene_of[sidx];
    const MpmScene& sc = ctx.scenes[s];
    const SceneAux& ax = ctx.aux[s];
    const R dx = (R)sc.dx, dt = (R)sc.dt, inv_dx = (R)(1.0 / sc.dx);
    const R k4 = R(4) * inv_dx * inv_dx;
    R x[3];
    ld3<R>(in.x, p, in.sp3, in.sc3, x);
    int base[3];
    R fx[3];
    bin_particle(x, inv_dx, sc.shape, base, fx);
    R w[3][3];
    bspline(fx, w);
    DenseStencil st;
    st.init(sc, ax, base);
    const R* __restrict__ dense = static_cast<const R*>(ctx.dense_f);
    // nC = k4 sum w g (o - fx)^T dx = k4 dx (G - nv fx^T),  G[i][d] = sum w g_i o_d
    R nv[3] = {0, 0, 0}, G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!st.vx[a]) continue;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            if (!st.vy[b]) continue;
            const long long rab = st.ox[a] + st.oy[b];
            // column sums over z: sum w_c g and sum c w_c g
            R Zg[3] = {0, 0, 0}, Zc[3] = {0, 0, 0};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (!st.vz[c]) continue;
                R g[4];
                if (!MPM_INB(rab + st.oz[c], ctx.n_nodes, 7)) continue;
                load_node(dense, rab + st.oz[c], g);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    Zg[i] += w[c][2] * g[1 + i];
                    if (c) Zc[i] += (R(c) * w[c][2]) * g[1 + i];
                }
            }
            const R wab = w[a][0] * w[b][1];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                nv[i] += wab * Zg[i];
                if (a) G[3 * i + 0] += (R(a) * wab) * Zg[i];
                if (b) G[3 * i + 1] += (R(b) * wab) * Zg[i];
                G[3 * i + 2] += wab * Zc[i];
            }
        }
    }
    R nC[9];
    const R kd = k4 * dx;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) nC[3 * i + d] = kd * (G[3 * i + d] - nv[i] * fx[d]);
    R F[9];
    ld9<R>(in.F, p, in.sp9, in.sc9, F);
    R xn[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) xn[i] = advect ? x[i] + dt * nv[i] : x[i];
    R A[9], Fn[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) A[i] = ((i % 4 == 0) ? R(1) : R(0)) + dt * nC[i];
    mm(A, F, Fn);
    st3<R>(out.x, p, out.sp3, out.sc3, xn);
    st3<R>(out.v, p, out.sp3, out.sc3, nv);
    st9<R>(out.C, p, out.sp9, out.sc9, nC);
    st9<R>(out.F, p, out.sp9, out.sc9, Fn);
    if (sc.growth_mode == 0 && out.Fg != nullptr && out.Fg != in.Fg) {
        R Fg[9];
        ld9<R>(in.Fg, p, in.sp9, in.sc9, Fg);
        st9<R>(out.Fg, p, out.sp9, out.sc9, Fg);
    }
    if (!finite9(Fn) || !(xn[0] * R(0) == R(0) && xn[1] * R(0) == R(0) && xn[2] * R(0) == R(0)))
        raise_status(ctx.status, MPM_ERR_NONFINITE);
    unmark_cell(ctx, ax, tp.skeys, sidx);
    if constexpr (EMIT) {
        // the next step's binning and P2G record of the new state (what the
        // bin and prepass kernels of step t+1 would compute from memory)
        R fxn[3], Fg[9], rec[PAYLOAD];
        const unsigned kn = particle_key<R>(ctx, sc, ax, xn, fxn);
        keys[p] = kn;
        // movers of this step's sorted order (the next step's incremental re-sort)
        if (ctx.mover_flag) {
            const unsigned char moved = kn != tp.skeys[sidx] ? 1 : 0;
            ctx.mover_flag[sidx] = moved;
            ctx.mover_pflag[p] = moved;
        }
        load_Fg<R>(ctx, sc, in, p, t + 1, Fg, nullptr);
        p2g_record<R, KIND>(ctx, sc, p, fxn, nv, nC, Fn, Fg, rec);
        store_record(payload, p, rec);
    }
}

// ---------------------------------------------------------------------------
// reverse: per-particle cotangents (transfer.py:99-119 x_b terms, 129-156).
// The x_b terms of the reference are regrouped per node as
//   x_b += [nv_b.gv + pm mb.v + pm gm_b + (M1 gv + M2 mb).dp] dW
// with M1 = k4 Cn_b'^T, M2 = pm C^T + dt sk^T, and the weight-only terms are
// summed once per particle: x_b -= M1 sum(w gv) + M2 sum(w mb).
// ---------------------------------------------------------------------------
// MAT: also the material-parameter gradients per slot, dmat[sidx] (mu) and
// dmat[n + sidx] (lambda).  EXT: the plan has MPM_MODEL_EXTERNAL scenes.
// Sorted slots [s_begin, s_end); KIND as in g2p_kernel.
template <typename R, bool MAT, bool EXT, int KIND>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 2 : 1)
bwd_particle_kernel(Ctx ctx, Tape<R> tp, MpmParticles in, const R* __restrict__ outC,
                    MpmCotangents ob, MpmCotangents ib, double* __restrict__ dA, double* __restrict__ dmat,
                    int advect, int t, long long s_begin, long long s_end) {
    long long sidx = s_begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= s_end) return;
    long long p = tp.perm[sidx];
    if (!MPM_INB(p, ctx.n, 9)) return;
    const int s = ctx.scene_of[sidx];
    const MpmScene& sc = ctx.scenes[s];
    const SceneAux& ax = ctx.aux[s];
    ModelParams<R> M;
    M.load(sc);
    if constexpr (KIND >= 0) M.kind = KIND;
    const R dx = (R)sc.dx, dt = (R)sc.dt, inv_dx = (R)(1.0 / sc.dx);
    const R k4 = R(4) * inv_dx * inv_dx;
    R pm, vol0;
    particle_mass<R>(ctx, sc, p, pm, vol0);
    R x[3], C[9], F[9], Fg[9];
    R gphi;
    ld3<R>(in.x, p, in.sp3, in.sc3, x);
    ld9<R>(in.C, p, in.sp9, in.sc9, C);
    ld9<R>(in.F, p, in.sp9, in.sc9, F);
    load_Fg<R>(ctx, sc, in, p, t, Fg, &gphi);

    R tau[9], keep[13];
    bool fb = false;
    if (EXT && M.kind == MPM_MODEL_EXTERNAL)
        ld9<R>(ctx.ext_tau, p, 9, 1, tau);      // the caller's stress
    else
        fb = model_stress_keep(M, ctx.gap_thresh, F, Fg, C, tau, keep);
    // the kept eigendecomposition waits in shared memory (one column per
    // thread) while the node loop holds the registers
    __shared__ R keep_s[13][256];
#pragma unroll
    for (int i = 0; i < 13; ++i) keep_s[i][threadIdx.x] = keep[i];
    const R c = -k4 * vol0 * det3(Fg);

    // per-particle matrices of the regrouped x_b terms
    R M1[9], M2[9], nvb[3], pv[3];
    {
        R xnb[3], vnb[3], Cnb[9], Fnb[9], v[3];
        ld3<R>(ob.x, p, ob.sp3, ob.sc3, xnb);
        ld3<R>(ob.v, p, ob.sp3, ob.sc3, vnb);
        ld9<R>(ob.C, p, ob.sp9, ob.sc9, Cnb);
        ld9<R>(ob.F, p, ob.sp9, ob.sc9, Fnb);
        ld3<R>(in.v, p, in.sp3, in.sc3, v);
        R FbFt[9];
        mmT(Fnb, F, FbFt);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            nvb[i] = advect ? vnb[i] + dt * xnb[i] : vnb[i];
            pv[i] = pm * v[i];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                M1[3 * i + j] = k4 * (Cnb[3 * j + i] + dt * FbFt[3 * j + i]);       // k4 Cn_b'^T
                M2[3 * i + j] = pm * C[3 * j + i] + dt * (c * tau[3 * j + i]);       // pm C^T + dt sk^T
            }
        }
    }
    int base[3];
    R fx[3];
    bin_particle(x, inv_dx, sc.shape, base, fx);
    R w[3][3], dw[3][3];
    bspline(fx, w);
    bspline_grad(fx, dw);
    DenseStencil st;
    st.init(sc, ax, base);

    // The node loop is evaluated as separable sums: per stencil column (a,b)
    // the z-weighted sums of gv, mb and c*mb, and of the advect factor
    //   sfac(o) = gv.U(o) + mb.V(o) + pm gm_b,  U(o) = nv_b + M1^T dp, V(o) = pm v + M2^T dp
    // (dp = (o - fx) dx, so U and V are affine in o: U = U0 + dx (a M1_0 + b M1_1 + c M1_2)
    // with M1_i the rows of M1), then the column sums are weighted by w_a w_b.
    // Sb = sum w mb (o - fx)^T dx = dx (GB - wmb fx^T),  GB[i][d] = sum w mb_i o_d
    R D1[9], D2[9], U0[3], V0[3];
#pragma unroll
    for (int q = 0; q < 9; ++q) { D1[q] = dx * M1[q]; D2[q] = dx * M2[q]; }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        U0[j] = nvb[j] - (D1[j] * fx[0] + D1[3 + j] * fx[1] + D1[6 + j] * fx[2]);
        V0[j] = pv[j] - (D2[j] * fx[0] + D2[3 + j] * fx[1] + D2[6 + j] * fx[2]);
    }
    const R* __restrict__ dfw = static_cast<const R*>(ctx.dense_f);
    const R* __restrict__ dbw = static_cast<const R*>(ctx.dense_b);
    R xs[3] = {0, 0, 0}, wgv[3] = {0, 0, 0}, wmb[3] = {0, 0, 0}, GB[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) GB[q] = R(0);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!st.vx[a]) continue;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            if (!st.vy[b]) continue;
            const long long rab = st.ox[a] + st.oy[b];
            R Zg[3] = {0, 0, 0}, Zm[3] = {0, 0, 0}, Zc[3] = {0, 0, 0}, Sab = 0, Tab = 0;
            R Uab[3], Vab[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                Uab[j] = U0[j] + R(a) * D1[j] + R(b) * D1[3 + j];
                Vab[j] = V0[j] + R(a) * D2[j] + R(b) * D2[3 + j];
            }
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                if (!st.vz[cc]) continue;
                R gf[4], gb[4];
                if (!MPM_INB(rab + st.oz[cc], ctx.n_nodes, 7)) continue;
                load_node(dfw, rab + st.oz[cc], gf);
                load_node(dbw, rab + st.oz[cc], gb);
                const R* gv = gf + 1;
                const R* mb = gb + 1;
                const R wz = w[cc][2];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    Zg[i] += wz * gv[i];
                    Zm[i] += wz * mb[i];
                    if (cc) Zc[i] += (R(cc) * wz) * mb[i];
                }
                if (advect) {
                    R sfac = gb[0] * pm;
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        sfac += gv[j] * (Uab[j] + R(cc) * D1[6 + j]) + mb[j] * (Vab[j] + R(cc) * D2[6 + j]);
                    Sab += wz * sfac;
                    Tab += dw[cc][2] * sfac;
                }
            }
            const R wab = w[a][0] * w[b][1];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                wgv[i] += wab * Zg[i];
                wmb[i] += wab * Zm[i];
                if (a) GB[3 * i + 0] += (R(a) * wab) * Zm[i];
                if (b) GB[3 * i + 1] += (R(b) * wab) * Zm[i];
                GB[3 * i + 2] += wab * Zc[i];
            }
            if (advect) {
                xs[0] += (dw[a][0] * w[b][1]) * Sab;
                xs[1] += (w[a][0] * dw[b][1]) * Sab;
                xs[2] += wab * Tab;
            }
        }
    }
    R xb[3] = {xs[0] * inv_dx, xs[1] * inv_dx, xs[2] * inv_dx};
    R Sb[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) Sb[3 * i + d] = dx * (GB[3 * i + d] - wmb[i] * fx[d]);
    // the constitutive VJP needs F, C, Fg again: reload rather than keep them live
    ld9<R>(in.C, p, in.sp9, in.sc9, C);
    ld9<R>(in.F, p, in.sp9, in.sc9, F);
    load_Fg<R>(ctx, sc, in, p, t, Fg, &gphi);
    R Fb[9], vb[3], Cb[9], skb[9], taub[9];
    {
        R Cn[9], Fnb[9];
        ld9<R>(outC, p, in.sp9, in.sc9, Cn);
        ld9<R>(ob.F, p, ob.sp9, ob.sc9, Fnb);
        R A[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) A[i] = ((i % 4 == 0) ? R(1) : R(0)) + dt * Cn[i];
        mTm(A, Fnb, Fb);   // (I + dt Cn)^T Fn_b
    }
    if (advect) {
        R xnb[3];
        ld3<R>(ob.x, p, ob.sp3, ob.sc3, xnb);
#pragma unroll
        for (int i = 0; i < 3; ++i)
            xb[i] += xnb[i] - inv_dx * (D1[3 * i] * wgv[0] + D1[3 * i + 1] * wgv[1] + D1[3 * i + 2] * wgv[2]
                                      + D2[3 * i] * wmb[0] + D2[3 * i + 1] * wmb[1] + D2[3 * i + 2] * wmb[2]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) vb[i] = pm * wmb[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        Cb[i] = pm * Sb[i];
        skb[i] = dt * Sb[i];
        taub[i] = c * skb[i];
    }
    R Fb2[9], Fgb[9], Cb2[9];
    {
        // volatile: reload here rather than keep the values live in registers
        volatile R* ks = &keep_s[0][threadIdx.x];
#pragma unroll
        for (int i = 0; i < 13; ++i) keep[i] = ks[i * 256];
    }
    if (EXT && M.kind == MPM_MODEL_EXTERNAL) {
        // the caller applies its own stress VJP to tau_bar
        st9<R>(ctx.ext_tau_bar, p, 9, 1, taub);
#pragma unroll
        for (int i = 0; i < 9; ++i) Fb2[i] = Fgb[i] = Cb2[i] = R(0);
    } else {
        fb |= model_vjp_keep(M, ctx.gap_thresh, F, Fg, C, taub, keep, Fb2, Fgb, Cb2);
    }
    if (fb) atomicAdd(ctx.fallbacks, 1ull);
    if constexpr (MAT) {
        double gm[2];
        model_param_grad(M, F, Fg, keep, taub, gm);
        dmat[sidx] = gm[0];
        dmat[ctx.n + sidx] = gm[1];
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        Fb[i] += Fb2[i];
        Cb[i] += Cb2[i];
    }
    // volume path: c = -k4 vol0 det(Fg)
    R Fgi[9];
    R dFg = inv3(Fg, Fgi);
    R vol = frob(skb, tau) * (-k4 * vol0) * dFg;
    double Fgl[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Fgl[3 * i + j] = (double)Fgb[3 * i + j] + (double)(vol * Fgi[3 * j + i]);

    st3<R>(ib.x, p, ib.sp3, ib.sc3, xb);
    st3<R>(ib.v, p, ib.sp3, ib.sc3, vb);
    st9<R>(ib.C, p, ib.sp9, ib.sc9, Cb);
    st9<R>(ib.F, p, ib.sp9, ib.sc9, Fb);
    if (ib.Fg) {
        double* o = ib.Fg + p * ib.sp9;
        const double* in_g = ob.Fg ? ob.Fg + p * ob.sp9 : nullptr;
#pragma unroll
        for (int i = 0; i < 9; ++i) o[i * ib.sc9] = (in_g ? in_g[i * ob.sc9] : 0.0) + Fgl[i];
    }
    if (dA) dA[sidx] = (sc.growth_mode == 1) ? (Fgl[0] + Fgl[4] + Fgl[8]) * (double)gphi : 0.0;
    if (!finite9(Fb) || !finite9(Cb)) raise_status(ctx.status, MPM_ERR_NONFINITE);
    unmark_cell(ctx, ax, tp.skeys, sidx);
}

// ---------------------------------------------------------------------------
// deterministic per-scene reduction of a per-slot double buffer:
// out[s * stride] = (accumulate ? out[s * stride] : 0) + scale_s * sum_{slots of s} v
// scale_s = 1 (mode 0) or 1/n_s (mode 1)
// ---------------------------------------------------------------------------
constexpr int REDUCE_THREADS = 1024;
__global__ void __launch_bounds__(REDUCE_THREADS)
scene_reduce_kernel(Ctx ctx, const double* __restrict__ v, double* __restrict__ out, int accumulate, int mean,
                    int stride = 1) {
    __shared__ double wsum[REDUCE_THREADS / 32];
    const int s = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const MpmScene& sc = ctx.scenes[s];
    // two interleaved chains per thread, then a fixed shuffle tree: the order
    // depends only on the scene's size
    double a0 = 0.0, a1 = 0.0;
    long long i = sc.p_begin + threadIdx.x;
    for (; i + REDUCE_THREADS < sc.p_end; i += 2 * REDUCE_THREADS) {
        a0 += v[i];
        a1 += v[i + REDUCE_THREADS];
    }
    if (i < sc.p_end) a0 += v[i];
    double acc = a0 + a1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) wsum[warp] = acc;
    __syncthreads();
    if (warp == 0) {
        double r = wsum[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
        if (lane == 0) {
            if (mean) r /= (double)(sc.p_end - sc.p_begin > 0 ? sc.p_end - sc.p_begin : 1);
            out[(long long)s * stride] = accumulate ? out[(long long)s * stride] + r : r;
        }
    }
}

// loss seeds (integrate.py:41-52): sum det F with F_bar = det F F^{-T};
// mean |x - x_obs|^2 with x_bar = 2 (x - x_obs) / n_s
template <typename R>
__global__ void __launch_bounds__(256)
loss_detF_kernel(Ctx ctx, const R* __restrict__ F, long long sp9, long long sc9, double* __restrict__ vals,
                 R* __restrict__ Fb) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ctx.n) return;
    R A[9], Ai[9];
    ld9<R>(F, p, sp9, sc9, A);
    R d = inv3(A, Ai);
    vals[p] = (double)d;
    if (Fb) {
        R o[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) o[3 * i + j] = d * Ai[3 * j + i];
        st9<R>(Fb, p, sp9, sc9, o);
    }
}
template <typename R>
__global__ void __launch_bounds__(256)
loss_mse_kernel(Ctx ctx, const R* __restrict__ x, long long sp3, long long sc3, const R* __restrict__ xo,
                double* __restrict__ vals, R* __restrict__ xb) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ctx.n) return;
    const MpmScene& sc = ctx.scenes[ctx.scene_of[p]];
    R a[3], b[3];
    ld3<R>(x, p, sp3, sc3, a);
    ld3<R>(xo, p, sp3, sc3, b);
    double n = (double)(sc.p_end - sc.p_begin);
    double acc = 0.0;
    R o[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R d = a[i] - b[i];
        acc += (double)d * (double)d;
        o[i] = (R)(2.0 / n) * d;
    }
    vals[p] = acc;
    if (xb) st3<R>(xb, p, sp3, sc3, o);
}

// ---------------------------------------------------------------------------
// constitutive seam, batched over n particles of one model
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256)
stress_kernel(MpmScene sc, long long n, const R* __restrict__ F, const R* __restrict__ Fg, const R* __restrict__ C,
              R* __restrict__ tau, float thresh) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    ModelParams<R> M;
    M.load(sc);
    R f[9], g[9], c[9], t[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        f[i] = F[9 * p + i];
        g[i] = Fg[9 * p + i];
        c[i] = C ? C[9 * p + i] : R(0);
    }
    model_stress(M, thresh, f, g, c, t);
#pragma unroll
    for (int i = 0; i < 9; ++i) tau[9 * p + i] = t[i];
}
template <typename R>
__global__ void __launch_bounds__(256)
stress_vjp_kernel(MpmScene sc, long long n, const R* __restrict__ F, const R* __restrict__ Fg,
                  const R* __restrict__ C, const R* __restrict__ tb, R* __restrict__ Fb, R* __restrict__ Fgb,
                  R* __restrict__ Cb, float thresh) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    ModelParams<R> M;
    M.load(sc);
    R f[9], g[9], c[9], t[9], a[9], b[9], e[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        f[i] = F[9 * p + i];
        g[i] = Fg[9 * p + i];
        c[i] = C ? C[9 * p + i] : R(0);
        t[i] = tb[9 * p + i];
    }
    model_vjp(M, thresh, f, g, c, t, a, b, e);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        Fb[9 * p + i] = a[i];
        Fgb[9 * p + i] = b[i];
        if (Cb) Cb[9 * p + i] = e[i];
    }
}

}  // namespace mpm
