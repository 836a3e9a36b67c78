// Kernels of one MLS-MPM growth step and of its reverse.
//
// Forward (python/morphompm/transfer.py:33-79):
//   bin_kernel       cell key of every particle (stencil base, exact rounding)
//   radix sort       (sort.cuh) cell-sorted particle order, deterministic
//   mark_kernel      first/last sorted slot of every occupied cell, tile flags
//   compact_tiles    active node tiles -> compact grid slots
//   prepass_kernel   stress and the P2G payload of every particle, sorted order
//   scatter_kernel   P2G into a node tile, fixed summation order, + grid update
//   g2p_kernel       gather, advect, F update; clears the cell marks
// Reverse (python/morphompm/transfer.py:82-158):
//   bwd_payload_kernel   G2P adjoint payload (nv_b, Cn_b') per particle
//   scatter_kernel<1>    gv_b scatter + grid adjoint (gmom_b, gm_b)
//   bwd_particle_kernel  P2G adjoint, constitutive VJP, volume path, x_b terms
//
// P2G determinism: particles are sorted by cell; a CTA owns one node tile and
// reads every cell of the tile's 2-cell halo.  A 16-lane half-warp takes one
// cell column (lane = cell), each lane accumulates its cell's particles in
// registers, and the column adds its sums into the shared-memory node tile.
// Columns are processed in 9 colour rounds ((x mod 3, y mod 3) of the column),
// so within a round no two columns touch the same node, and inside a column the
// three z-offsets are written in order between __syncwarp()s.  Every node thus
// sums its contributions in one fixed order and no global atomics are used.
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
template <typename R>
__global__ void __launch_bounds__(256)
bin_kernel(Ctx ctx, MpmParticles P, unsigned* __restrict__ keys) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ctx.n) return;
    int s = ctx.scene_of[p];
    const MpmScene& sc = ctx.scenes[s];
    const SceneAux& ax = ctx.aux[s];
    R x[3];
    ld3<R>(P.x, p, P.sp3, P.sc3, x);
    R inv_dx = (R)(1.0 / sc.dx);
    int base[3];
    R fx[3];
    bool inside = bin_particle(x, inv_dx, sc.shape, base, fx);
    unsigned key;
    if (inside) {
        long long c = ((long long)(base[0] + 2) * (sc.shape[1] + 2) + (base[1] + 2)) * (sc.shape[2] + 2) + (base[2] + 2);
        key = (unsigned)(ax.cell_begin + c);
    } else {
        key = (unsigned)(ax.cell_begin + ax.ncells);
        raise_status(ctx.status, MPM_WARN_OUTSIDE);
    }
    keys[p] = key;
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
// cell marks and tile flags
// ---------------------------------------------------------------------------
__device__ __forceinline__ void decode_cell(const MpmScene& sc, long long c, int cell[3]) {
    long long P1 = sc.shape[1] + 2, P2 = sc.shape[2] + 2;
    cell[2] = (int)(c % P2);
    long long r = c / P2;
    cell[1] = (int)(r % P1);
    cell[0] = (int)(r / P1);
}

__global__ void __launch_bounds__(256)
mark_kernel(Ctx ctx, const unsigned* __restrict__ skeys, int flag_tiles) {
    long long sidx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= ctx.n) return;
    unsigned k = skeys[sidx];
    bool first = sidx == 0 || skeys[sidx - 1] != k;
    bool last = sidx == ctx.n - 1 || skeys[sidx + 1] != k;
    if (!first && !last) return;
    int s = ctx.scene_of[sidx];
    const SceneAux& ax = ctx.aux[s];
    long long c = (long long)k - ax.cell_begin;
    if (c >= ax.ncells) return;     // outside key
    if (first) ctx.cell_first[k] = (int)sidx;
    if (last) ctx.cell_last[k] = (int)(sidx + 1);
    if (first && flag_tiles) {
        const MpmScene& sc = ctx.scenes[s];
        int cell[3];
        decode_cell(sc, c, cell);
        int tlo[3], thi[3];
        const int T[3] = {ctx.tile_xy, ctx.tile_xy, TILE_Z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            int b = cell[d] - 2;
            int lo = b < 0 ? 0 : b;
            int hi = b + 2 > sc.shape[d] - 1 ? sc.shape[d] - 1 : b + 2;
            tlo[d] = lo / T[d];
            thi[d] = hi / T[d];
        }
        for (int a = tlo[0]; a <= thi[0]; ++a)
            for (int b = tlo[1]; b <= thi[1]; ++b)
                for (int e = tlo[2]; e <= thi[2]; ++e)
                    ctx.tile_flag[ax.tile_begin + ((long long)a * ax.ntile[1] + b) * ax.ntile[2] + e] = 1;
    }
}

// ---------------------------------------------------------------------------
// forward prepass: stress -> payload record (sorted order)
// record: fx[0..2], pmass, a = pmass v, B = (pmass C + dt sk) dx
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256)
prepass_kernel(Ctx ctx, MpmParticles P, const unsigned* __restrict__ perm, R* __restrict__ payload, int t) {
    long long sidx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= ctx.n) return;
    long long p = perm[sidx];
    const MpmScene& sc = ctx.scenes[ctx.scene_of[sidx]];
    ModelParams<R> M;
    M.load(sc);
    R x[3], v[3], C[9], F[9], Fg[9];
    ld3<R>(P.x, p, P.sp3, P.sc3, x);
    ld3<R>(P.v, p, P.sp3, P.sc3, v);
    ld9<R>(P.C, p, P.sp9, P.sc9, C);
    ld9<R>(P.F, p, P.sp9, P.sc9, F);
    load_Fg<R>(ctx, sc, P, p, t, Fg, nullptr);
    const R dx = (R)sc.dx, dt = (R)sc.dt, inv_dx = (R)(1.0 / sc.dx);
    const R k4 = R(4) * inv_dx * inv_dx;
    R tau[9];
    bool fb = model_stress(M, ctx.gap_thresh, F, Fg, C, tau);
    if (fb) atomicAdd(ctx.fallbacks, 1ull);
    R c = -k4 * (R)sc.vol0 * det3(Fg);
    const R pm = (R)sc.pmass;
    int base[3];
    R fx[3];
    bin_particle(x, inv_dx, sc.shape, base, fx);
    R rec[PAYLOAD];
    rec[0] = fx[0]; rec[1] = fx[1]; rec[2] = fx[2]; rec[3] = pm;
#pragma unroll
    for (int i = 0; i < 3; ++i) rec[4 + i] = pm * v[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) rec[7 + i] = (pm * C[i] + dt * (c * tau[i])) * dx;
    if (!finite9(tau)) raise_status(ctx.status, MPM_ERR_NONFINITE);
    store_record(payload, sidx, rec);
}

// ---------------------------------------------------------------------------
// P2G scatter into one node tile per CTA iteration (see file header).
// MODE 0: channels (m, mom[3]); epilogue = grid update -> (m, v[3]).
// MODE 1: channels (gv_b[3]);  epilogue = grid adjoint -> (gm_b, gmom_b[3]).
// OXB: stencil x-offsets accumulated per pass over a cell's particles.
// ---------------------------------------------------------------------------
template <typename R, int T, int MODE, int OXB>
__global__ void __launch_bounds__(256)
scatter_kernel(Ctx ctx, const R* __restrict__ payload, const int* __restrict__ active,
               const int* __restrict__ n_active, R* __restrict__ grid_out, const R* __restrict__ grid_fwd,
               int advect) {
    constexpr int TN = T * T * TILE_Z;
    constexpr int NCH = MODE == 0 ? 4 : 3;
    constexpr int HALO = T + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* acc_s = reinterpret_cast<R*>(smem_raw);   // [NCH][TN]

    const int grp = threadIdx.x >> 4;   // 16 column groups
    const int l = threadIdx.x & 15;     // cell within the column
    const int nact = *n_active;

    for (int it = blockIdx.x; it < nact; it += gridDim.x) {
        const int tile = active[it];
        const int s = ctx.tile_scene[tile];
        const MpmScene& sc = ctx.scenes[s];
        const SceneAux& ax = ctx.aux[s];
        long long lt = tile - ax.tile_begin;
        const int tz = (int)(lt % ax.ntile[2]);
        const int ty = (int)((lt / ax.ntile[2]) % ax.ntile[1]);
        const int tx = (int)(lt / ((long long)ax.ntile[2] * ax.ntile[1]));
        const int L0 = tx * T, L1 = ty * T, L2 = tz * TILE_Z;
        const int P0 = sc.shape[0] + 2, P1 = sc.shape[1] + 2, P2 = sc.shape[2] + 2;

        for (int i = threadIdx.x; i < NCH * TN; i += blockDim.x) acc_s[i] = R(0);
        __syncthreads();

        for (int color = 0; color < 9; ++color) {
            const int ca = color / 3, cb = color % 3;
            const int ncy = (HALO - cb + 2) / 3;
            const int ncol = ((HALO - ca + 2) / 3) * ncy;
            for (int c0 = 0; c0 < ncol; c0 += 16) {
                const int col = c0 + grp;
                int first = 0, last = 0, hx = 0, hy = 0;
                if (col < ncol) {
                    hx = ca + 3 * (col / ncy);
                    hy = cb + 3 * (col % ncy);
                    const int cx = L0 + hx, cy = L1 + hy, cz = L2 + l;
                    if (cx < P0 && cy < P1 && cz < P2) {
                        long long key = ax.cell_begin + ((long long)cx * P1 + cy) * P2 + cz;
                        first = ctx.cell_first[key];
                        last = ctx.cell_last[key];
                    }
                }
#pragma unroll 1
                for (int ox0 = 0; ox0 < 3; ox0 += OXB) {
                    R acc[OXB][3][3][NCH];
#pragma unroll
                    for (int a = 0; a < OXB; ++a)
#pragma unroll
                        for (int b = 0; b < 3; ++b)
#pragma unroll
                            for (int c = 0; c < 3; ++c)
#pragma unroll
                                for (int h = 0; h < NCH; ++h) acc[a][b][c][h] = R(0);
                    for (int q = first; q < last; ++q) {
                        R r[PAYLOAD];
                        load_record(payload, q, r);
                        R w[3][3];
                        bspline(r, w);
#pragma unroll
                        for (int a = 0; a < OXB; ++a) {
                            const int ox = ox0 + a;
                            const R dpx = R(ox) - r[0];
                            const R wx = w[ox][0];
#pragma unroll
                            for (int oy = 0; oy < 3; ++oy) {
                                const R dpy = R(oy) - r[1];
                                const R wxy = wx * w[oy][1];
#pragma unroll
                                for (int oz = 0; oz < 3; ++oz) {
                                    const R dpz = R(oz) - r[2];
                                    const R wt = wxy * w[oz][2];
                                    R q0 = r[4] + r[7] * dpx + r[8] * dpy + r[9] * dpz;
                                    R q1 = r[5] + r[10] * dpx + r[11] * dpy + r[12] * dpz;
                                    R q2 = r[6] + r[13] * dpx + r[14] * dpy + r[15] * dpz;
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
                    const bool has = last > first;
#pragma unroll
                    for (int a = 0; a < OXB; ++a) {
                        const int nx = hx - 2 + ox0 + a;
#pragma unroll
                        for (int oz = 0; oz < 3; ++oz) {
                            __syncwarp();
                            const int nz = l - 2 + oz;
#pragma unroll
                            for (int oy = 0; oy < 3; ++oy) {
                                const int ny = hy - 2 + oy;
                                if (has && nx >= 0 && nx < T && ny >= 0 && ny < T && nz >= 0 && nz < TILE_Z) {
                                    const int node = (nx * T + ny) * TILE_Z + nz;
#pragma unroll
                                    for (int h = 0; h < NCH; ++h) acc_s[h * TN + node] += acc[a][oy][oz][h];
                                }
                            }
                        }
                        __syncwarp();
                    }
                }
            }
            __syncthreads();
        }

        // epilogue: node tile -> compact grid records
        const R s_damp = (R)(1.0 - sc.damping);
        const R dt = (R)sc.dt;
        const R eps = (R)sc.mass_eps;
        const R g0 = (R)sc.gravity[0], g1 = (R)sc.gravity[1], g2 = (R)sc.gravity[2];
        for (int node = threadIdx.x; node < TN; node += blockDim.x) {
            const int nz = node % TILE_Z, ny = (node / TILE_Z) % T, nx = node / (TILE_Z * T);
            const int i = L0 + nx, j = L1 + ny, k = L2 + nz;
            if (i >= sc.shape[0] || j >= sc.shape[1] || k >= sc.shape[2]) continue;
            const long long gidx = (long long)it * TN + node;
            R rec[4];
            if constexpr (MODE == 0) {
                const R m = acc_s[node];
                rec[0] = m; rec[1] = R(0); rec[2] = R(0); rec[3] = R(0);
                if (m > eps && node_free(sc, i, j, k)) {
                    rec[1] = (s_damp * acc_s[TN + node]) / m + s_damp * dt * g0;
                    rec[2] = (s_damp * acc_s[2 * TN + node]) / m + s_damp * dt * g1;
                    rec[3] = (s_damp * acc_s[3 * TN + node]) / m + s_damp * dt * g2;
                }
            } else {
                R f[4];
                load_node(grid_fwd, gidx, f);
                rec[0] = R(0); rec[1] = R(0); rec[2] = R(0); rec[3] = R(0);
                const R m = f[0];
                if (m > eps && node_free(sc, i, j, k)) {
                    const R b0 = acc_s[node], b1 = acc_s[TN + node], b2 = acc_s[2 * TN + node];
                    rec[1] = (s_damp * b0) / m;
                    rec[2] = (s_damp * b1) / m;
                    rec[3] = (s_damp * b2) / m;
                    if (advect) {
                        const R sd = s_damp * dt;
                        rec[0] = -(b0 * (f[1] - sd * g0) + b1 * (f[2] - sd * g1) + b2 * (f[3] - sd * g2)) / m;
                    }
                }
            }
            store_node(grid_out, gidx, rec);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// stencil addressing into the compact per-tile grid
// ---------------------------------------------------------------------------
template <int T>
struct Stencil {
    int node[3][3];     // node index per axis and offset (-1 if out of range)
    int tl[3][3];       // tile coordinate
    int lc[3][3];       // coordinate inside the tile
    __device__ __forceinline__ void init(const MpmScene& sc, const int base[3]) {
        const int TT[3] = {T, T, TILE_Z};
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int o = 0; o < 3; ++o) {
                int n = base[d] + o;
                bool ok = n >= 0 && n < sc.shape[d];
                node[d][o] = ok ? n : -1;
                int t = ok ? n / TT[d] : 0;
                tl[d][o] = t;
                lc[d][o] = ok ? n - t * TT[d] : 0;
            }
    }
    // compact record index or -1
    __device__ __forceinline__ long long rec(const Ctx& ctx, const SceneAux& ax, const int* __restrict__ tile_slot,
                                             int a, int b, int c) const {
        if (node[0][a] < 0 || node[1][b] < 0 || node[2][c] < 0) return -1;
        long long tile = ax.tile_begin + ((long long)tl[0][a] * ax.ntile[1] + tl[1][b]) * ax.ntile[2] + tl[2][c];
        int slot = tile_slot[tile];
        if (slot < 0) return -1;
        return (long long)slot * (T * T * TILE_Z) + (lc[0][a] * T + lc[1][b]) * TILE_Z + lc[2][c];
    }
};

// ---------------------------------------------------------------------------
// G2P + advection + F update (transfer.py:61-79); writes the output state in
// the input's particle order and clears the cell marks of this step.
// ---------------------------------------------------------------------------
template <typename R, int T>
__global__ void __launch_bounds__(256)
g2p_kernel(Ctx ctx, Tape<R> tp, MpmParticles in, MpmParticles out, int advect) {
    long long sidx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= ctx.n) return;
    long long p = tp.perm[sidx];
    const int s = ctx.scene_of[sidx];
    const MpmScene& sc = ctx.scenes[s];
    const SceneAux& ax = ctx.aux[s];
    const R dx = (R)sc.dx, dt = (R)sc.dt, inv_dx = (R)(1.0 / sc.dx);
    const R k4 = R(4) * inv_dx * inv_dx;
    R x[3], F[9];
    ld3<R>(in.x, p, in.sp3, in.sc3, x);
    ld9<R>(in.F, p, in.sp9, in.sc9, F);
    int base[3];
    R fx[3];
    bin_particle(x, inv_dx, sc.shape, base, fx);
    R w[3][3];
    bspline(fx, w);
    Stencil<T> st;
    st.init(sc, base);
    R nv[3] = {0, 0, 0}, nC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                long long r = st.rec(ctx, ax, tp.tile_slot, a, b, c);
                if (r < 0) continue;
                R g[4];
                load_node(tp.grid, r, g);
                const R wt = w[a][0] * w[b][1] * w[c][2];
                const R dp[3] = {(R(a) - fx[0]) * dx, (R(b) - fx[1]) * dx, (R(c) - fx[2]) * dx};
                const R kw = k4 * wt;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    nv[i] += wt * g[1 + i];
#pragma unroll
                    for (int j = 0; j < 3; ++j) nC[3 * i + j] += kw * (g[1 + i] * dp[j]);
                }
            }
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
    // clear this step's cell marks
    unsigned k = tp.skeys[sidx];
    if (sidx == 0 || tp.skeys[sidx - 1] != k) {
        if ((long long)k - ax.cell_begin < ax.ncells) {
            ctx.cell_first[k] = 0;
            ctx.cell_last[k] = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// reverse: G2P-adjoint payload (transfer.py:99-119)
// record: fx, m = 0, a = nv_b, B = k4 dx Cn_b'   with
//   nv_b = vn_b + dt xn_b (advect),  Cn_b' = Cn_b + dt Fn_b F^T
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256)
bwd_payload_kernel(Ctx ctx, const unsigned* __restrict__ perm, MpmParticles in, MpmCotangents ob,
                   R* __restrict__ payload, int advect) {
    long long sidx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= ctx.n) return;
    long long p = perm[sidx];
    const MpmScene& sc = ctx.scenes[ctx.scene_of[sidx]];
    const R dx = (R)sc.dx, dt = (R)sc.dt, inv_dx = (R)(1.0 / sc.dx);
    const R k4 = R(4) * inv_dx * inv_dx;
    R x[3], F[9], xb[3], vb[3], Cb[9], Fb[9];
    ld3<R>(in.x, p, in.sp3, in.sc3, x);
    ld9<R>(in.F, p, in.sp9, in.sc9, F);
    ld3<R>(ob.x, p, ob.sp3, ob.sc3, xb);
    ld3<R>(ob.v, p, ob.sp3, ob.sc3, vb);
    ld9<R>(ob.C, p, ob.sp9, ob.sc9, Cb);
    ld9<R>(ob.F, p, ob.sp9, ob.sc9, Fb);
    int base[3];
    R fx[3];
    bin_particle(x, inv_dx, sc.shape, base, fx);
    R FbFt[9];
    mmT(Fb, F, FbFt);
    R rec[PAYLOAD];
    rec[0] = fx[0]; rec[1] = fx[1]; rec[2] = fx[2]; rec[3] = R(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) rec[4 + i] = advect ? vb[i] + dt * xb[i] : vb[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) rec[7 + i] = k4 * (Cb[i] + dt * FbFt[i]) * dx;
    store_record(payload, sidx, rec);
}

// ---------------------------------------------------------------------------
// reverse: per-particle cotangents (transfer.py:99-119 x_b terms, 129-156)
// ---------------------------------------------------------------------------
template <typename R, int T>
__global__ void __launch_bounds__(256)
bwd_particle_kernel(Ctx ctx, Tape<R> tp, const R* __restrict__ gridb, MpmParticles in, const R* __restrict__ outC,
                    MpmCotangents ob, MpmCotangents ib, double* __restrict__ dA, int advect, int t) {
    long long sidx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sidx >= ctx.n) return;
    long long p = tp.perm[sidx];
    const int s = ctx.scene_of[sidx];
    const MpmScene& sc = ctx.scenes[s];
    const SceneAux& ax = ctx.aux[s];
    ModelParams<R> M;
    M.load(sc);
    const R dx = (R)sc.dx, dt = (R)sc.dt, inv_dx = (R)(1.0 / sc.dx);
    const R k4 = R(4) * inv_dx * inv_dx;
    const R pm = (R)sc.pmass;
    R x[3], v[3], C[9], F[9], Fg[9], Cn[9];
    R gphi;
    ld3<R>(in.x, p, in.sp3, in.sc3, x);
    ld3<R>(in.v, p, in.sp3, in.sc3, v);
    ld9<R>(in.C, p, in.sp9, in.sc9, C);
    ld9<R>(in.F, p, in.sp9, in.sc9, F);
    load_Fg<R>(ctx, sc, in, p, t, Fg, &gphi);
    ld9<R>(outC, p, in.sp9, in.sc9, Cn);
    R xnb[3], vnb[3], Cnb_in[9], Fnb[9];
    ld3<R>(ob.x, p, ob.sp3, ob.sc3, xnb);
    ld3<R>(ob.v, p, ob.sp3, ob.sc3, vnb);
    ld9<R>(ob.C, p, ob.sp9, ob.sc9, Cnb_in);
    ld9<R>(ob.F, p, ob.sp9, ob.sc9, Fnb);

    int base[3];
    R fx[3];
    bin_particle(x, inv_dx, sc.shape, base, fx);
    R w[3][3], dw[3][3];
    bspline(fx, w);
    bspline_grad(fx, dw);

    R tau[9];
    bool fb = model_stress(M, ctx.gap_thresh, F, Fg, C, tau);
    R c = -k4 * (R)sc.vol0 * det3(Fg);
    R sk[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) sk[i] = c * tau[i];

    R nvb[3], Cnb[9], Fb[9], xb[3], vb[3] = {0, 0, 0}, Sb[9];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        nvb[i] = advect ? vnb[i] + dt * xnb[i] : vnb[i];
        xb[i] = advect ? xnb[i] : R(0);
    }
    {
        R FbFt[9];
        mmT(Fnb, F, FbFt);
#pragma unroll
        for (int i = 0; i < 9; ++i) Cnb[i] = Cnb_in[i] + dt * FbFt[i];
        R A[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) A[i] = ((i % 4 == 0) ? R(1) : R(0)) + dt * Cn[i];
        mTm(A, Fnb, Fb);   // (I + dt Cn)^T Fn_b
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) Sb[i] = R(0);

    Stencil<T> st;
    st.init(sc, base);
#pragma unroll 1
    for (int a = 0; a < 3; ++a)
#pragma unroll 1
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                long long r = st.rec(ctx, ax, tp.tile_slot, a, b, cc);
                if (r < 0) continue;
                R gf[4], gb[4];
                load_node(tp.grid, r, gf);
                load_node(gridb, r, gb);
                const R wt = w[a][0] * w[b][1] * w[cc][2];
                const R dp[3] = {(R(a) - fx[0]) * dx, (R(b) - fx[1]) * dx, (R(cc) - fx[2]) * dx};
                const R* gv = gf + 1;
                const R* mb = gb + 1;
                if (advect) {
                    const R dW[3] = {dw[a][0] * w[b][1] * w[cc][2] * inv_dx, w[a][0] * dw[b][1] * w[cc][2] * inv_dx,
                                     w[a][0] * w[b][1] * dw[cc][2] * inv_dx};
                    // G2P adjoint through the weights and dpos
                    R t1 = nvb[0] * gv[0] + nvb[1] * gv[1] + nvb[2] * gv[2];
                    R Cd[3];
#pragma unroll
                    for (int i = 0; i < 3; ++i) Cd[i] = Cnb[3 * i] * dp[0] + Cnb[3 * i + 1] * dp[1] + Cnb[3 * i + 2] * dp[2];
                    R t2 = k4 * (gv[0] * Cd[0] + gv[1] * Cd[1] + gv[2] * Cd[2]);
                    const R kw = k4 * wt;
#pragma unroll
                    for (int i = 0; i < 3; ++i)
                        xb[i] += (t1 + t2) * dW[i] - kw * (Cnb[i] * gv[0] + Cnb[3 + i] * gv[1] + Cnb[6 + i] * gv[2]);
                    // P2G adjoint through the weights and dpos
                    R Q2[3];
#pragma unroll
                    for (int i = 0; i < 3; ++i)
                        Q2[i] = pm * (v[i] + C[3 * i] * dp[0] + C[3 * i + 1] * dp[1] + C[3 * i + 2] * dp[2])
                              + (sk[3 * i] * dp[0] + sk[3 * i + 1] * dp[1] + sk[3 * i + 2] * dp[2]) * dt;
                    R mq = mb[0] * Q2[0] + mb[1] * Q2[1] + mb[2] * Q2[2] + gb[0] * pm;
#pragma unroll
                    for (int i = 0; i < 3; ++i)
                        xb[i] += mq * dW[i]
                               - (pm * (C[i] * mb[0] + C[3 + i] * mb[1] + C[6 + i] * mb[2])
                                  + dt * (sk[i] * mb[0] + sk[3 + i] * mb[1] + sk[6 + i] * mb[2])) * wt;
                }
                const R wp = wt * pm;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    vb[i] += wp * mb[i];
#pragma unroll
                    for (int j = 0; j < 3; ++j) Sb[3 * i + j] += wt * (mb[i] * dp[j]);
                }
            }
    R Cb[9], skb[9], taub[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        Cb[i] = pm * Sb[i];
        skb[i] = dt * Sb[i];
        taub[i] = c * skb[i];
    }
    R Fb2[9], Fgb[9], Cb2[9];
    fb |= model_vjp(M, ctx.gap_thresh, F, Fg, C, taub, Fb2, Fgb, Cb2);
    if (fb) atomicAdd(ctx.fallbacks, 1ull);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        Fb[i] += Fb2[i];
        Cb[i] += Cb2[i];
    }
    // volume path: c = -k4 vol0 det(Fg)
    R Fgi[9];
    R dFg = inv3(Fg, Fgi);
    R vol = frob(skb, tau) * (-k4 * (R)sc.vol0) * dFg;
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
    unsigned k = tp.skeys[sidx];
    if (sidx == 0 || tp.skeys[sidx - 1] != k) {
        if ((long long)k - ax.cell_begin < ax.ncells) {
            ctx.cell_first[k] = 0;
            ctx.cell_last[k] = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// deterministic per-scene reduction of a per-slot double buffer:
// out[s] = (accumulate ? out[s] : 0) + scale_s * sum_{slots of s} v
// scale_s = 1 (mode 0) or 1/n_s (mode 1)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
scene_reduce_kernel(Ctx ctx, const double* __restrict__ v, double* __restrict__ out, int accumulate, int mean) {
    __shared__ double red[256];
    const int s = blockIdx.x;
    const MpmScene& sc = ctx.scenes[s];
    double acc = 0.0;
    for (long long i = sc.p_begin + threadIdx.x; i < sc.p_end; i += 256) acc += v[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double r = red[0];
        if (mean) r /= (double)(sc.p_end - sc.p_begin > 0 ? sc.p_end - sc.p_begin : 1);
        out[s] = accumulate ? out[s] + r : r;
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
