// Host side of the C ABI (include/morphompm_b200.h): plan construction,
// workspace/tape layout, and the launch sequences of one forward and one
// reverse growth step.  No device memory is allocated here.
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <mutex>
#include <new>
#include <type_traits>
#include <vector>

#include "../../include/morphompm_b200.h"
#include "mpm_common.cuh"
#include "constitutive.cuh"
#include "sort.cuh"
#include "mpm_kernels.cuh"

using namespace mpm;

namespace {

constexpr size_t ALIGN = 256;
inline size_t align_up(size_t v) { return (v + ALIGN - 1) / ALIGN * ALIGN; }

struct Layout {
    size_t off = 0;
    size_t take(size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes);
        return o;
    }
};

}  // namespace

struct MpmPlan {
    std::vector<MpmScene> scenes;
    std::vector<SceneAux> aux;
    std::vector<int> scene_of;
    std::vector<int> tile_scene;
    int real_bytes = 8;
    MpmTuning tune{};
    long long n = 0, n_tiles = 0, n_keys = 0;
    int key_bits = 1, passes = 1, nblk_sort = 1;
    int TN = 0, active_cap = 0;
    bool any_growth = false;
    // workspace offsets
    size_t o_scenes, o_aux, o_scene_of, o_tile_scene, o_status, o_cell_seg, o_blk, o_tblk;
    size_t o_tile_flag, o_keys, o_kalt0, o_valt0, o_kalt1, o_valt1, o_hist, o_totals, o_payload, o_sums;
    size_t o_dense_f = 0, o_dense_b = 0;
    // incremental re-sort of chained steps (SIZE_MAX: not laid out)
    size_t o_mflag = SIZE_MAX, o_pflag = 0, o_mask = 0, o_pmask = 0, o_wpre = 0, o_rblk = 0, o_pblk = 0;
    size_t o_mkey = 0, o_mpart = 0, o_okey = 0, o_opart = 0, o_rint = 0, o_hist1 = 0;
    int nblk_sort1 = 1;     // blocks of the movers' radix sort (one key per thread)
    int nblk_resort = 1;
    char* chain_tape = nullptr;    // the tape whose sorted order the emitted mover flags refer to
    // runs of consecutive scenes with one material model (their slot ranges);
    // grouped: every model has one run, so each run gets a kernel for its model
    std::vector<int> run_kind;
    std::vector<long long> run_begin, run_end;
    bool runs_grouped = false;
    long long n_nodes = 0;
    size_t o_dbuf, o_tape;
    int nblk_seg = 1, nblk_tile = 1;
    // the state whose keys and P2G records the last MPM_FWD_EMIT call formed
    bool chain_valid = false;
    int chain_t = 0;
    bool tile_flags_pending = false;   // an emitting G2P flagged the next step's tiles
    MpmParticles chain_state{};
    size_t ws_bytes = 0;
    // tape offsets
    size_t t_skeys, t_perm, t_seg_first, t_seg_last, t_nseg, t_active, t_nact, t_grid, tape_bytes = 0;
    char* ws = nullptr;
    const void* phi = nullptr;
    const void* pmass_p = nullptr;     // per-particle masses / reference volumes (optional)
    const void* vol0_p = nullptr;
    const void* ext_tau = nullptr;     // caller-supplied stress and its cotangent (MPM_MODEL_EXTERNAL)
    void* ext_tau_bar = nullptr;
    bool any_external = false;
    int n_sm = 148;
    // profiling
    uint32_t prof_mask = 0;
    int prof_max = 0, prof_n = 0;
    std::vector<cudaEvent_t> ev0, ev1;
    std::vector<int> ev_kind;
    long long launches = 0;
};

namespace {

template <typename T>
T* at(MpmPlan* P, size_t off) { return reinterpret_cast<T*>(P->ws + off); }

Ctx make_ctx(MpmPlan* P) {
    Ctx c;
    c.scenes = at<const MpmScene>(P, P->o_scenes);
    c.aux = at<const SceneAux>(P, P->o_aux);
    c.scene_of = at<const int>(P, P->o_scene_of);
    c.tile_scene = at<const int>(P, P->o_tile_scene);
    c.status = at<int>(P, P->o_status);
    c.fallbacks = reinterpret_cast<unsigned long long*>(P->ws + P->o_status + 64);
    c.cell_seg = at<int>(P, P->o_cell_seg);
    c.seg_first = nullptr;    // in the step's tape (bind_segments)
    c.seg_last = nullptr;
    c.n_seg = nullptr;
    c.blk_count = at<unsigned>(P, P->o_blk);
    c.tile_flag = at<int>(P, P->o_tile_flag);
    c.phi = P->phi;
    c.pmass_p = P->pmass_p;
    c.vol0_p = P->vol0_p;
    c.ext_tau = P->ext_tau;
    c.ext_tau_bar = P->ext_tau_bar;
    c.dense_f = P->ws + P->o_dense_f;
    c.dense_b = P->ws + P->o_dense_b;
    c.mover_flag = P->o_mflag == SIZE_MAX ? nullptr : at<unsigned char>(P, P->o_mflag);
    c.mover_pflag = P->o_mflag == SIZE_MAX ? nullptr : at<unsigned char>(P, P->o_pflag);
    c.n = P->n;
    c.n_tiles = P->n_tiles;
    c.n_keys = P->n_keys;
    c.n_nodes = P->n_nodes;
    c.grid_nodes = (long long)P->active_cap * P->TN;
    c.n_scenes = (int)P->scenes.size();
    c.tile_xy = P->tune.tile_xy;
    c.tile_z = P->tune.tile_z;
    c.tile_xy_shift = P->tune.tile_xy == 16 ? 4 : (P->tune.tile_xy == 8 ? 3 : 2);
    c.tile_z_shift = P->tune.tile_z == 16 ? 4 : (P->tune.tile_z == 8 ? 3 : 2);
    c.active_cap = P->active_cap;
    c.gap_thresh = P->tune.fp64_gap_thresh < 0 ? 0.0f : P->tune.fp64_gap_thresh;
    return c;
}

// the segment table of a step lives in its tape: the reverse step reuses it
void bind_segments(MpmPlan* P, Ctx& c, const char* t) {
    c.seg_first = reinterpret_cast<int*>(const_cast<char*>(t) + P->t_seg_first);
    c.seg_last = reinterpret_cast<int*>(const_cast<char*>(t) + P->t_seg_last);
    c.n_seg = reinterpret_cast<int*>(const_cast<char*>(t) + P->t_nseg);
}

template <typename R>
Tape<R> make_tape(MpmPlan* P, char* t) {
    Tape<R> tp;
    tp.skeys = reinterpret_cast<unsigned*>(t + P->t_skeys);
    tp.perm = reinterpret_cast<unsigned*>(t + P->t_perm);
    tp.active = reinterpret_cast<int*>(t + P->t_active);
    tp.n_active = reinterpret_cast<int*>(t + P->t_nact);
    tp.grid = reinterpret_cast<R*>(t + P->t_grid);
    return tp;
}

void record_event(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    cudaEventRecordWithFlags(e, st, cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal
                                                                        : cudaEventRecordDefault);
}

// NVTX range names of the kernel kinds (MPM_K_*), for profilers' filters
const char* const KIND_NAME[MPM_K_COUNT] = {"mpm.bin", "mpm.sort", "mpm.mark", "mpm.compact",
                                            "mpm.prepass", "mpm.p2g", "mpm.g2p", "mpm.bwd_payload",
                                            "mpm.bwd_p2g", "mpm.bwd_particle", "mpm.reduce"};

// Brackets one launch site: an NVTX range named for its kind, the launch
// count, and, when profiling this kind, start/stop events around it.
struct Site {
    MpmPlan* P;
    cudaStream_t st;
    bool on;
    Site(MpmPlan* p, int kind, int kernels, cudaStream_t s) : P(p), st(s) {
        nvtxRangePushA(KIND_NAME[kind]);
        P->launches += kernels;
        on = ((P->prof_mask >> kind) & 1u) && P->prof_n < P->prof_max;
        if (on) {
            P->ev_kind[P->prof_n] = kind;
            record_event(P->ev0[P->prof_n], st);
        }
    }
    ~Site() {
        if (on) {
            record_event(P->ev1[P->prof_n], st);
            ++P->prof_n;
        }
        nvtxRangePop();
    }
};

inline int grid_for(long long n, int block) { return (int)std::max<long long>(1, (n + block - 1) / block); }

inline int check_launch() {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}

// segment table of the sorted keys (and, in the forward, the active tile flags)
int build_segments(MpmPlan* P, const Ctx& ctx, const unsigned* skeys, cudaStream_t st) {
    Site site(P, MPM_K_MARK, 3, st);
    seg_count_kernel<<<P->nblk_seg, SEG_THREADS, 0, st>>>(ctx, skeys);
    scan_counts_kernel<<<1, 1024, 0, st>>>(ctx.blk_count, P->nblk_seg, ctx.n_seg, INT_MAX, ctx.status);
    seg_write_kernel<<<P->nblk_seg, SEG_THREADS, 0, st>>>(ctx, skeys);
    return check_launch();
}

template <typename R, int MODE>
void* sums_fn(int oxb) {
    if constexpr (sizeof(R) == 4) {
        if (oxb == 3) return (void*)cell_sums_kernel<R, MODE, 3>;
    }
    return (void*)cell_sums_kernel<R, MODE, 1>;
}

template <typename R, int T, int MODE>
void* nodes_fn_z(int TZ) {
    if (TZ == 8) return (void*)node_sums_kernel<R, T, 8, MODE>;
    if (TZ == 16) return (void*)node_sums_kernel<R, T, 16, MODE>;
    return (void*)node_sums_kernel<R, T, 4, MODE>;
}
template <typename R, int MODE>
void* nodes_fn(int T, int TZ) {
    if (T == 8) return nodes_fn_z<R, 8, MODE>(TZ);
    if (T == 16) return nodes_fn_z<R, 16, MODE>(TZ);
    return nodes_fn_z<R, 4, MODE>(TZ);
}

// P2G phase 2 (node gather + grid epilogue) over the active tiles
template <typename R>
int launch_nodes(MpmPlan* P, int mode, const Ctx& ctx, const int* active, const int* nact, R* grid_out,
                 const R* grid_fwd, int advect, cudaStream_t st) {
    const R* Sc = at<R>(P, P->o_sums);
    long long cap = P->n;
    int ctas = P->n_sm * std::max(1, P->tune.scatter_ctas_per_sm);
    ctas = std::max(1, std::min(ctas, P->active_cap));
    void* f2 = mode == 0 ? nodes_fn<R, 0>(P->tune.tile_xy, P->tune.tile_z)
                         : nodes_fn<R, 1>(P->tune.tile_xy, P->tune.tile_z);
    void* a2[] = {(void*)&ctx, (void*)&Sc, (void*)&cap, (void*)&active, (void*)&nact, (void*)&grid_out,
                  (void*)&grid_fwd, (void*)&advect};
    return cudaLaunchKernel(f2, dim3(ctas), dim3(1024), a2, 0, st) == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}

// two-phase P2G: per-cell stencil sums, then per-node gather + grid epilogue
template <typename R>
int launch_p2g(MpmPlan* P, int mode, const Ctx& ctx, const unsigned* perm, const R* payload, const int* active,
               const int* nact,
               R* grid_out, const R* grid_fwd, int advect, cudaStream_t st) {
    R* S = at<R>(P, P->o_sums);
    long long cap = P->n;
    int blocks1 = (int)std::min<long long>((P->n + 127) / 128, (long long)P->n_sm * 16);
    blocks1 = std::max(1, blocks1);
    void* f1 = mode == 0 ? sums_fn<R, 0>(P->tune.scatter_oxb) : sums_fn<R, 1>(P->tune.scatter_oxb);
    void* a1[] = {(void*)&ctx, (void*)&perm, (void*)&payload, (void*)&S, (void*)&cap};
    if (cudaLaunchKernel(f1, dim3(blocks1), dim3(128), a1, 0, st) != cudaSuccess) return MPM_ERR_CUDA;
    P->launches += 1;   // the Site around this call counts one
    return launch_nodes<R>(P, mode, ctx, active, nact, grid_out, grid_fwd, advect, st);
}

// Stable LSD radix sort of kin (with payload vin, or the index when null)
// into (kout, vout), through the alternate buffers a0 and a1 (a1 may be the
// input's own buffers), ITEMS keys per thread over nblk blocks with the digit
// counts in hist; n_dev (may be null): sort the first *n_dev keys.
template <int ITEMS>
int run_radix(MpmPlan* P, const unsigned* kin, const unsigned* vin, unsigned* kout, unsigned* vout, unsigned* a0k,
              unsigned* a0v, unsigned* a1k, unsigned* a1v, unsigned* hist, int nblk, const int* n_dev,
              cudaStream_t st) {
    unsigned* totals = at<unsigned>(P, P->o_totals);
    const int tile = SORT_THREADS * ITEMS;
    const unsigned* ksrc = kin;
    const unsigned* vsrc = vin;
    // the movers' sort (a device-side count, typically about a hundred of the nblk
    // possible 256-key tiles): 4 blocks per SM stride over the active tiles
    // instead of one block per possible tile
    const int grid = ITEMS == 1 ? std::max(1, std::min(nblk, P->n_sm * 4)) : nblk;
    for (int pass = 0; pass < P->passes; ++pass) {
        const int shift = pass * RADIX_BITS;
        const bool last = pass == P->passes - 1;
        unsigned* kdst = last ? kout : ((pass & 1) ? a1k : a0k);
        unsigned* vdst = last ? vout : ((pass & 1) ? a1v : a0v);
        radix_hist_kernel<ITEMS><<<grid, SORT_THREADS, 0, st>>>(ksrc, P->n, shift, hist, nblk, n_dev);
        radix_rowsum_kernel<<<RADIX, 256, 0, st>>>(hist, nblk, totals, tile, n_dev);
        radix_rowscan_kernel<<<RADIX, 256, 0, st>>>(hist, nblk, totals, tile, n_dev);
        radix_scatter_kernel<ITEMS><<<grid, SORT_THREADS, 0, st>>>(ksrc, vsrc, P->n, shift, hist, nblk, kdst, vdst,
                                                                  n_dev);
        ksrc = kdst;
        vsrc = vdst;
    }
    return check_launch();
}

// Calls f(model constant, first slot, end slot) once per run of scenes with
// one material model when the plan's scenes are grouped by model (f then
// launches the kernel specialised for that model), else once over all slots
// with the runtime model switch (constant -1).  Returns the number of calls.
template <typename Fn>
int for_model_runs(const MpmPlan* P, Fn&& f) {
    if (!P->runs_grouped) {
        f(std::integral_constant<int, -1>{}, 0LL, P->n);
        return 1;
    }
    int k = 0;
    for (size_t r = 0; r < P->run_kind.size(); ++r) {
        const long long b = P->run_begin[r], e = P->run_end[r];
        switch (P->run_kind[r]) {
            case MPM_MODEL_NEOHOOKEAN: f(std::integral_constant<int, MPM_MODEL_NEOHOOKEAN>{}, b, e); break;
            case MPM_MODEL_HENCKY: f(std::integral_constant<int, MPM_MODEL_HENCKY>{}, b, e); break;
            case MPM_MODEL_HERSCHEL_BULKLEY:
                f(std::integral_constant<int, MPM_MODEL_HERSCHEL_BULKLEY>{}, b, e);
                break;
            default: f(std::integral_constant<int, -1>{}, b, e); break;
        }
        ++k;
    }
    return k;
}

int model_run_count(const MpmPlan* P) { return P->runs_grouped ? (int)P->run_kind.size() : 1; }

// stable LSD radix sort of the binning keys -> tape (skeys, perm)
int run_sort(MpmPlan* P, const unsigned* keys, unsigned* skeys, unsigned* perm, cudaStream_t st) {
    Site site(P, MPM_K_SORT, 4 * P->passes, st);
    return run_radix<SORT_ITEMS>(P, keys, nullptr, skeys, perm, at<unsigned>(P, P->o_kalt0),
                                 at<unsigned>(P, P->o_valt0), at<unsigned>(P, P->o_kalt1),
                                 at<unsigned>(P, P->o_valt1), at<unsigned>(P, P->o_hist), P->nblk_sort, nullptr, st);
}

// Sorted order of a chained step from the previous step's (old_tape) and the
// mover flags its emitting G2P wrote (sort.cuh, incremental re-sort): the
// movers, gathered in particle order, are radix-sorted by key on their count
// held on the device and merged with the slots that kept their key.
int run_resort(MpmPlan* P, const char* old_tape, char* tape, const unsigned* keys, cudaStream_t st) {
    const unsigned* ok = reinterpret_cast<const unsigned*>(old_tape + P->t_skeys);
    const unsigned* op = reinterpret_cast<const unsigned*>(old_tape + P->t_perm);
    unsigned* nk = reinterpret_cast<unsigned*>(tape + P->t_skeys);
    unsigned* np = reinterpret_cast<unsigned*>(tape + P->t_perm);
    const size_t nb4 = (size_t)P->n * 4;
    if (old_tape == tape) {
        // the old order is overwritten by the new one: read it from a copy
        unsigned* ck = at<unsigned>(P, P->o_kalt0);
        unsigned* cp = at<unsigned>(P, P->o_valt0);
        if (cudaMemcpyAsync(ck, ok, nb4, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(cp, op, nb4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return MPM_ERR_CUDA;
        ok = ck;
        op = cp;
    }
    unsigned* mask = at<unsigned>(P, P->o_mask);
    unsigned* pmask = at<unsigned>(P, P->o_pmask);
    unsigned* wpre = at<unsigned>(P, P->o_wpre);
    unsigned* rblk = at<unsigned>(P, P->o_rblk);
    unsigned* pblk = at<unsigned>(P, P->o_pblk);
    unsigned* mk = at<unsigned>(P, P->o_mkey);
    unsigned* mp = at<unsigned>(P, P->o_mpart);
    unsigned* sk = at<unsigned>(P, P->o_okey);
    unsigned* sp = at<unsigned>(P, P->o_opart);
    int* n_movers = at<int>(P, P->o_rint);
    const unsigned char* sflag = at<const unsigned char>(P, P->o_mflag);
    const unsigned char* pflag = at<const unsigned char>(P, P->o_pflag);
    int* status = at<int>(P, P->o_status);
    // count, two scans, compact; per radix pass hist, row sums, row scans, scatter; the two placements
    Site site(P, MPM_K_SORT, 6 + 4 * P->passes, st);
    const int nb = P->nblk_resort;
    resort_count_kernel<<<nb, RESORT_THREADS, 0, st>>>(sflag, pflag, P->n, mask, pmask, rblk, pblk);
    scan_counts_kernel<<<1, 1024, 0, st>>>(rblk, nb, n_movers + 1, INT_MAX, status);
    scan_counts_kernel<<<1, 1024, 0, st>>>(pblk, nb, n_movers, INT_MAX, status);
    resort_compact_kernel<<<nb, RESORT_THREADS, 0, st>>>(mask, pmask, P->n, rblk, pblk, keys, wpre, mk, mp);
    int rc = check_launch();
    if (rc) return rc;
    // movers in particle order -> (key, particle) order, in (sk, sp); one key per
    // thread, so that the movers spread over many blocks
    rc = run_radix<1>(P, mk, mp, sk, sp, at<unsigned>(P, P->o_kalt1), at<unsigned>(P, P->o_valt1), mk, mp,
                      at<unsigned>(P, P->o_hist1), P->nblk_sort1, n_movers, st);
    if (rc) return rc;
    const int gs = grid_for(P->n, (RESORT_THREADS / 32) * 32 * STAY_ROUNDS);    // a warp per 256 slots
    resort_place_stayers_kernel<<<gs, RESORT_THREADS, 0, st>>>(mask, wpre, P->n, ok, op, sk, sp, n_movers, nk, np);
    const int gm = (int)std::max<long long>(1, std::min<long long>(grid_for(P->n, RESORT_THREADS), (long long)P->n_sm * 8));
    resort_place_movers_kernel<<<gm, RESORT_THREADS, 0, st>>>(mask, wpre, P->n, ok, op, sk, sp, n_movers, nk, np);
    return check_launch();
}

// flags: MPM_FWD_CHAINED (keys and P2G records of `in` already formed by the
// previous step's G2P), MPM_FWD_EMIT (form them for `out` in this G2P)
template <typename R>
int step_fwd_R(MpmPlan* P, const MpmParticles& in, MpmParticles& out, int advect, int t, char* tape,
               int flags, cudaStream_t st) {
    const bool chained = (flags & MPM_FWD_CHAINED) != 0, emit = (flags & MPM_FWD_EMIT) != 0;
    Ctx ctx = make_ctx(P);
    bind_segments(P, ctx, tape);
    Tape<R> tp = make_tape<R>(P, tape);
    const int B = P->tune.particle_block;
    const int g = grid_for(P->n, B);
    unsigned* keys = at<unsigned>(P, P->o_keys);
    R* payload = at<R>(P, P->o_payload);
    if (!chained) { Site s(P, MPM_K_BIN, 1, st); bin_kernel<R><<<g, B, 0, st>>>(ctx, in, keys); }
    int rc = chained && P->chain_tape && ctx.mover_flag ? run_resort(P, P->chain_tape, tape, keys, st)
                                                        : run_sort(P, keys, tp.skeys, tp.perm, st);
    if (rc) return rc;
    rc = build_segments(P, ctx, tp.skeys, st);
    if (rc) return rc;
    {
        Site s(P, MPM_K_COMPACT, 3, st);
        unsigned* tblk = at<unsigned>(P, P->o_tblk);
        tile_count_kernel<<<P->nblk_tile, SEG_THREADS, 0, st>>>(ctx.tile_flag, P->n_tiles, tblk);
        scan_counts_kernel<<<1, 1024, 0, st>>>(tblk, P->nblk_tile, tp.n_active, P->active_cap, ctx.status);
        tile_write_kernel<<<P->nblk_tile, SEG_THREADS, 0, st>>>(ctx.tile_flag, P->n_tiles, tblk, tp.active,
                                                                P->active_cap);
    }
    if (!chained) { Site s(P, MPM_K_PREPASS, 1, st); prepass_kernel<R><<<g, B, 0, st>>>(ctx, in, payload, t); }
    rc = check_launch();
    if (rc) return rc;
    {
        Site s(P, MPM_K_P2G, 1, st);
        rc = launch_p2g<R>(P, 0, ctx, tp.perm, payload, tp.active, tp.n_active, tp.grid, nullptr, advect, st);
    }
    if (rc) return rc;
    {
        Site s(P, MPM_K_G2P, model_run_count(P), st);
        for_model_runs(P, [&](auto kind, long long b, long long e) {
            constexpr int K = decltype(kind)::value;
            const int gr = grid_for(e - b, B);
            if (emit)
                g2p_kernel<R, true, K><<<gr, B, 0, st>>>(ctx, tp, in, out, advect, keys, payload, t, b, e);
            else
                g2p_kernel<R, false, K><<<gr, B, 0, st>>>(ctx, tp, in, out, advect, keys, payload, t, b, e);
        });
    }
    return check_launch();
}

template <typename R>
int step_bwd_R(MpmPlan* P, const MpmParticles& in, const void* outC, const MpmCotangents& ob, MpmCotangents& ib,
               double* growth_grad, double* material_grad, int advect, int t, const char* tape, cudaStream_t st) {
    Ctx ctx = make_ctx(P);
    bind_segments(P, ctx, tape);
    Tape<R> tp = make_tape<R>(P, const_cast<char*>(tape));
    const int B = P->tune.particle_block;
    const int g = grid_for(P->n, B);
    double* dbuf = at<double>(P, P->o_dbuf);
    {
        // the forward step's segment table is in the tape: restore the cell marks
        Site s(P, MPM_K_MARK, 1, st);
        const int blocks = (int)std::max<long long>(1, std::min<long long>((P->n + 255) / 256, (long long)P->n_sm * 8));
        remark_cells_kernel<<<blocks, 256, 0, st>>>(ctx, tp.skeys);
    }
    int rc = check_launch();
    if (rc) return rc;
    {
        Site s(P, MPM_K_BWD_P2G, 2, st);
        R* S = at<R>(P, P->o_sums);
        long long cap = P->n;
        int blocks1 = (int)std::min<long long>((P->n + 127) / 128, (long long)P->n_sm * 16);
        blocks1 = std::max(1, blocks1);
        if (P->tune.scatter_oxb == 3 && sizeof(R) == 4)
            cell_sums_adj_kernel<R, 3><<<blocks1, 128, 0, st>>>(ctx, tp.perm, in, ob, S, cap, advect);
        else
            cell_sums_adj_kernel<R, 1><<<blocks1, 128, 0, st>>>(ctx, tp.perm, in, ob, S, cap, advect);
        rc = check_launch();
        if (rc) return rc;
        rc = launch_nodes<R>(P, 1, ctx, tp.active, tp.n_active, nullptr, tp.grid, advect, st);
    }
    if (rc) return rc;
    bool want_dA = growth_grad != nullptr && P->any_growth;
    double* dmat = dbuf + P->n;     // material gradients per slot: mu, then lambda
    {
        Site s(P, MPM_K_BWD_PARTICLE, 1, st);
        const R* oC = static_cast<const R*>(outC);
        double* dAp = want_dA ? dbuf : nullptr;
        if (P->any_external) {
            const long long n = P->n;
            if (material_grad)
                bwd_particle_kernel<R, true, true, -1><<<g, B, 0, st>>>(ctx, tp, in, oC, ob, ib, dAp, dmat, advect,
                                                                        t, 0, n);
            else
                bwd_particle_kernel<R, false, true, -1><<<g, B, 0, st>>>(ctx, tp, in, oC, ob, ib, dAp, nullptr,
                                                                         advect, t, 0, n);
        } else {
            P->launches += model_run_count(P) - 1;
            for_model_runs(P, [&](auto kind, long long b, long long e) {
                constexpr int K = decltype(kind)::value;
                const int gr = grid_for(e - b, B);
                if (material_grad)
                    bwd_particle_kernel<R, true, false, K><<<gr, B, 0, st>>>(ctx, tp, in, oC, ob, ib, dAp, dmat,
                                                                             advect, t, b, e);
                else
                    bwd_particle_kernel<R, false, false, K><<<gr, B, 0, st>>>(ctx, tp, in, oC, ob, ib, dAp, nullptr,
                                                                              advect, t, b, e);
            });
        }
    }
    if (want_dA) {
        Site s(P, MPM_K_REDUCE, 1, st);
        scene_reduce_kernel<<<(int)P->scenes.size(), REDUCE_THREADS, 0, st>>>(ctx, dbuf, growth_grad, 1, 0);
    }
    if (material_grad) {
        Site s(P, MPM_K_REDUCE, 2, st);
        scene_reduce_kernel<<<(int)P->scenes.size(), REDUCE_THREADS, 0, st>>>(ctx, dmat, material_grad, 1, 0, 2);
        scene_reduce_kernel<<<(int)P->scenes.size(), REDUCE_THREADS, 0, st>>>(ctx, dmat + P->n, material_grad + 1,
                                                                             1, 0, 2);
    }
    return check_launch();
}

bool scene_ok(const MpmScene& s) {
    for (int d = 0; d < 3; ++d)
        if (s.shape[d] < 1 || s.shape[d] > 4096) return false;
    if (s.model < 0 || s.model > MPM_MODEL_EXTERNAL) return false;
    if (!(s.dx > 0) || !(s.dt >= 0)) return false;
    if (s.p_end < s.p_begin) return false;
    return true;
}

}  // namespace

extern "C" {

int mpm_version(void) { return 1; }

int mpm_check_violations(int64_t* count, int32_t* first_site, int64_t* first_index, void* stream) {
    if (!count) return MPM_ERR_ARG;
    *count = 0;
#ifdef MPM_CHECK_BOUNDS
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long c = 0;
    long long first[2] = {0, -1};
    const unsigned long long zero = 0;
    if (cudaMemcpyFromSymbolAsync(&c, g_oob_count, sizeof(c), 0, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyFromSymbolAsync(first, g_oob_first, sizeof(first), 0, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyToSymbolAsync(g_oob_count, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return MPM_ERR_CUDA;
    *count = (int64_t)c;
    if (first_site) *first_site = c ? (int32_t)first[0] : 0;
    if (first_index) *first_index = c ? (int64_t)first[1] : -1;
    return MPM_OK;
#else
    (void)stream;
    if (first_site) *first_site = 0;
    if (first_index) *first_index = -1;
    return MPM_ERR_UNSUPPORTED;
#endif
}

int mpm_plan_create(const MpmScene* scenes, int32_t n_scenes, int32_t real_bytes, const MpmTuning* tuning,
                    MpmPlan** out) {
    if (!scenes || n_scenes < 1 || !out || (real_bytes != 4 && real_bytes != 8)) return MPM_ERR_ARG;
    MpmPlan* P = new (std::nothrow) MpmPlan();
    if (!P) return MPM_ERR_ARG;
    P->real_bytes = real_bytes;
    if (tuning) P->tune = *tuning;
    if (P->tune.tile_xy != 8 && P->tune.tile_xy != 16) P->tune.tile_xy = 4;
    if (P->tune.tile_z != 8 && P->tune.tile_z != 16) P->tune.tile_z = 4;
    if (P->tune.scatter_ctas_per_sm <= 0) P->tune.scatter_ctas_per_sm = 1;
    if (P->tune.scatter_oxb != 1 && P->tune.scatter_oxb != 3) P->tune.scatter_oxb = real_bytes == 4 ? 3 : 1;
    if (real_bytes == 8) P->tune.scatter_oxb = 1;
    // the per-particle kernels are compiled for at most 256 threads per block
    if (P->tune.particle_block != 64 && P->tune.particle_block != 128) P->tune.particle_block = 256;
    if (P->tune.fp64_gap_thresh == 0.0f) P->tune.fp64_gap_thresh = 1e-6f;
    const int T = P->tune.tile_xy, TZ = P->tune.tile_z;
    P->TN = T * T * TZ;
    long long cell = 0, tile = 0, pcur = 0, nodes = 0;
    for (int s = 0; s < n_scenes; ++s) {
        const MpmScene& sc = scenes[s];
        if (!scene_ok(sc) || sc.p_begin != pcur) { delete P; return MPM_ERR_ARG; }
        pcur = sc.p_end;
        SceneAux a;
        a.cell_begin = cell;
        // padded cells of the scene, in 64 bits: cell keys are 32-bit, so a
        // scene (or batch) beyond 2^31 cells is refused rather than wrapped
        const long long nc = (long long)(sc.shape[0] + 2) * (sc.shape[1] + 2) * (sc.shape[2] + 2);
        if (nc >= (1LL << 31)) { delete P; return MPM_ERR_ARG; }
        a.ncells = (int)nc;
        a.ntile[0] = (sc.shape[0] + T - 1) / T;
        a.ntile[1] = (sc.shape[1] + T - 1) / T;
        a.ntile[2] = (sc.shape[2] + TZ - 1) / TZ;
        a.tile_begin = tile;
        a.node_begin = nodes;
        nodes += (long long)sc.shape[0] * sc.shape[1] * sc.shape[2];
        cell += (long long)a.ncells + 1;
        tile += (long long)a.ntile[0] * a.ntile[1] * a.ntile[2];
        P->scenes.push_back(sc);
        P->aux.push_back(a);
        if (sc.growth_mode == 1) P->any_growth = true;
        if (sc.model == MPM_MODEL_EXTERNAL) P->any_external = true;
        for (long long p = sc.p_begin; p < sc.p_end; ++p) P->scene_of.push_back(s);
        for (long long k = a.tile_begin; k < tile; ++k) P->tile_scene.push_back(s);
    }
    if (cell >= (1LL << 31) || pcur >= (1LL << 31) || pcur < 1) { delete P; return MPM_ERR_ARG; }
    // runs of consecutive non-empty scenes with one model; grouped when no
    // model has two runs (and no scene supplies its own stress)
    for (const MpmScene& sc : P->scenes) {
        if (sc.p_end == sc.p_begin) continue;
        if (!P->run_kind.empty() && P->run_kind.back() == sc.model) {
            P->run_end.back() = sc.p_end;
        } else {
            P->run_kind.push_back(sc.model);
            P->run_begin.push_back(sc.p_begin);
            P->run_end.push_back(sc.p_end);
        }
    }
    P->runs_grouped = !P->any_external && !P->run_kind.empty();
    for (size_t a = 0; a < P->run_kind.size(); ++a)
        for (size_t b = a + 1; b < P->run_kind.size(); ++b)
            if (P->run_kind[a] == P->run_kind[b]) P->runs_grouped = false;
    P->n = pcur;
    P->n_tiles = tile;
    P->n_keys = cell;
    P->n_nodes = nodes;
    int bits = 1;
    while ((1LL << bits) < cell) ++bits;
    P->key_bits = bits;
    P->passes = (bits + RADIX_BITS - 1) / RADIX_BITS;
    P->nblk_sort = (int)((P->n + SORT_TILE - 1) / SORT_TILE);
    P->active_cap = (int)P->n_tiles;
    if (P->tune.active_tile_cap > 0 && P->tune.active_tile_cap < P->active_cap) P->active_cap = P->tune.active_tile_cap;

    const size_t R = (size_t)real_bytes, n = (size_t)P->n, nt = (size_t)P->n_tiles;
    Layout tl;
    P->t_skeys = tl.take(n * 4);
    P->t_perm = tl.take(n * 4);
    P->t_seg_first = tl.take(n * 4);
    P->t_seg_last = tl.take(n * 4);
    P->t_nseg = tl.take(4);
    P->t_active = tl.take((size_t)P->active_cap * 4);
    P->t_nact = tl.take(4);
    P->t_grid = tl.take((size_t)P->active_cap * P->TN * 4 * R);
    P->tape_bytes = tl.off;

    Layout L;
    P->o_scenes = L.take(sizeof(MpmScene) * P->scenes.size());
    P->o_aux = L.take(sizeof(SceneAux) * P->aux.size());
    P->o_scene_of = L.take(n * 4);
    P->o_tile_scene = L.take(nt * 4);
    P->o_status = L.take(128);
    P->nblk_seg = (int)((P->n + SEGK_TILE - 1) / SEGK_TILE);
    P->o_cell_seg = L.take((size_t)P->n_keys * 4);
    P->o_blk = L.take((size_t)P->nblk_seg * 4);
    P->nblk_tile = (int)((P->n_tiles + TILEK_TILE - 1) / TILEK_TILE);
    P->o_tblk = L.take((size_t)P->nblk_tile * 4);
    P->o_tile_flag = L.take(nt * 4);
    P->o_keys = L.take(n * 4);
    P->o_kalt0 = L.take(n * 4);
    P->o_valt0 = L.take(n * 4);
    P->o_kalt1 = L.take(n * 4);
    P->o_valt1 = L.take(n * 4);
    P->o_hist = L.take((size_t)RADIX * P->nblk_sort * 4);
    P->o_totals = L.take(RADIX * 4);
    P->o_payload = L.take(n * PAYLOAD * R);
    P->o_sums = L.take(27 * n * 4 * R);
    P->o_dense_f = L.take((size_t)P->n_nodes * 4 * R);
    P->o_dense_b = L.take((size_t)P->n_nodes * 4 * R);
    P->o_dbuf = L.take(3 * n * 8);      // dL/dA, dL/dmu, dL/dlambda per slot
    const size_t nw = (n + 31) / 32;
    P->nblk_resort = (int)((nw + RESORT_THREADS - 1) / RESORT_THREADS);
    P->o_mflag = L.take(nw * 32);
    P->o_pflag = L.take(nw * 32);
    P->o_mask = L.take(nw * 4);
    P->o_pmask = L.take(nw * 4);
    P->o_wpre = L.take(nw * 4);
    P->o_rblk = L.take((size_t)P->nblk_resort * 4);
    P->o_pblk = L.take((size_t)P->nblk_resort * 4);
    P->o_mkey = L.take(n * 4);
    P->o_mpart = L.take(n * 4);
    P->o_okey = L.take(n * 4);
    P->o_opart = L.take(n * 4);
    P->o_rint = L.take(8);
    P->nblk_sort1 = (int)((P->n + SORT_THREADS - 1) / SORT_THREADS);
    P->o_hist1 = L.take((size_t)RADIX * P->nblk_sort1 * 4);
    P->o_tape = L.take(P->tape_bytes);
    P->ws_bytes = L.off;
    *out = P;
    return MPM_OK;
}

void mpm_plan_destroy(MpmPlan* plan) {
    if (!plan) return;
    for (cudaEvent_t e : plan->ev0) cudaEventDestroy(e);
    for (cudaEvent_t e : plan->ev1) cudaEventDestroy(e);
    delete plan;
}

int mpm_plan_profile_begin(MpmPlan* P, uint32_t kind_mask, int32_t max_launches) {
    if (!P || max_launches < 1 || (kind_mask >> MPM_K_COUNT) != 0) return MPM_ERR_ARG;
    while ((int)P->ev0.size() < max_launches) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return MPM_ERR_CUDA;
        P->ev0.push_back(a);
        P->ev1.push_back(b);
    }
    P->ev_kind.assign(P->ev0.size(), -1);
    P->prof_mask = kind_mask;
    P->prof_max = max_launches;
    P->prof_n = 0;
    return MPM_OK;
}

int mpm_plan_profile_end(MpmPlan* P, double* ms_per_kind, int32_t* launches_per_kind) {
    if (!P || !ms_per_kind || !launches_per_kind) return MPM_ERR_ARG;
    for (int k = 0; k < MPM_K_COUNT; ++k) {
        ms_per_kind[k] = 0.0;
        launches_per_kind[k] = 0;
    }
    for (int i = 0; i < P->prof_n; ++i) {
        if (cudaEventSynchronize(P->ev1[i]) != cudaSuccess) return MPM_ERR_CUDA;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, P->ev0[i], P->ev1[i]) != cudaSuccess) return MPM_ERR_CUDA;
        int k = P->ev_kind[i];
        if (k >= 0 && k < MPM_K_COUNT) {
            ms_per_kind[k] += ms;
            launches_per_kind[k] += 1;
        }
    }
    P->prof_mask = 0;
    return MPM_OK;
}

int64_t mpm_plan_launch_count(const MpmPlan* P) { return P ? P->launches : -1; }

int mpm_plan_active_tiles(MpmPlan* P, const void* tape, int32_t* n_active, void* stream) {
    if (!P || !P->ws || !n_active) return MPM_ERR_ARG;
    const char* t = tape ? static_cast<const char*>(tape) : P->ws + P->o_tape;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(n_active, t + P->t_nact, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return MPM_ERR_CUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}

int mpm_plan_workspace_bytes(const MpmPlan* P, size_t* bytes) {
    if (!P || !bytes) return MPM_ERR_ARG;
    *bytes = P->ws_bytes;
    return MPM_OK;
}
int mpm_plan_tape_bytes(const MpmPlan* P, size_t* bytes) {
    if (!P || !bytes) return MPM_ERR_ARG;
    *bytes = P->tape_bytes;
    return MPM_OK;
}
int64_t mpm_plan_num_particles(const MpmPlan* P) { return P ? P->n : -1; }

int mpm_plan_bind(MpmPlan* P, void* workspace, void* stream) {
    if (!P || !workspace || (reinterpret_cast<uintptr_t>(workspace) % ALIGN) != 0) return MPM_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    P->ws = static_cast<char*>(workspace);
    // a new workspace holds no emitted keys, records or tile flags: end any chain
    P->chain_valid = false;
    P->tile_flags_pending = false;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MPM_ERR_CUDA;
    cudaDeviceGetAttribute(&P->n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaMemcpyAsync(P->ws + P->o_scenes, P->scenes.data(), sizeof(MpmScene) * P->scenes.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(P->ws + P->o_aux, P->aux.data(), sizeof(SceneAux) * P->aux.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(P->ws + P->o_scene_of, P->scene_of.data(), 4 * P->scene_of.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(P->ws + P->o_tile_scene, P->tile_scene.data(), 4 * P->tile_scene.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(P->ws + P->o_status, 0, 128, st) != cudaSuccess ||
        cudaMemsetAsync(P->ws + P->o_cell_seg, 0, (size_t)P->n_keys * 4, st) != cudaSuccess ||
        cudaMemsetAsync(P->ws + P->o_tile_flag, 0, (size_t)P->n_tiles * 4, st) != cudaSuccess)
        return MPM_ERR_CUDA;
    // the host tables are read by the copies above: wait before returning
    if (cudaStreamSynchronize(st) != cudaSuccess) return MPM_ERR_CUDA;
    return MPM_OK;
}

int mpm_plan_read_status(MpmPlan* P, int32_t* status, void* stream) {
    if (!P || !P->ws || !status) return MPM_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(status, P->ws + P->o_status, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return MPM_ERR_CUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}

int mpm_plan_read_fp64_fallbacks(MpmPlan* P, int64_t* count, void* stream) {
    if (!P || !P->ws || !count) return MPM_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(count, P->ws + P->o_status + 64, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return MPM_ERR_CUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}

int mpm_plan_update_scenes(MpmPlan* P, const MpmScene* scenes, int32_t n_scenes, void* stream) {
    if (!P || !P->ws || !scenes || n_scenes != (int)P->scenes.size()) return MPM_ERR_ARG;
    for (int s = 0; s < n_scenes; ++s) {
        const MpmScene& a = P->scenes[s];
        const MpmScene& b = scenes[s];
        if (!scene_ok(b) || a.p_begin != b.p_begin || a.p_end != b.p_end || a.model != b.model ||
            a.growth_mode != b.growth_mode || a.shape[0] != b.shape[0] || a.shape[1] != b.shape[1] ||
            a.shape[2] != b.shape[2])
            return MPM_ERR_ARG;
    }
    for (int s = 0; s < n_scenes; ++s) P->scenes[s] = scenes[s];
    P->chain_valid = false;     // records formed with the old parameters
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(P->ws + P->o_scenes, P->scenes.data(), sizeof(MpmScene) * P->scenes.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return MPM_ERR_CUDA;
    return MPM_OK;
}

int mpm_plan_set_external_stress(MpmPlan* P, const void* tau, void* tau_bar) {
    if (!P) return MPM_ERR_ARG;
    P->ext_tau = tau;
    P->ext_tau_bar = tau_bar;
    P->chain_valid = false;
    return MPM_OK;
}

int mpm_plan_set_particle_mass(MpmPlan* P, const void* mass, const void* vol0) {
    if (!P) return MPM_ERR_ARG;
    P->pmass_p = mass;
    P->vol0_p = vol0;
    P->chain_valid = false;     // records formed with the old masses
    return MPM_OK;
}

int mpm_plan_set_growth_field(MpmPlan* P, const void* phi) {
    if (!P) return MPM_ERR_ARG;
    P->phi = phi;
    P->chain_valid = false;     // records formed with the old growth field
    return MPM_OK;
}

int mpm_step_fwd_chain(MpmPlan* P, const MpmParticles* in, MpmParticles* out, int32_t advect, int32_t step_index,
                       void* tape, int32_t flags, void* stream) {
    if (!P || !P->ws || !in || !out || !in->x || !in->v || !in->C || !in->F || !out->x || !out->v || !out->C ||
        !out->F || in->x == out->x || in->F == out->F || (flags & ~(MPM_FWD_CHAINED | MPM_FWD_EMIT)) != 0)
        return MPM_ERR_ARG;
    for (const MpmScene& s : P->scenes)
        if (s.growth_mode == 0 && !in->Fg) return MPM_ERR_ARG;
    char* tp = tape ? static_cast<char*>(tape) : P->ws + P->o_tape;
    if (reinterpret_cast<uintptr_t>(tp) % ALIGN) return MPM_ERR_ARG;
    // external stress: supplied per call, so no chaining (the chain would
    // evaluate the next step's stress inside G2P)
    if (P->any_external && (!P->ext_tau || flags != 0)) return MPM_ERR_ARG;
    // a chained step must continue the last emitting call on this plan
    if (flags & MPM_FWD_CHAINED) {
        if (!P->chain_valid || P->chain_t != step_index ||
            std::memcmp(&P->chain_state, in, sizeof(MpmParticles)) != 0)
            return MPM_ERR_ARG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the active-tile flags of the next step are set where its keys are formed
    // (bin or an emitting G2P); an emitted state that is not continued leaves
    // its flags behind, so they are cleared before binning another state
    if (P->tile_flags_pending && !(flags & MPM_FWD_CHAINED) &&
        cudaMemsetAsync(P->ws + P->o_tile_flag, 0, (size_t)P->n_tiles * 4, st) != cudaSuccess)
        return MPM_ERR_CUDA;
    P->chain_valid = false;
    P->tile_flags_pending = false;
    int rc = P->real_bytes == 4 ? step_fwd_R<float>(P, *in, *out, advect, step_index, tp, flags, st)
                                : step_fwd_R<double>(P, *in, *out, advect, step_index, tp, flags, st);
    if (rc == MPM_OK && (flags & MPM_FWD_EMIT)) {
        P->tile_flags_pending = true;
        P->chain_valid = true;
        P->chain_t = step_index + 1;
        P->chain_state = *out;
        P->chain_tape = tp;
    }
    return rc;
}

int mpm_step_fwd(MpmPlan* P, const MpmParticles* in, MpmParticles* out, int32_t advect, int32_t step_index,
                 void* tape, void* stream) {
    return mpm_step_fwd_chain(P, in, out, advect, step_index, tape, 0, stream);
}

int mpm_step_bwd_params(MpmPlan* P, const MpmParticles* in, const void* out_C, const MpmCotangents* out_bar,
                        MpmCotangents* in_bar, double* growth_grad, double* material_grad, int32_t advect,
                        int32_t step_index, const void* tape, void* stream) {
    if (!P || !P->ws || !in || !out_C || !out_bar || !in_bar || !tape) return MPM_ERR_ARG;
    if (!out_bar->x || !out_bar->v || !out_bar->C || !out_bar->F || !in_bar->x || !in_bar->v || !in_bar->C ||
        !in_bar->F)
        return MPM_ERR_ARG;
    if (in_bar->x == out_bar->x || in_bar->v == out_bar->v || in_bar->C == out_bar->C || in_bar->F == out_bar->F)
        return MPM_ERR_ARG;
    for (const MpmScene& s : P->scenes)
        if (s.growth_mode == 0 && !in->Fg) return MPM_ERR_ARG;
    if (P->any_external && (!P->ext_tau || !P->ext_tau_bar)) return MPM_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(tape) % ALIGN) return MPM_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return P->real_bytes == 4
               ? step_bwd_R<float>(P, *in, out_C, *out_bar, *in_bar, growth_grad, material_grad, advect, step_index,
                                   static_cast<const char*>(tape), st)
               : step_bwd_R<double>(P, *in, out_C, *out_bar, *in_bar, growth_grad, material_grad, advect,
                                    step_index, static_cast<const char*>(tape), st);
}

int mpm_step_bwd(MpmPlan* P, const MpmParticles* in, const void* out_C, const MpmCotangents* out_bar,
                 MpmCotangents* in_bar, double* growth_grad, int32_t advect, int32_t step_index, const void* tape,
                 void* stream) {
    return mpm_step_bwd_params(P, in, out_C, out_bar, in_bar, growth_grad, nullptr, advect, step_index, tape,
                               stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Whole trajectories (integrate.py:15-28 rollout / rollout_vjp, with the
// per-step caches replaced by checkpoint-every-k recomputation).  The caller's
// rollout workspace holds, 256-byte aligned and in this order:
//   ckpt[n_seg]       state at the start of every segment   (recompute only)
//   seg[k + 1]        the states of one segment
//   scratch[2]        intermediate forward states           (recompute only)
//   bars[2]           cotangent ping-pong of the reverse sweep
//   tapes[k]          the tapes of one segment
// Every slab is (24, n) in the plan's real type: rows x(3) v(3) C(9) F(9).
// ---------------------------------------------------------------------------
namespace {

struct RolloutLayout {
    int T = 0, k = 1, n_seg = 0;
    bool recompute = false;
    size_t slab = 0, tape = 0;
    size_t o_ckpt = 0, o_seg = 0, o_scr = 0, o_bar = 0, o_tape = 0, total = 0;
};

bool rollout_layout(const MpmPlan* P, int n_steps, int ckpt_every, RolloutLayout& L) {
    if (n_steps < 0 || ckpt_every < 0) return false;
    L.T = n_steps;
    L.k = ckpt_every > 0 ? std::min(ckpt_every, std::max(n_steps, 1)) : std::max(n_steps, 1);
    L.n_seg = (n_steps + L.k - 1) / L.k;
    L.recompute = L.k < n_steps;
    L.slab = align_up((size_t)24 * (size_t)P->n * (size_t)P->real_bytes);
    L.tape = align_up(P->tape_bytes);
    Layout lay;
    L.o_ckpt = lay.off;
    if (L.recompute) lay.off += L.slab * L.n_seg;
    L.o_seg = lay.off;
    lay.off += L.slab * (L.k + 1);
    L.o_scr = lay.off;
    if (L.recompute) lay.off += L.slab * 2;
    L.o_bar = lay.off;
    lay.off += L.slab * 2;
    L.o_tape = lay.off;
    lay.off += L.tape * L.k;
    L.total = n_steps == 0 ? 0 : lay.off;
    return true;
}

MpmParticles slab_state(const MpmPlan* P, const void* slab, const void* Fg) {
    const size_t row = (size_t)P->n * (size_t)P->real_bytes;
    char* b = static_cast<char*>(const_cast<void*>(slab));
    MpmParticles s{};
    s.x = b;
    s.v = b + 3 * row;
    s.C = b + 6 * row;
    s.F = b + 15 * row;
    s.Fg = const_cast<void*>(Fg);
    s.sp3 = s.sp9 = 1;
    s.sc3 = s.sc9 = P->n;
    return s;
}

MpmCotangents slab_cot(const MpmPlan* P, const void* slab, double* Fg_bar) {
    MpmParticles v = slab_state(P, slab, nullptr);
    MpmCotangents c{};
    c.x = v.x;
    c.v = v.v;
    c.C = v.C;
    c.F = v.F;
    c.Fg = Fg_bar;
    c.sp3 = c.sp9 = 1;
    c.sc3 = c.sc9 = P->n;
    return c;
}

int rollout_args(const MpmPlan* P, const void* Fg, const void* ws, const void* a, const void* b) {
    if (!P || !P->ws || !a || !b || a == b) return MPM_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(ws) % ALIGN) return MPM_ERR_ARG;
    if (P->any_external) return MPM_ERR_UNSUPPORTED;    // the stress is a per-step callback
    for (const MpmScene& s : P->scenes)
        if (s.growth_mode == 0 && !Fg) return MPM_ERR_ARG;
    return MPM_OK;
}

inline int async_copy(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st) == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}

// the chain flags of step t in a run of steps [t0, t1)
inline int chain_flags(int t, int t0, int t1) {
    return (t > t0 ? MPM_FWD_CHAINED : 0) | (t + 1 < t1 ? MPM_FWD_EMIT : 0);
}

}  // namespace

extern "C" {

int mpm_rollout_workspace_bytes(const MpmPlan* P, int32_t n_steps, int32_t ckpt_every, size_t* bytes) {
    if (!P || !bytes) return MPM_ERR_ARG;
    RolloutLayout L;
    if (!rollout_layout(P, n_steps, ckpt_every, L)) return MPM_ERR_ARG;
    *bytes = L.total;
    return MPM_OK;
}

int mpm_rollout_fwd(MpmPlan* P, const void* state0, const void* Fg, int32_t n_steps, int32_t ckpt_every,
                    int32_t advect, void* rollout_ws, void* final_state, void* stream) {
    int rc = rollout_args(P, Fg, rollout_ws, state0, final_state);
    if (rc) return rc;
    RolloutLayout L;
    if (!rollout_layout(P, n_steps, ckpt_every, L) || (L.total && !rollout_ws)) return MPM_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* w = static_cast<char*>(rollout_ws);
    const size_t sb = (size_t)24 * (size_t)P->n * (size_t)P->real_bytes;
    if (L.T == 0) return async_copy(final_state, state0, sb, st);
    if (!L.recompute) {
        // one segment: every state and tape is kept for the reverse sweep
        if ((rc = async_copy(w + L.o_seg, state0, sb, st))) return rc;
        for (int t = 0; t < L.T; ++t) {
            MpmParticles a = slab_state(P, w + L.o_seg + L.slab * t, Fg);
            MpmParticles b = slab_state(P, w + L.o_seg + L.slab * (t + 1), Fg);
            rc = mpm_step_fwd_chain(P, &a, &b, advect, t, w + L.o_tape + L.tape * t, chain_flags(t, 0, L.T), st);
            if (rc) return rc;
        }
        return async_copy(final_state, w + L.o_seg + L.slab * L.T, sb, st);
    }
    // checkpoints only; the intermediate states alternate between two scratch slabs
    if ((rc = async_copy(w + L.o_ckpt, state0, sb, st))) return rc;
    const char* cur = w + L.o_ckpt;
    for (int t = 0; t < L.T; ++t) {
        char* nxt;
        if (t + 1 == L.T)
            nxt = static_cast<char*>(final_state);
        else if ((t + 1) % L.k == 0)
            nxt = w + L.o_ckpt + L.slab * ((t + 1) / L.k);
        else
            nxt = w + L.o_scr + L.slab * ((cur == w + L.o_scr + L.slab * (t % 2)) ? (t + 1) % 2 : t % 2);
        MpmParticles a = slab_state(P, cur, Fg), b = slab_state(P, nxt, Fg);
        rc = mpm_step_fwd_chain(P, &a, &b, advect, t, nullptr, chain_flags(t, 0, L.T), st);
        if (rc) return rc;
        cur = nxt;
    }
    return MPM_OK;
}

int mpm_rollout_bwd(MpmPlan* P, const void* Fg, const void* final_bar, int32_t n_steps, int32_t ckpt_every,
                    int32_t advect, void* rollout_ws, void* state0_bar, double* Fg_bar, double* growth_grad,
                    double* material_grad, void* stream) {
    int rc = rollout_args(P, Fg, rollout_ws, final_bar, state0_bar);
    if (rc) return rc;
    RolloutLayout L;
    if (!rollout_layout(P, n_steps, ckpt_every, L) || (L.total && !rollout_ws)) return MPM_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t S = P->scenes.size();
    if ((Fg_bar && cudaMemsetAsync(Fg_bar, 0, (size_t)9 * P->n * sizeof(double), st) != cudaSuccess) ||
        (growth_grad && cudaMemsetAsync(growth_grad, 0, S * sizeof(double), st) != cudaSuccess) ||
        (material_grad && cudaMemsetAsync(material_grad, 0, 2 * S * sizeof(double), st) != cudaSuccess))
        return MPM_ERR_CUDA;
    char* w = static_cast<char*>(rollout_ws);
    const size_t sb = (size_t)24 * (size_t)P->n * (size_t)P->real_bytes;
    if (L.T == 0) return async_copy(state0_bar, final_bar, sb, st);
    const void* cur = final_bar;
    int flip = 0;
    for (int seg = L.n_seg - 1; seg >= 0; --seg) {
        const int t0 = seg * L.k, t1 = std::min(L.T, t0 + L.k);
        if (L.recompute) {
            // the segment's states and tapes again, from its checkpoint
            if ((rc = async_copy(w + L.o_seg, w + L.o_ckpt + L.slab * seg, sb, st))) return rc;
            for (int t = t0; t < t1; ++t) {
                const int j = t - t0;
                MpmParticles a = slab_state(P, w + L.o_seg + L.slab * j, Fg);
                MpmParticles b = slab_state(P, w + L.o_seg + L.slab * (j + 1), Fg);
                rc = mpm_step_fwd_chain(P, &a, &b, advect, t, w + L.o_tape + L.tape * j, chain_flags(t, t0, t1),
                                        st);
                if (rc) return rc;
            }
        }
        for (int t = t1 - 1; t >= t0; --t) {
            const int j = t - t0;
            void* nxt = t == 0 ? state0_bar : static_cast<void*>(w + L.o_bar + L.slab * flip);
            flip ^= 1;
            MpmParticles a = slab_state(P, w + L.o_seg + L.slab * j, Fg);
            const char* outC = w + L.o_seg + L.slab * (j + 1) + (size_t)6 * P->n * P->real_bytes;
            MpmCotangents ob = slab_cot(P, cur, Fg_bar), ib = slab_cot(P, nxt, Fg_bar);
            rc = mpm_step_bwd_params(P, &a, outC, &ob, &ib, growth_grad, material_grad, advect, t,
                                     w + L.o_tape + L.tape * j, st);
            if (rc) return rc;
            cur = nxt;
        }
    }
    return MPM_OK;
}

int mpm_stress(const MpmScene* scene, int32_t real_bytes, int64_t n, const void* F, const void* Fg, const void* C,
               void* tau, void* stream) {
    if (!scene || n < 0 || !F || !Fg || !tau || (real_bytes != 4 && real_bytes != 8)) return MPM_ERR_ARG;
    if (scene->model == MPM_MODEL_EXTERNAL) return MPM_ERR_UNSUPPORTED;
    if (n == 0) return MPM_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int g = grid_for(n, 256);
    if (real_bytes == 4)
        stress_kernel<float><<<g, 256, 0, st>>>(*scene, n, (const float*)F, (const float*)Fg, (const float*)C,
                                                (float*)tau, 1e-6f);
    else
        stress_kernel<double><<<g, 256, 0, st>>>(*scene, n, (const double*)F, (const double*)Fg,
                                                 (const double*)C, (double*)tau, 0.0f);
    return check_launch();
}

int mpm_stress_vjp(const MpmScene* scene, int32_t real_bytes, int64_t n, const void* F, const void* Fg,
                   const void* C, const void* tau_bar, void* F_bar, void* Fg_bar, void* C_bar, void* stream) {
    if (!scene || n < 0 || !F || !Fg || !tau_bar || !F_bar || !Fg_bar || (real_bytes != 4 && real_bytes != 8))
        return MPM_ERR_ARG;
    if (scene->model == MPM_MODEL_EXTERNAL) return MPM_ERR_UNSUPPORTED;
    if (n == 0) return MPM_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int g = grid_for(n, 256);
    if (real_bytes == 4)
        stress_vjp_kernel<float><<<g, 256, 0, st>>>(*scene, n, (const float*)F, (const float*)Fg, (const float*)C,
                                                    (const float*)tau_bar, (float*)F_bar, (float*)Fg_bar,
                                                    (float*)C_bar, 1e-6f);
    else
        stress_vjp_kernel<double><<<g, 256, 0, st>>>(*scene, n, (const double*)F, (const double*)Fg,
                                                     (const double*)C, (const double*)tau_bar, (double*)F_bar,
                                                     (double*)Fg_bar, (double*)C_bar, 0.0f);
    return check_launch();
}

int mpm_bin_keys(const MpmScene* scene, int32_t real_bytes, int64_t n, const void* x, int32_t* keys, void* stream) {
    if (!scene || n < 0 || !x || !keys || (real_bytes != 4 && real_bytes != 8)) return MPM_ERR_ARG;
    // the keys are int32: the padded cells (and the "outside" key after them) must fit
    if (!scene_ok(*scene) ||
        (long long)(scene->shape[0] + 2) * (scene->shape[1] + 2) * (scene->shape[2] + 2) >= (1LL << 31))
        return MPM_ERR_ARG;
    if (n == 0) return MPM_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int g = grid_for(n, 256);
    if (real_bytes == 4)
        bin_keys_single<float><<<g, 256, 0, st>>>(*scene, n, (const float*)x, keys);
    else
        bin_keys_single<double><<<g, 256, 0, st>>>(*scene, n, (const double*)x, keys);
    return check_launch();
}

int mpm_loss_detF(MpmPlan* P, const void* F, int64_t sp9, int64_t sc9, double* loss, void* F_bar, void* stream) {
    if (!P || !P->ws || !F || !loss) return MPM_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Ctx ctx = make_ctx(P);
    double* dbuf = at<double>(P, P->o_dbuf);
    int g = grid_for(P->n, 256);
    Site site(P, MPM_K_REDUCE, 2, st);
    if (P->real_bytes == 4)
        loss_detF_kernel<float><<<g, 256, 0, st>>>(ctx, (const float*)F, sp9, sc9, dbuf, (float*)F_bar);
    else
        loss_detF_kernel<double><<<g, 256, 0, st>>>(ctx, (const double*)F, sp9, sc9, dbuf, (double*)F_bar);
    scene_reduce_kernel<<<(int)P->scenes.size(), REDUCE_THREADS, 0, st>>>(ctx, dbuf, loss, 0, 0);
    return check_launch();
}

int mpm_loss_mse(MpmPlan* P, const void* x, int64_t sp3, int64_t sc3, const void* x_obs, double* loss, void* x_bar,
                 void* stream) {
    if (!P || !P->ws || !x || !x_obs || !loss) return MPM_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Ctx ctx = make_ctx(P);
    double* dbuf = at<double>(P, P->o_dbuf);
    int g = grid_for(P->n, 256);
    Site site(P, MPM_K_REDUCE, 2, st);
    if (P->real_bytes == 4)
        loss_mse_kernel<float><<<g, 256, 0, st>>>(ctx, (const float*)x, sp3, sc3, (const float*)x_obs, dbuf,
                                                  (float*)x_bar);
    else
        loss_mse_kernel<double><<<g, 256, 0, st>>>(ctx, (const double*)x, sp3, sc3, (const double*)x_obs, dbuf,
                                                   (double*)x_bar);
    scene_reduce_kernel<<<(int)P->scenes.size(), REDUCE_THREADS, 0, st>>>(ctx, dbuf, loss, 0, 1);
    return check_launch();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Forward step without device allocation (mpm_step_fwd_noalloc).  The whole
// workspace of one single-scene forward step is carved out of one fixed
// file-scope device array; the launch sequence is the same step_fwd_R that
// mpm_step_fwd runs.
// ---------------------------------------------------------------------------
namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[MPM_NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
struct NoallocDevice {
    std::mutex mu;
    unsigned long long ctx_id = 0;   // driver id of the context the address belongs to (0: none yet)
    void* ptr = nullptr;
    int n_sm = 0;
};
NoallocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];

// Unique id of the calling thread's current driver context (0 when none is
// current yet).  A device reset destroys the context and the module loaded in
// it; the next context has a new id, so the scratch address is looked up
// again.  The two driver calls are fetched through the runtime once, so the
// library does not link the driver library itself.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
int current_context_id(unsigned long long* id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
    });
    if (!get_current || !get_id) return MPM_ERR_CUDA;
    CUcontext c = nullptr;
    *id = 0;
    if (get_current(&c) != CUDA_SUCCESS) return MPM_ERR_CUDA;
    if (c && get_id(c, id) != CUDA_SUCCESS) return MPM_ERR_CUDA;
    return MPM_OK;
}

// Device address of the scratch array in the current device's context.  The
// lookup (cudaGetSymbolAddress) runs with that device current, once per
// context: on the first call on a device, and again on the first call after a
// device reset.
int noalloc_scratch(void** out, int* n_sm) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MPM_ERR_CUDA;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return MPM_ERR_UNSUPPORTED;
    NoallocDevice& d = g_noalloc_dev[dev];
    std::lock_guard<std::mutex> lock(d.mu);
    unsigned long long id = 0;
    if (current_context_id(&id)) return MPM_ERR_CUDA;
    if (id == 0 || id != d.ctx_id || !d.ptr) {
        void* p = nullptr;
        // creates the device's context when none is current yet
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return MPM_ERR_CUDA;
        int sm = 0;
        if (cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return MPM_ERR_CUDA;
        if (current_context_id(&id) || id == 0) return MPM_ERR_CUDA;
        d.ptr = p;
        d.n_sm = sm;
        d.ctx_id = id;
    }
    *out = d.ptr;
    *n_sm = d.n_sm;
    return MPM_OK;
}

// Forward-only workspace layout of one scene (the fields step_fwd_R reads),
// on a plan object that owns no heap memory.
bool noalloc_layout(MpmPlan& P, const MpmScene& sc, int real_bytes, SceneAux& a) {
    P.real_bytes = real_bytes;
    P.tune.tile_xy = 4;
    P.tune.tile_z = 4;
    P.tune.scatter_ctas_per_sm = 1;
    P.tune.scatter_oxb = real_bytes == 4 ? 3 : 1;
    P.tune.particle_block = 256;
    P.tune.fp64_gap_thresh = 1e-6f;
    const int T = P.tune.tile_xy, TZ = P.tune.tile_z;
    P.TN = T * T * TZ;
    a.cell_begin = 0;
    a.tile_begin = 0;
    a.node_begin = 0;
    const long long nc = (long long)(sc.shape[0] + 2) * (sc.shape[1] + 2) * (sc.shape[2] + 2);
    if (nc >= (1LL << 31)) return false;     // beyond the 32-bit keys (and far beyond the scratch)
    a.ncells = (int)nc;
    a.ntile[0] = (sc.shape[0] + T - 1) / T;
    a.ntile[1] = (sc.shape[1] + T - 1) / T;
    a.ntile[2] = (sc.shape[2] + TZ - 1) / TZ;
    P.n = sc.p_end;
    P.n_tiles = (long long)a.ntile[0] * a.ntile[1] * a.ntile[2];
    P.n_keys = (long long)a.ncells + 1;
    P.n_nodes = (long long)sc.shape[0] * sc.shape[1] * sc.shape[2];
    P.any_growth = sc.growth_mode == 1;
    int bits = 1;
    while ((1LL << bits) < P.n_keys) ++bits;
    P.key_bits = bits;
    P.passes = (bits + RADIX_BITS - 1) / RADIX_BITS;
    P.nblk_sort = (int)((P.n + SORT_TILE - 1) / SORT_TILE);
    P.nblk_seg = (int)((P.n + SEGK_TILE - 1) / SEGK_TILE);
    P.active_cap = (int)P.n_tiles;
    const size_t R = (size_t)real_bytes, n = (size_t)P.n, nt = (size_t)P.n_tiles;
    Layout tl;
    P.t_skeys = tl.take(n * 4);
    P.t_perm = tl.take(n * 4);
    P.t_seg_first = tl.take(n * 4);
    P.t_seg_last = tl.take(n * 4);
    P.t_nseg = tl.take(4);
    P.t_active = tl.take((size_t)P.active_cap * 4);
    P.t_nact = tl.take(4);
    P.t_grid = tl.take((size_t)P.active_cap * P.TN * 4 * R);
    P.tape_bytes = tl.off;
    Layout L;
    P.o_scenes = L.take(sizeof(MpmScene));
    P.o_aux = L.take(sizeof(SceneAux));
    P.o_scene_of = L.take(n * 4);
    P.o_tile_scene = L.take(nt * 4);
    P.o_status = L.take(128);
    P.o_cell_seg = L.take((size_t)P.n_keys * 4);
    P.o_blk = L.take((size_t)P.nblk_seg * 4);
    P.nblk_tile = (int)((P.n_tiles + TILEK_TILE - 1) / TILEK_TILE);
    P.o_tblk = L.take((size_t)P.nblk_tile * 4);
    P.o_tile_flag = L.take(nt * 4);
    P.o_keys = L.take(n * 4);
    P.o_kalt0 = L.take(n * 4);
    P.o_valt0 = L.take(n * 4);
    P.o_kalt1 = L.take(n * 4);
    P.o_valt1 = L.take(n * 4);
    P.o_hist = L.take((size_t)RADIX * P.nblk_sort * 4);
    P.o_totals = L.take(RADIX * 4);
    P.o_payload = L.take(n * PAYLOAD * R);
    P.o_sums = L.take(27 * n * 4 * R);
    P.o_dense_f = L.take((size_t)P.n_nodes * 4 * R);
    P.o_dense_b = P.o_dense_f;      // the forward step writes no reverse records
    P.o_tape = L.take(P.tape_bytes);
    P.ws_bytes = L.off;
    return P.ws_bytes <= (size_t)MPM_NOALLOC_SCRATCH_BYTES;
}

}  // namespace

extern "C" int mpm_step_fwd_noalloc(const MpmScene* scene, int32_t real_bytes, const MpmParticles* in,
                                    MpmParticles* out, int32_t advect, int32_t step_index, int32_t* status,
                                    void* stream) {
    if (!scene || !in || !out || (real_bytes != 4 && real_bytes != 8)) return MPM_ERR_ARG;
    if (!scene_ok(*scene) || scene->p_begin != 0 || scene->p_end < 1 || scene->p_end >= (1LL << 31))
        return MPM_ERR_ARG;
    if (scene->model == MPM_MODEL_EXTERNAL) return MPM_ERR_UNSUPPORTED;
    if (!in->x || !in->v || !in->C || !in->F || !out->x || !out->v || !out->C || !out->F || in->x == out->x ||
        in->F == out->F || (scene->growth_mode == 0 && !in->Fg))
        return MPM_ERR_ARG;
    MpmPlan P;                 // owns no heap memory: its vectors stay empty
    SceneAux aux;
    if (!noalloc_layout(P, *scene, real_bytes, aux)) return MPM_ERR_TOO_LARGE;
    void* ws = nullptr;
    int rc = noalloc_scratch(&ws, &P.n_sm);
    if (rc) return rc;
    P.ws = static_cast<char*>(ws);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the scene tables, and everything the step expects to start at zero
    if (cudaMemcpyAsync(P.ws + P.o_scenes, scene, sizeof(MpmScene), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(P.ws + P.o_aux, &aux, sizeof(SceneAux), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(P.ws + P.o_scene_of, 0, (size_t)P.n * 4, st) != cudaSuccess ||
        cudaMemsetAsync(P.ws + P.o_tile_scene, 0, (size_t)P.n_tiles * 4, st) != cudaSuccess ||
        cudaMemsetAsync(P.ws + P.o_status, 0, 128, st) != cudaSuccess ||
        cudaMemsetAsync(P.ws + P.o_cell_seg, 0, (size_t)P.n_keys * 4, st) != cudaSuccess ||
        cudaMemsetAsync(P.ws + P.o_tile_flag, 0, (size_t)P.n_tiles * 4, st) != cudaSuccess)
        return MPM_ERR_CUDA;
    rc = real_bytes == 4 ? step_fwd_R<float>(&P, *in, *out, advect, step_index, P.ws + P.o_tape, 0, st)
                         : step_fwd_R<double>(&P, *in, *out, advect, step_index, P.ws + P.o_tape, 0, st);
    if (rc) return rc;
    if (status) {
        if (cudaMemcpyAsync(status, P.ws + P.o_status, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return MPM_ERR_CUDA;
    }
    return MPM_OK;
}
