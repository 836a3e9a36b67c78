// Device-side building blocks shared by every kernel of the growth step:
// exact-rounding helpers for the binning arithmetic, register-resident 3x3
// matrix algebra (row-major, templated on float/double), the scene-table
// side structures and the workspace context passed by value to kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "../../include/morphompm_b200.h"

namespace mpm {

// ---------------------------------------------------------------------------
// Bounds-checked build (compiled with -DMPM_CHECK_BOUNDS): every index the
// kernels compute into the node, sum, segment, tile and sort arrays is checked
// against the array's size before the access.  An index out of range is
// counted, the first one is recorded (site id, index), and the access is
// skipped, so a wrong index shows up as a count instead of a memory fault.
// The release build compiles the checks away (MPM_INB is the constant true).
// Site ids: 1 tile flag, 2 cell mark, 3 segment table write, 4 cell-sum
// store, 5 cell-sum load, 6 cell mark read, 7 dense node record, 8 tape grid
// record, 9 sort permutation value, 10 sort scatter, 11 segment range read.
// ---------------------------------------------------------------------------
#ifdef MPM_CHECK_BOUNDS
__device__ unsigned long long g_oob_count;
__device__ long long g_oob_first[2];
__device__ __forceinline__ bool in_bounds(long long i, long long n, int site) {
    if (i >= 0 && i < n) return true;
    if (atomicAdd(&g_oob_count, 1ull) == 0ull) {
        g_oob_first[0] = site;
        g_oob_first[1] = i;
    }
    return false;
}
#define MPM_INB(i, n, site) ::mpm::in_bounds((long long)(i), (long long)(n), (site))
#else
#define MPM_INB(i, n, site) true
#endif

// Node tiles are tile_xy x tile_xy x tile_z nodes (z fastest inside a tile).

// Per-scene data derived on the host from MpmScene.
struct SceneAux {
    long long cell_begin;   // first padded cell key of the scene
    long long tile_begin;   // first node tile of the scene
    long long node_begin;   // first node of the scene in the dense node scratch
    int ntile[3];           // tiles per axis
    int ncells;             // (shape+2)^3 padded cells; key cell_begin+ncells = "outside"
};

// Workspace pointers and sizes, passed by value to every kernel.
struct Ctx {
    const MpmScene* scenes;
    const SceneAux* aux;
    const int* scene_of;         // scene of each particle slot (same ranges sorted or not)
    const int* tile_scene;       // scene of each tile
    int* status;                 // device status word (MPM_* bits)
    unsigned long long* fallbacks;  // FP32 Hencky evaluations redone in FP64
    int* cell_seg;               // dense over padded cells: 1 + segment id of an occupied cell, 0 if empty
    int* seg_first;              // per segment (occupied cell, sorted order): first sorted slot
    int* seg_last;               // one past its last slot
    int* n_seg;                  // number of segments
    unsigned* blk_count;         // per-block segment counts of the segment scan
    int* tile_flag;              // 1 if the tile receives mass this step
    const void* phi;             // growth field phi_p (growth_mode 1), may be null
    const void* pmass_p;         // per-particle mass, may be null (scene pmass)
    const void* vol0_p;          // per-particle reference volume, may be null (scene vol0)
    const void* ext_tau;         // MPM_MODEL_EXTERNAL scenes: Kirchhoff stress per particle (n x 9)
    void* ext_tau_bar;           // and its cotangent, written by the reverse step (n x 9)
    void* dense_f;               // dense node scratch, forward record (m, v[3]) per node
    void* dense_b;               // dense node scratch, reverse record (gm_b, gmom_b[3]) per node
    unsigned char* mover_flag;   // emitting G2P: per sorted slot, its particle changed cell (may be null)
    unsigned char* mover_pflag;  // and the same flag per particle
    long long n;
    long long n_tiles;
    long long n_keys;            // padded cells of all scenes (cell_seg entries)
    long long n_nodes;           // nodes of all scenes (dense_f / dense_b records)
    long long grid_nodes;        // node records of a tape's grid (active_cap x nodes per tile)
    int n_scenes;
    int tile_xy;
    int tile_z;
    int tile_xy_shift;           // log2 of the tile edges (tiles are 4, 8 or 16 nodes)
    int tile_z_shift;
    int active_cap;              // capacity of a tape's active-tile list
    float gap_thresh;            // FP32 Hencky FP64-fallback threshold (relative sv gap)
};

// Pointers into one step's tape (or into the workspace scratch when no tape is
// recorded).  Grid records are stored compactly per active tile.
template <typename R>
struct Tape {
    unsigned* skeys;    // sorted cell keys
    unsigned* perm;     // sorted slot -> particle index
    int* active;        // active tile ids
    int* n_active;      // number of active tiles
    R* grid;            // forward node records (m, v0, v1, v2) per slot*TN + local
};

// ---------------------------------------------------------------------------
// scalar helpers
// ---------------------------------------------------------------------------
template <typename R> struct Num;
template <> struct Num<float> {
    static __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
    static constexpr float eps = 1.1920929e-7f;
};
template <> struct Num<double> {
    static __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
    static constexpr double eps = 2.220446049250313e-16;
};

__device__ __forceinline__ float  d_log(float a)  { return logf(a); }
__device__ __forceinline__ double d_log(double a) { return log(a); }
__device__ __forceinline__ float  d_log1p(float a)  { return log1pf(a); }
__device__ __forceinline__ double d_log1p(double a) { return log1p(a); }
__device__ __forceinline__ float  d_exp(float a)  { return expf(a); }
__device__ __forceinline__ double d_exp(double a) { return exp(a); }
__device__ __forceinline__ float  d_sqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double d_sqrt(double a) { return sqrt(a); }
__device__ __forceinline__ float  d_pow(float a, float b)  { return powf(a, b); }
__device__ __forceinline__ double d_pow(double a, double b) { return pow(a, b); }
__device__ __forceinline__ float  d_floor(float a)  { return floorf(a); }
__device__ __forceinline__ double d_floor(double a) { return floor(a); }
__device__ __forceinline__ float  d_abs(float a)  { return fabsf(a); }
__device__ __forceinline__ double d_abs(double a) { return fabs(a); }

// ---------------------------------------------------------------------------
// strided particle-field access
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void ld3(const void* base, long long p, long long sp, long long sc, R o[3]) {
    const R* b = static_cast<const R*>(base) + p * sp;
#pragma unroll
    for (int c = 0; c < 3; ++c) o[c] = b[c * sc];
}
template <typename R>
__device__ __forceinline__ void ld9(const void* base, long long p, long long sp, long long sc, R o[9]) {
    const R* b = static_cast<const R*>(base) + p * sp;
#pragma unroll
    for (int c = 0; c < 9; ++c) o[c] = b[c * sc];
}
template <typename R>
__device__ __forceinline__ void st3(void* base, long long p, long long sp, long long sc, const R o[3]) {
    R* b = static_cast<R*>(base) + p * sp;
#pragma unroll
    for (int c = 0; c < 3; ++c) b[c * sc] = o[c];
}
template <typename R>
__device__ __forceinline__ void st9(void* base, long long p, long long sp, long long sc, const R o[9]) {
    R* b = static_cast<R*>(base) + p * sp;
#pragma unroll
    for (int c = 0; c < 9; ++c) b[c * sc] = o[c];
}

// ---------------------------------------------------------------------------
// 3x3 algebra (row-major arrays)
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void mm(const R A[9], const R B[9], R O[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            O[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
// O = A * B^T
template <typename R>
__device__ __forceinline__ void mmT(const R A[9], const R B[9], R O[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            O[3 * i + j] = A[3 * i] * B[3 * j] + A[3 * i + 1] * B[3 * j + 1] + A[3 * i + 2] * B[3 * j + 2];
}
// O = A^T * B
template <typename R>
__device__ __forceinline__ void mTm(const R A[9], const R B[9], R O[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            O[3 * i + j] = A[i] * B[j] + A[3 + i] * B[3 + j] + A[6 + i] * B[6 + j];
}
template <typename R>
__device__ __forceinline__ void transpose(const R A[9], R O[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) O[3 * i + j] = A[3 * j + i];
}
template <typename R>
__device__ __forceinline__ R det3(const R A[9]) {
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6])
         + A[2] * (A[3] * A[7] - A[4] * A[6]);
}
// inverse by cofactors; returns the determinant
template <typename R>
__device__ __forceinline__ R inv3(const R A[9], R O[9]) {
    R c00 = A[4] * A[8] - A[5] * A[7];
    R c01 = A[5] * A[6] - A[3] * A[8];
    R c02 = A[3] * A[7] - A[4] * A[6];
    R d = A[0] * c00 + A[1] * c01 + A[2] * c02;
    R id = R(1) / d;
    O[0] = c00 * id;
    O[1] = (A[2] * A[7] - A[1] * A[8]) * id;
    O[2] = (A[1] * A[5] - A[2] * A[4]) * id;
    O[3] = c01 * id;
    O[4] = (A[0] * A[8] - A[2] * A[6]) * id;
    O[5] = (A[2] * A[3] - A[0] * A[5]) * id;
    O[6] = c02 * id;
    O[7] = (A[1] * A[6] - A[0] * A[7]) * id;
    O[8] = (A[0] * A[4] - A[1] * A[3]) * id;
    return d;
}
template <typename R>
__device__ __forceinline__ R frob(const R A[9], const R B[9]) {
    R s = 0;
#pragma unroll
    for (int i = 0; i < 9; ++i) s += A[i] * B[i];
    return s;
}
template <typename R>
__device__ __forceinline__ void sym(const R A[9], R O[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) O[3 * i + j] = R(0.5) * (A[3 * i + j] + A[3 * j + i]);
}
template <typename R>
__device__ __forceinline__ bool finite9(const R A[9]) {
    R s = 0;
#pragma unroll
    for (int i = 0; i < 9; ++i) s += A[i] * R(0);
    return s == R(0);   // any Inf/NaN makes the product NaN
}

// ---------------------------------------------------------------------------
// binning: base = floor(x*inv_dx - 0.5), fx = x*inv_dx - base, each operation
// rounded on its own (no FMA contraction), as numpy evaluates
// python/morphompm/transfer.py:19-21.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ bool bin_particle(const R x[3], R inv_dx, const int shape[3], int base[3], R fx[3]) {
    bool inside = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        R X = Num<R>::mul_rn(x[d], inv_dx);
        R t = Num<R>::sub_rn(X, R(0.5));
        R f = d_floor(t);
        if (!(f > R(-1.0e6) && f < R(1.0e6))) {   // NaN or far away
            base[d] = -1000000;
            fx[d] = R(1);
            inside = false;
            continue;
        }
        base[d] = (int)f;
        fx[d] = Num<R>::sub_rn(X, f);
        if (base[d] < -2 || base[d] > shape[d] - 1) inside = false;
    }
    return inside;
}

template <typename R>
__device__ __forceinline__ void bspline(const R fx[3], R w[3][3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        R a = R(1.5) - fx[d], b = fx[d] - R(1.0), c = fx[d] - R(0.5);
        w[0][d] = R(0.5) * a * a;
        w[1][d] = R(0.75) - b * b;
        w[2][d] = R(0.5) * c * c;
    }
}
template <typename R>
__device__ __forceinline__ void bspline_grad(const R fx[3], R dw[3][3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        dw[0][d] = -(R(1.5) - fx[d]);
        dw[1][d] = R(-2.0) * (fx[d] - R(1.0));
        dw[2][d] = fx[d] - R(0.5);
    }
}

// mass and reference volume of particle p: per particle when the plan has
// them, else the scene's
template <typename R>
__device__ __forceinline__ void particle_mass(const Ctx& ctx, const MpmScene& sc, long long p, R& pm, R& vol0) {
    pm = ctx.pmass_p ? static_cast<const R*>(ctx.pmass_p)[p] : (R)sc.pmass;
    vol0 = ctx.vol0_p ? static_cast<const R*>(ctx.vol0_p)[p] : (R)sc.vol0;
}

__device__ __forceinline__ void raise_status(int* status, int bits) {
    if (bits) atomicOr(status, bits);
}

// Growth law g_p(t) = 1 + A * ramp(t) * phi_p (growth_mode 1)
__device__ __forceinline__ double growth_ramp(const MpmScene& sc, int t) {
    if (sc.ramp_steps <= 0.0) return 1.0;
    double r = (double)(t + 1) / sc.ramp_steps;
    return r < 1.0 ? r : 1.0;
}

}  // namespace mpm
