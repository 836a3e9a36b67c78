/*
 * morphompm_b200 -- C ABI of the B200 (sm_100a) MLS-MPM growth step.
 *
 * Plain C types only: device pointers, sizes, a cudaStream_t passed as void*.
 * Every entry point returns an int status (MPM_OK == 0).  The library never
 * allocates device memory: the caller sizes one workspace with
 * mpm_plan_workspace_bytes() and one tape per recorded step with
 * mpm_plan_tape_bytes(), and passes them in.  Device-side failures (non-finite
 * state, particles that left the grid) are recorded in a status word that
 * mpm_plan_read_status() returns.
 *
 * The reference implementation is the numpy package of 2nugu/morphompm; each
 * entry point below names the reference function whose behaviour it replaces.
 */
#ifndef MORPHOMPM_B200_H
#define MORPHOMPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (return values and bits of the device status word) ---- */
#define MPM_OK               0
#define MPM_ERR_ARG          1    /* bad argument (null pointer, bad size)            */
#define MPM_ERR_CUDA         2    /* a CUDA runtime call failed                       */
#define MPM_ERR_NONFINITE    4    /* NaN/Inf produced in state, stress or gradient    */
#define MPM_WARN_OUTSIDE     8    /* a particle's stencil left the grid entirely     */
#define MPM_ERR_TAPE        16    /* tape missing or recorded for another plan        */
#define MPM_ERR_UNSUPPORTED 32    /* model kind / dtype not built                     */
#define MPM_ERR_TOO_LARGE   64    /* scene does not fit the fixed no-allocation scratch */

/* ---- constitutive model kinds (python/morphompm/constitutive.py) ---- */
#define MPM_MODEL_NEOHOOKEAN        0   /* constitutive.py:25-39  */
#define MPM_MODEL_HENCKY            1   /* constitutive.py:42-75  */
#define MPM_MODEL_HERSCHEL_BULKLEY  2   /* constitutive.py:106-147 */
#define MPM_MODEL_EXTERNAL          3   /* stress supplied by the caller (mpm_plan_set_external_stress) */

/* ---- kernel kinds (for mpm_plan_profile_begin) ---- */
#define MPM_K_BIN           0   /* cell keys                                 */
#define MPM_K_SORT          1   /* radix-sort passes (4 kernels per pass)    */
#define MPM_K_MARK          2   /* cell ranges + tile flags                  */
#define MPM_K_COMPACT       3   /* active-tile list                          */
#define MPM_K_PREPASS       4   /* stress + P2G payload                      */
#define MPM_K_P2G           5   /* P2G scatter + grid update                 */
#define MPM_K_G2P           6   /* G2P + advection + F update                */
#define MPM_K_BWD_PAYLOAD   7   /* reserved: no kernel of this kind (the reverse P2G forms its records) */
#define MPM_K_BWD_P2G       8   /* gv_b scatter + grid adjoint               */
#define MPM_K_BWD_PARTICLE  9   /* P2G adjoint + constitutive VJP            */
#define MPM_K_REDUCE       10   /* per-scene reductions                      */
#define MPM_K_COUNT        11

/* ---- arithmetic types ---- */
#define MPM_F32 4
#define MPM_F64 8

/* One scene of a batch: its grid, its material and its growth law.  A batch
 * of one scene with growth_mode 0 is the reference's transfer.step on one
 * SimConfig (python/morphompm/config.py:21-40). */
typedef struct MpmScene {
    int32_t shape[3];        /* nodes per axis (the reference has N,N,N)              */
    int32_t model;           /* MPM_MODEL_*                                           */
    int64_t p_begin, p_end;  /* this scene's particle range in the batch arrays       */
    int32_t wall;            /* sticky nodes: index < wall or >= shape-wall (0 = none) */
    int32_t clamp_lo[3];     /* sticky box [clamp_lo, clamp_hi) (empty if lo >= hi)    */
    int32_t clamp_hi[3];
    int32_t growth_mode;     /* 0: Fg read per particle; 1: Fg = g_p(t) I (see below) */
    double dx, dt, damping, pmass, vol0;
    double mass_eps;         /* grid nodes with mass <= mass_eps are inactive (1e-12)  */
    double gravity[3];
    double mu, lam;          /* neo-Hookean / Hencky Lame parameters                  */
    double kappa, K, n_exp, tau_y, m_pap, eps; /* Herschel-Bulkley (constitutive.py:115) */
    double growth_A;         /* growth_mode 1: g_p(t) = 1 + A*ramp(t)*phi_p            */
    double ramp_steps;       /* ramp(t) = min(1,(t+1)/ramp_steps); 1 when <= 0          */
} MpmScene;

/* Particle arrays.  Element (p, c) of a 3-vector field lives at
 * ptr[p*sp3 + c*sc3]; of a 3x3 field (row-major c = 3*i+j) at ptr[p*sp9 + c*sc9].
 * (n,3)/(n,3,3) C-contiguous arrays use sp3=3,sc3=1,sp9=9,sc9=1.
 * Fg may be NULL when every scene uses growth_mode 1. */
typedef struct MpmParticles {
    void *x, *v, *C, *F, *Fg;
    int64_t sp3, sc3, sp9, sc9;
} MpmParticles;

/* Cotangents of a particle state.  Same layout rules as MpmParticles; the Fg
 * cotangent is always double (it carries the growth-parameter gradient) and is
 * indexed with the strides of F: element c of particle p at Fg[p*sp9 + c*sc9]
 * (in doubles), so it must have the layout of the F cotangent. */
typedef struct MpmCotangents {
    void *x, *v, *C, *F;
    double *Fg;              /* may be NULL when every scene uses growth_mode 1 */
    int64_t sp3, sc3, sp9, sc9;
} MpmCotangents;

/* Schedule knobs (picked by the autotuner; zeros select the defaults). */
typedef struct MpmTuning {
    int32_t tile_xy;             /* node tile edge in x and y: 4, 8 or 16 (default 4)       */
    int32_t scatter_ctas_per_sm; /* persistent P2G node-gather grid = SMs x this (1024-thread CTAs, default 1) */
    int32_t scatter_oxb;         /* stencil x-offsets per pass: 3 (FP32 default) or 1       */
    int32_t particle_block;      /* threads per block of the per-particle kernels: 64, 128 or 256 (default) */
    int32_t active_tile_cap;     /* capacity of the active-tile list (0 = every tile)       */
    float fp64_gap_thresh;       /* FP32 Hencky: relative singular-value gap below this is
                                    recomputed in FP64 (0 selects 1e-6; <0 disables)        */
    int32_t tile_z;              /* node tile edge in z: 4, 8 or 16 (default 4)             */
} MpmTuning;

typedef struct MpmPlan MpmPlan;   /* host-side plan (offsets, tile tables)         */

/* ---- plans: no counterpart in the reference, whose step allocates its grid
 * and caches as numpy arrays on every call (transfer.py:33-79). ---- */

/* Build a plan for a batch of scenes (host only, no CUDA calls).
 * real_bytes is MPM_F32 or MPM_F64. */
int mpm_plan_create(const MpmScene* scenes, int32_t n_scenes, int32_t real_bytes,
                    const MpmTuning* tuning, MpmPlan** out);
void mpm_plan_destroy(MpmPlan* plan);
int mpm_plan_workspace_bytes(const MpmPlan* plan, size_t* bytes);
int mpm_plan_tape_bytes(const MpmPlan* plan, size_t* bytes);
int64_t mpm_plan_num_particles(const MpmPlan* plan);
/* Upload the scene table and index tables into the workspace and clear the
 * status word (stream-ordered; call once before the first step).  Binding
 * again (another workspace) ends any chain of mpm_step_fwd_chain calls. */
int mpm_plan_bind(MpmPlan* plan, void* workspace, void* stream);
/* Copy the device status word into *status (synchronises the stream). */
int mpm_plan_read_status(MpmPlan* plan, int32_t* status, void* stream);
/* Number of FP32 Hencky evaluations that took the FP64 path since bind. */
int mpm_plan_read_fp64_fallbacks(MpmPlan* plan, int64_t* count, void* stream);

/* Bracket every launch of the kernel kinds in kind_mask (bit k = MPM_K_k) with
 * CUDA events, recorded as external event nodes when the stream is being
 * captured, so graph replays re-record them.  At most max_launches launches
 * are bracketed.  mpm_plan_profile_end synchronises and writes, per kind, the
 * summed device time (ms) and the number of bracketed launches (arrays of
 * MPM_K_COUNT entries); for a captured graph the times are those of its last
 * replay. */
int mpm_plan_profile_begin(MpmPlan* plan, uint32_t kind_mask, int32_t max_launches);
int mpm_plan_profile_end(MpmPlan* plan, double* ms_per_kind, int32_t* launches_per_kind);
/* Number of active node tiles recorded in a tape (NULL: the workspace's own
 * scratch tape of the last untaped step).  Synchronises the stream. */
int mpm_plan_active_tiles(MpmPlan* plan, const void* tape, int32_t* n_active, void* stream);

/* Kernel launches issued by this plan so far (host-side count; a captured
 * graph's launches are counted once, at capture). */
int64_t mpm_plan_launch_count(const MpmPlan* plan);

/* Replace the physical parameters of the plan's scenes (growth amplitude and
 * ramp, Lame and Herschel-Bulkley parameters, damping, dt, dx, masses,
 * gravity, walls ...) without rebuilding it.  The structure must not change:
 * the same number of scenes with the same p_begin/p_end, shape, model and
 * growth_mode, else MPM_ERR_ARG.  Kernels read the table from device memory,
 * so a captured CUDA graph replays with the new values.  Ends any chain of
 * mpm_step_fwd_chain calls.  Synchronises `stream`.  No counterpart in the
 * reference (its scene parameters are Python objects rebuilt per call). */
int mpm_plan_update_scenes(MpmPlan* plan, const MpmScene* scenes, int32_t n_scenes, void* stream);

/* Stress supplied by the caller for scenes of kind MPM_MODEL_EXTERNAL (a
 * material defined outside this library, evaluated by the caller before the
 * step): tau is the Kirchhoff stress of every particle, n x 3 x 3 row-major,
 * real type, in particle order.  mpm_step_fwd uses it in place of a built-in
 * model; mpm_step_bwd writes the cotangent of that stress to tau_bar (same
 * layout) and leaves the stress's own VJP (its F, Fg and C cotangents) to the
 * caller, who adds them.  The device counterpart of the reference's seam,
 * which takes any material object with stress / stress_vjp (constitutive.py:
 * 3-5, 79-103).  Both buffers must stay valid while the steps run; a plan with an
 * external scene refuses chained steps and, without tau (tau_bar in the
 * reverse), returns MPM_ERR_ARG. */
int mpm_plan_set_external_stress(MpmPlan* plan, const void* tau, void* tau_bar);

/* Optional per-particle mass and reference volume (real type, n entries in
 * particle order, in place of the scene's pmass / vol0; either may be NULL),
 * as the reference's C++ Particle carries them (growth_solver.h:31-39).
 * The arrays must stay valid while the plan is used.  Ends any chain of
 * mpm_step_fwd_chain calls. */
int mpm_plan_set_particle_mass(MpmPlan* plan, const void* mass, const void* vol0);

/* Optional per-particle growth field phi_p (growth_mode 1), real type: the
 * field growth law g_p(t) = 1 + A ramp(t) phi_p of the reference's growth
 * drivers (docs/PHASE3_morphogenesis.md:55-57), evaluated on the device; the
 * reference's own driver sets Fg = g I per call (integrate.py:31-34).
 * Ends any chain of mpm_step_fwd_chain calls. */
int mpm_plan_set_growth_field(MpmPlan* plan, const void* phi);

/* One forward MLS-MPM step for every scene of the batch:
 * binning + cell sort, stress, P2G, grid update with boundary conditions,
 * G2P with advection and the F update.
 * Replaces python/morphompm/transfer.py:33-79 (step).
 * `in` and `out` must not alias.  `tape` (mpm_plan_tape_bytes) may be NULL; if
 * given it records what mpm_step_bwd needs for this step.  step_index is the t
 * of the growth ramp. */
int mpm_step_fwd(MpmPlan* plan, const MpmParticles* in, MpmParticles* out, int32_t advect,
                 int32_t step_index, void* tape, void* stream);

/* Flags of mpm_step_fwd_chain. */
#define MPM_FWD_CHAINED 1   /* `in` is the `out` of the previous MPM_FWD_EMIT call on this plan */
#define MPM_FWD_EMIT    2   /* also bin `out` and form its P2G records for step_index + 1 */

/* mpm_step_fwd for consecutive steps of one trajectory.  No counterpart in the
 * reference, whose step (python/morphompm/transfer.py:33-79) re-derives the
 * binning and the stress of its input every call.  With MPM_FWD_EMIT the G2P
 * pass also bins the new state and evaluates its stress (Fg of the growth law
 * at step_index + 1, or the same explicit Fg); a following call with
 * MPM_FWD_CHAINED then skips its binning and stress passes.  The results are
 * those of mpm_step_fwd.  The caller must not change the state or an explicit
 * Fg between the EMIT call and the CHAINED call.  A CHAINED call whose `in` (every pointer and stride)
 * or step_index does not continue the last EMIT call, or that follows any
 * other forward call on the plan, returns MPM_ERR_ARG. */
int mpm_step_fwd_chain(MpmPlan* plan, const MpmParticles* in, MpmParticles* out, int32_t advect,
                       int32_t step_index, void* tape, int32_t flags, void* stream);

/* Reverse of mpm_step_fwd for the step recorded in `tape`.
 * Replaces python/morphompm/transfer.py:82-158 (step_vjp).
 * `in` is the step's input state, `out_C` the C of its output state.
 * out_bar: cotangents of the output state; in_bar receives those of the input
 * (Fg cotangent: in_bar->Fg = out_bar->Fg + local term; they may alias).
 * growth_grad (per scene, double, may be NULL) is incremented by d loss / d A
 * for scenes in growth_mode 1. */
int mpm_step_bwd(MpmPlan* plan, const MpmParticles* in, const void* out_C,
                 const MpmCotangents* out_bar, MpmCotangents* in_bar,
                 double* growth_grad, int32_t advect, int32_t step_index,
                 const void* tape, void* stream);

/* mpm_step_bwd that also accumulates the material-parameter gradients: when
 * material_grad is not NULL, material_grad[2 s] += d loss / d mu_s and
 * material_grad[2 s + 1] += d loss / d lambda_s for every scene s (double,
 * deterministic order; zero for Herschel-Bulkley scenes).  No counterpart in
 * the reference, whose constitutive VJPs stop at F, Fg and C
 * (constitutive.py:36-39, 62-75); d/dE and d/dnu follow on the host from
 * mu = E / (2 (1 + nu)), lambda = E nu / ((1 + nu)(1 - 2 nu)). */
int mpm_step_bwd_params(MpmPlan* plan, const MpmParticles* in, const void* out_C,
                        const MpmCotangents* out_bar, MpmCotangents* in_bar,
                        double* growth_grad, double* material_grad, int32_t advect,
                        int32_t step_index, const void* tape, void* stream);

/* ---- whole trajectories: checkpointed forward and adjoint ----
 * Replace python/morphompm/integrate.py:15-28 (rollout, rollout_vjp), whose
 * per-step caches are replaced here by checkpoint-every-k recomputation: the
 * forward keeps the state at the start of every k-step segment, and the
 * reverse recomputes one segment's states and tapes just before reversing it
 * (ckpt_every = 0 or >= n_steps keeps every step and recomputes nothing).
 * A state is a (24, n) slab of the plan's real type: rows x(3), v(3), C(9),
 * F(9), row r of particle p at slab[r n + p]; cotangent slabs have the same
 * layout.  Fg is NULL when every scene uses growth_mode 1, else a (9, n) slab
 * of the real type (row c = 3 i + j).  Both calls are stream-ordered and
 * capturable in one CUDA graph; neither allocates.  External-stress plans
 * (MPM_MODEL_EXTERNAL) return MPM_ERR_UNSUPPORTED: their stress is a
 * callback of every step (mpm_step_fwd / mpm_step_bwd). */

/* Bytes of the rollout workspace for n_steps with checkpoints every ckpt_every
 * (0 for n_steps == 0). */
int mpm_rollout_workspace_bytes(const MpmPlan* plan, int32_t n_steps, int32_t ckpt_every, size_t* bytes);

/* n_steps forward steps from state0 (not modified) into final_state, keeping
 * in rollout_ws (256-byte aligned) what mpm_rollout_bwd needs.  Step t uses
 * step_index t.  state0 and final_state must differ. */
int mpm_rollout_fwd(MpmPlan* plan, const void* state0, const void* Fg, int32_t n_steps, int32_t ckpt_every,
                    int32_t advect, void* rollout_ws, void* final_state, void* stream);

/* Reverse sweep of the trajectory that the last mpm_rollout_fwd on
 * rollout_ws ran (same Fg, n_steps, ckpt_every, advect; rollout_ws untouched
 * in between).  final_bar (not modified) holds the cotangents of the final
 * state, e.g. seeded by mpm_loss_detF / mpm_loss_mse into a zeroed slab;
 * state0_bar (distinct from final_bar) receives those of state0.  Outputs,
 * each overwritten and each optional: Fg_bar (9, n) double, d loss / d Fg
 * summed over the steps (required when Fg is given and wanted); growth_grad
 * (S) double, d loss / d A of growth_mode 1 scenes; material_grad (2 S)
 * double, d loss / d (mu, lambda) per scene as in mpm_step_bwd_params. */
int mpm_rollout_bwd(MpmPlan* plan, const void* Fg, const void* final_bar, int32_t n_steps, int32_t ckpt_every,
                    int32_t advect, void* rollout_ws, void* state0_bar, double* Fg_bar, double* growth_grad,
                    double* material_grad, void* stream);

/* Batched constitutive seam: tau = model.stress(F, Fg, C) for n particles of one
 * scene's model.  Replaces constitutive.py:88-89,126-132. Arrays (n,3,3) C-contiguous. */
int mpm_stress(const MpmScene* scene, int32_t real_bytes, int64_t n, const void* F,
               const void* Fg, const void* C, void* tau, void* stream);
/* (F_bar, Fg_bar, C_bar) = model.stress_vjp(F, Fg, C, tau_bar).
 * Replaces constitutive.py:91-93,134-147. */
int mpm_stress_vjp(const MpmScene* scene, int32_t real_bytes, int64_t n, const void* F,
                   const void* Fg, const void* C, const void* tau_bar, void* F_bar,
                   void* Fg_bar, void* C_bar, void* stream);

/* Cell keys of the binning step (the stencil base of transfer.py:18-21, shifted
 * by +2 per axis and flattened over the (shape+2)^3 padded cells, z fastest;
 * particles whose stencil misses the grid get (shape+2)^3).  x is (n,3). */
int mpm_bin_keys(const MpmScene* scene, int32_t real_bytes, int64_t n, const void* x,
                 int32_t* keys, void* stream);

/* Loss seeds and values (python/morphompm/integrate.py:41-52). Per scene,
 * double loss[s]; F_bar / x_bar are written (not accumulated). */
int mpm_loss_detF(MpmPlan* plan, const void* F, int64_t sp9, int64_t sc9, double* loss,
                  void* F_bar, void* stream);
int mpm_loss_mse(MpmPlan* plan, const void* x, int64_t sp3, int64_t sc3, const void* x_obs,
                 double* loss, void* x_bar, void* stream);

/* Forward growth step of ONE scene that allocates nothing and needs no plan or
 * workspace.  No counterpart in the reference.  It exists for callers that
 * cannot call cudaMalloc: host applications (simulation plugins, real-time
 * controllers) that own every device allocation themselves, and code paths
 * that must not fail on an allocation in the middle of a run.  The caller
 * passes the scene, the input state and the output buffers (same layout rules
 * and semantics as mpm_step_fwd); every intermediate (keys, sort buffers, cell
 * tables, stencil sums, grid) lives in one fixed device array of
 * MPM_NOALLOC_SCRATCH_BYTES compiled into the library, which every GPU that
 * loads the library holds until the process exits.
 *   - A scene whose intermediates exceed that size returns MPM_ERR_TOO_LARGE
 *     (e.g. FP64 fits about 25k particles on a 32^3 grid).
 *   - scene->p_begin must be 0; scene->p_end is the particle count.
 *   - The first call on a device looks the array up (cudaGetSymbolAddress)
 *     with that device current; make that first call before any stream
 *     capture.  The address belongs to the device's context: after a device
 *     reset (cudaDeviceReset) the next call looks it up again, so that call
 *     too must come before any stream capture.
 *   - All calls share the one array: calls whose GPU work overlaps (two
 *     streams, two host threads) race and must be serialised by the caller.
 *     Each call clears the parts that must start at zero.
 *   - status (may be NULL): if given, the call synchronises the stream and
 *     stores the device status word (MPM_ERR_NONFINITE, MPM_WARN_OUTSIDE). */
#define MPM_NOALLOC_SCRATCH_BYTES (32u << 20)
int mpm_step_fwd_noalloc(const MpmScene* scene, int32_t real_bytes, const MpmParticles* in, MpmParticles* out,
                         int32_t advect, int32_t step_index, int32_t* status, void* stream);

/* Bounds-checked build (the same sources compiled with MPM_CHECK_BOUNDS into
 * libmorphompm_b200_checked.so): every index the kernels compute into node,
 * cell-sum, segment, tile and sort arrays is checked; an index out of range is
 * counted and its access skipped.  Returns the number counted since the last
 * call with the site id and index of the first, and resets the count
 * (stream-ordered, synchronizes the stream).  The release library returns
 * MPM_ERR_UNSUPPORTED. */
int mpm_check_violations(int64_t* count, int32_t* first_site, int64_t* first_index, void* stream);

/* ABI version of this header (1). */
int mpm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MORPHOMPM_B200_H */
