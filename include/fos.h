/*
 * fos.h -- C ABI of the B200 foam hot path (libfos.so).
 *
 * Plain pointers and sizes only.  Every pointer argument named pos/rad/... is a
 * DEVICE pointer (cudaMalloc'd, or a torch CUDA tensor's data_ptr()) unless
 * its name ends in _host.  Every entry point returns an int status (FOS_OK = 0)
 * and is asynchronous on the given stream, except where it says it
 * synchronises (the ones that hand a scalar back to the host, as the
 * reference's Taichi kernels with a return value do).  A context is not
 * thread safe; use one per host thread.
 *
 * Reference interface each entry replaces (VirtualOrganics/Fabric-of-Space-
 * Taichi-JFA, file:line) is cited beside it.  Layouts: pos is [n][3] float32,
 * rad [n] float32, face_ids/face_counts/neighbor_list [n][32] int32, voxel
 * (x,y,z) at linear index (x*R + y)*R + z.
 */
#ifndef FOS_H
#define FOS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* fos_stream_t; /* == cudaStream_t; NULL = legacy default stream */

#define FOS_MAX_NEIGHBORS 32 /* jfa.py:74 MAX_NEIGHBORS */
#define FOS_MAX_PASSES 64

enum FosStatus {
    FOS_OK = 0,
    FOS_E_ARG = 1,           /* bad argument (null pointer, n out of range, ...) */
    FOS_E_CAPACITY = 2,      /* n or res above the context's capacity, table full */
    FOS_E_CUDA = 3,          /* a CUDA runtime call failed */
    FOS_E_TIMEOUT = 4,       /* a bounded device-side wait gave up */
    FOS_E_DEVICE = 5,        /* a device-side check recorded an error word */
    FOS_E_STATE = 6          /* call out of order (e.g. no JFA has run yet) */
};

/* Constants of config.py / jfa.py that the reference bakes into its kernels.
 * Python-float constants are doubles here and are folded to float32 exactly as
 * Taichi folds a Python float into a kernel literal. */
typedef struct FosParams {
    double domain_size;             /* DOMAIN_SIZE (config.py:21), L */
    int grid_res;                   /* GRID_RES (config.py:317) */
    double power_beta;              /* power_beta_current (jfa.py:184) */
    int early_exit;                 /* JFA_EARLY_EXIT_ENABLED (config.py:208) */
    int min_jfa_passes;             /* MIN_JFA_PASSES (config.py:210) */
    double th_pass_delta;           /* TH_PASS_DELTA (config.py:209) */
    int tie_lower_index;            /* 0: reference scan-order ties; 1: lower seed index wins */
    double expected_face_scale;     /* EXPECTED_FACE_SCALE (jfa.py:58) */
    double t_add;                   /* T_ADD (jfa.py:63) */
    double t_drop;                  /* T_DROP (jfa.py:64) */
    double ema_alpha;               /* JFA_EMA_ALPHA (config.py:81) */
    double gap_fraction;            /* GAP_FRACTION (config.py:353) */
    double max_displacement_frac;   /* MAX_DISPLACEMENT_FRAC (config.py:349) */
    double displacement_multiplier; /* DISPLACEMENT_MULTIPLIER (config.py:350) */
    double eps;                     /* EPS (config.py:324) */
    double contact_tol;             /* CONTACT_TOL (config.py:254) */
    double fsc_deadband;            /* FSC_DEADBAND (config.py:100) */
} FosParams;

typedef struct FosCtx FosCtx;

/* Fills *p with the reference defaults (config.py / jfa.py). */
void fos_params_default(FosParams* p);

/* jfa.init_jfa (jfa.py:120-204): allocates every JFA/FSC field at capacity
 * (max_n particles, max_res^3 voxels) on `device`.  The only entry point,
 * with fos_ctx_destroy, that allocates or frees device memory. */
int fos_ctx_create(const FosParams* p, int max_n, int max_res, int device, FosCtx** out);
int fos_ctx_destroy(FosCtx* ctx);
int fos_set_params(FosCtx* ctx, const FosParams* p);

/* jfa.set_resolution (jfa.py:207-227) without the [JFA_RES_MIN, JFA_RES_MAX]
 * clamp (the caller clamps): sets JFA_RES, VOXEL_SIZE = L/R and
 * JFA_NUM_PASSES = ceil(log2 R) + 1.  res must be in [2, max_res]. */
int fos_set_resolution(FosCtx* ctx, int res);
int fos_get_resolution(FosCtx* ctx, int* res, int* num_passes, float* voxel_size);

/* Device pointers of the context-owned fields (jfa.py module fields).  Any out
 * pointer may be NULL.  labels is the final JFA owner grid of the last run
 * (int32, R^3), label_filtered the majority-filtered grid. */
typedef struct FosJfaFields {
    int32_t* fsc;                  /* jfa.fsc            [max_n] */
    float* fsc_ema;                /* jfa.fsc_ema        [max_n] */
    int32_t* face_ids;             /* jfa.face_ids       [max_n][32] */
    int32_t* face_counts;          /* jfa.face_counts    [max_n][32] */
    int32_t* neighbor_list;        /* jfa.neighbor_list  [max_n][32] */
    int32_t* neighbor_used_count;  /* jfa.neighbor_used_count [max_n] (== neighbor_count) */
    float* neighbor_prev_scores;   /* jfa.neighbor_prev_scores [max_n][32] */
    int32_t* labels;               /* final owner labels of the last run, R^3 */
    int32_t* label_filtered;       /* jfa.label_filtered, R^3 */
} FosJfaFields;
int fos_jfa_fields(FosCtx* ctx, FosJfaFields* out);

/* jfa.run_jfa (jfa.py:1056-1197), device part: jfa_init, the pass loop (with
 * the optional device-side early exit), majority_filter_labels,
 * accumulate_face_area, finalize_faces_kernel and update_fsc_ema.  Results
 * land in the context's fields; nothing is copied to the host. */
int fos_jfa_run(FosCtx* ctx, const float* pos, const float* rad, int n, fos_stream_t s);

/* Warm-started JFA (no reference counterpart; run.py only plans it,
 * docs/GITHUB_ISSUES.md:225-300): the previous run's final owner grid is the
 * starting point, every seed is planted again at its current voxel, and the
 * passes run with steps first_step, first_step/2, ..., 1, 1 (first_step a
 * power of two <= res/2) instead of res/2 ... 1, 1.  Needs a previous run at
 * the same resolution.  An approximation of fos_jfa_init + fos_jfa_passes:
 * agreement with the exact run is measured, not guaranteed. */
int fos_jfa_warm(FosCtx* ctx, const float* pos, const float* rad, int n, int first_step,
                 fos_stream_t s);

/* The stages of fos_jfa_run one by one (for tests and the Python mirror). */
int fos_jfa_init(FosCtx* ctx, const float* pos, const float* rad, int n, fos_stream_t s); /* jfa.py:484-520 */
int fos_jfa_passes(FosCtx* ctx, int n, fos_stream_t s);          /* jfa.py:1082-1116 (uses the seed table) */
int fos_jfa_majority_filter(FosCtx* ctx, fos_stream_t s);        /* jfa.py:639-699 */
int fos_jfa_accumulate_faces(FosCtx* ctx, int n, fos_stream_t s);/* jfa.py:702-762 */
int fos_jfa_finalize(FosCtx* ctx, const float* rad, int n, fos_stream_t s); /* jfa.py:788-857 */
int fos_jfa_update_ema(FosCtx* ctx, int n, fos_stream_t s);      /* jfa.py:765-785 */

/* Load an owner grid (R^3 int32, device) as the "final labels" so the FSC
 * stages can run on given labels (parity tests of the stages in isolation). */
int fos_jfa_load_labels(FosCtx* ctx, const int32_t* labels, fos_stream_t s);

/* run_jfa's stats dict (jfa.py:1149-1195) plus build diagnostics.  Synchronises. */
typedef struct FosJfaStats {
    int num_passes;
    int early_exit;
    long long changes[FOS_MAX_PASSES]; /* label_changes per pass (delta_history * V) */
    int jfa_res;
    float voxel_size;
    float mean_score, std_score;       /* compute_score_stats (jfa.py:1257-1330) */
    int p_dir, p_und_accepted;         /* compute_pair_symmetry (jfa.py:1204-1220) */
    int overflow_count;                /* compute_overflow_count (jfa.py:1223-1234) */
    float overflow_pct;
    float mean_fsc;                    /* compute_fsc_stats (jfa.py:1237-1254) */
    int min_fsc, max_fsc;
    float mean_fsc_ema;
    int finalize_iterations;           /* fixed-point sweeps the exact finalize took */
    int face_pairs;                    /* distinct {a,b} pairs found this run */
    int max_row_candidates;            /* largest per-particle candidate count */
    int zero_fsc_count;                /* particles with fsc == 0 */
} FosJfaStats;
int fos_jfa_stats(FosCtx* ctx, int n, const float* rad, FosJfaStats* out, fos_stream_t s);

/* validate_jfa (jfa.py:1400-1426).  Synchronises. */
typedef struct FosValidate {
    int passed, asymmetric_pairs, overflow_count, self_loops;
} FosValidate;
int fos_jfa_validate(FosCtx* ctx, int n, FosValidate* out, fos_stream_t s);

/* ------------------------------------------------------------------- grid.py
 * Cell arrays are [GRID_RES^3] int32, cell_indices [n] int32. */
int fos_grid_clear(FosCtx* ctx, int32_t* cell_count, fos_stream_t s);                  /* grid.py:145-155 */
int fos_grid_count(FosCtx* ctx, const float* pos, int32_t* cell_count, int n, fos_stream_t s); /* grid.py:186-222 */
int fos_grid_prefix_sum(FosCtx* ctx, const int32_t* cell_count, int32_t* cell_start, fos_stream_t s); /* grid.py:229-243 */
int fos_grid_copy_pointers(FosCtx* ctx, const int32_t* cell_start, int32_t* cell_write, fos_stream_t s); /* grid.py:250-261 */
/* scatter_particles (grid.py:268-309): wraps pos in place; each cell's slice of
 * cell_indices is ascending (the serial order), cell_write ends at cell end. */
int fos_grid_scatter(FosCtx* ctx, float* pos, int32_t* cell_write, int32_t* cell_indices, int n,
                     fos_stream_t s);
/* rebuild_grid (run.py:476-504) in one call: clear, count, scan, scatter. */
int fos_grid_build(FosCtx* ctx, float* pos, int n, int32_t* cell_count, int32_t* cell_start,
                   int32_t* cell_indices, fos_stream_t s);

/* No counterpart in the reference.  The hash-grid rebuild of fos_grid_build for
 * callers that cannot allocate device memory at the point where they need the
 * grid: a host whose own pool or caching allocator owns all device memory, a
 * frame loop that cannot afford cudaMalloc/cudaFree synchronising the device,
 * or a C host that holds raw buffers and no context.  It takes no context and
 * allocates nothing.  The per-particle scratch (cell and arrival rank) lives in
 * a static device array compiled into the library: 512 KiB on every GPU that
 * loads it, held until the process exits.  That caps n at
 * FOS_NOALLOC_MAX_PARTICLES; a larger n returns FOS_E_CAPACITY and launches
 * nothing.  Outside stream capture every call looks up the array's device
 * address (cudaGetSymbolAddress: no allocation, no synchronisation), so a
 * device reset between calls is harmless.  During capture the address of an
 * earlier call on the same device is reused; a first call on a device made
 * during capture returns FOS_E_ARG, so make one call before capturing.
 * All calls share the one array: calls that overlap on the GPU (other streams,
 * other host threads) race and must be serialised.  Outputs equal
 * fos_grid_build's: cell_count and cell_start [grid_res^3], cell_indices
 * ascending inside each cell, pos wrapped in place.  grid_res (GRID_RES, at most
 * FOS_NOALLOC_MAX_GRID_RES: the cell-count scan runs in one thread block) and
 * domain_size (DOMAIN_SIZE) are the grid's. */
#define FOS_NOALLOC_MAX_PARTICLES 65536
#define FOS_NOALLOC_MAX_GRID_RES 256
int fos_grid_build_noalloc(float* pos, int n, int grid_res, double domain_size,
                           int32_t* cell_count, int32_t* cell_start, int32_t* cell_indices,
                           fos_stream_t s);

/* --------------------------------------------------------------- dynamics.py */
/* project_overlaps (dynamics.py:77-171) as one Jacobi sweep; pos updated in place. */
int fos_project_overlaps(FosCtx* ctx, float* pos, const float* rad, const int32_t* cell_start,
                         const int32_t* cell_count, const int32_t* cell_indices, int n,
                         fos_stream_t s);
/* compute_max_overlap (dynamics.py:304-372): fills local_max_depth; the global
 * max goes to *max_host (synchronises) and/or *max_dev (async); either may be NULL. */
int fos_compute_max_overlap(FosCtx* ctx, const float* pos, const float* rad,
                            const int32_t* cell_start, const int32_t* cell_count,
                            const int32_t* cell_indices, float* local_max_depth, int n,
                            float* max_dev, float* max_host, fos_stream_t s);
/* equilibrate_pressure (dynamics.py:1454-1557), `sweeps` Jacobi sweeps with the
 * same frame.  max_abs_dr_host/changed_host (of the last sweep) synchronise
 * when non-NULL. */
int fos_equilibrate_pressure(FosCtx* ctx, int n, int frame, float* rad, float* delta_r,
                             const int32_t* face_ids, const int32_t* fsc, float k, float p_exp,
                             float pair_cap, int max_nei, float r_min, float r_max, int sweeps,
                             float* max_abs_dr_host, int* changed_host, fos_stream_t s);
/* apply_brownian_motion (dynamics.py:1596-1634) with Philox-4x32-10 keyed by
 * (seed, frame, particle) in place of ti.random(). */
int fos_apply_brownian(FosCtx* ctx, float* pos, int n, float strength, float domain_size,
                       uint64_t seed, uint32_t frame, fos_stream_t s);
/* OU jitter (dynamics.py:600-690).  The uniform draws U[-0.5, 0.5)^3 of
 * ti.random() come from Philox-4x32-10 with counter (i, frame, 'OUJT', 0) and
 * key = seed.
 * init_jitter_velocities (dynamics.py:600-605): v_jit = 0. */
int fos_init_jitter_velocities(FosCtx* ctx, float* v_jit, int n, fos_stream_t s);
/* compute_mean_radius (dynamics.py:675-689) into a device float.  The sum is
 * exact (each radius as a 2^-40 fixed-point integer, summed in 64 bits), so
 * the result does not depend on the order of the additions. */
int fos_compute_mean_radius(FosCtx* ctx, const float* rad, int n, float* mean_radius,
                            fos_stream_t s);
/* apply_brownian (dynamics.py:607-646): OU update of v_jit with the mean
 * radius read from the device float mean_radius, capped per step at
 * max_drift_fraction * gap_fraction * 2 r_i. */
int fos_apply_jitter(FosCtx* ctx, float* v_jit, const float* rad, const float* mean_radius, int n,
                     float dt, double jitter_rms, double jitter_tau, double max_drift_fraction,
                     double gap_fraction, uint64_t seed, uint32_t frame, fos_stream_t s);
/* integrate_jitter (dynamics.py:649-660): pos = wrapP(pos + v_jit * dt). */
int fos_integrate_jitter(FosCtx* ctx, float* pos, const float* v_jit, int n, float dt,
                         fos_stream_t s);
/* set_fsc_targets (dynamics.py:1242-1320) */
int fos_set_fsc_targets(FosCtx* ctx, const float* rad, float* rad_target, const int32_t* fsc,
                        const float* fsc_ema, int n, int f_low, int f_high, float growth_pct,
                        float r_min, float r_max, fos_stream_t s);
/* nudge_radii_adaptive_ema (dynamics.py:1366-1427); mode 0 off, 1 global, 2 local */
int fos_nudge_radii(FosCtx* ctx, float* rad, const float* rad_target, const float* local_max_depth,
                    int n, float alpha, float max_step_pct, float r_min, float r_max,
                    float back_global, int mode, fos_stream_t s);
/* compute_controller_stats (dynamics.py:1322-1363).  Synchronises. */
int fos_controller_stats(FosCtx* ctx, const float* rad, const float* rad_target,
                         const float* fsc_ema, int n, int f_low, int f_high, int* grow,
                         int* shrink, int* idle, float* mean_dr, float* max_dr, fos_stream_t s);
/* compute_pressure_stats (dynamics.py:1560-1589).  Synchronises. */
int fos_pressure_stats(FosCtx* ctx, int n, const float* rad, float* rmin, float* rmax,
                       fos_stream_t s);

/* ------------------------------------------------------------ frame driver
 * One headless frame in run.py's order (run.py:699-1261): grid build; max
 * overlap; settle nudge while the device settle counter is > 0; `pressure_iters`
 * pressure sweeps on the last JFA's face_ids/fsc; Brownian jitter; pbd_iters x
 * {grid build; PBD}; OU jitter when ou_jitter; grid build; and on a JFA frame run_jfa, the warm-start
 * gate (frame < warmstart_frames or zero-FSC fraction > zero_rate_thresh) and
 * set_fsc_targets + settle = adjustment_frames.  The frame index, settle
 * counter and gate live on the device, so a frame does no host sync and can be
 * replayed from a CUDA graph. */
typedef struct FosFrameParams {
    int pbd_iters;
    int pressure_iters;
    int f_low, f_high;            /* FSC band */
    double growth_pct;            /* GROWTH_PCT */
    double max_step_pct;          /* MAX_STEP_PCT */
    int adjustment_frames;        /* ADJUSTMENT_FRAMES */
    int bp_mode;                  /* BACKPRESSURE_MODE: 0 off, 1 global, 2 local */
    int warmstart_frames;         /* WARMSTART_FRAMES */
    double zero_rate_thresh;      /* FSC_ZERO_RATE_THRESH */
    double r_min, r_max;          /* R_MIN, R_MAX */
    double pressure_k, pressure_exp, pressure_pair_cap; /* PRESSURE_K/EXP/PAIR_CAP */
    int max_eq_nei;               /* MAX_EQ_NEI */
    double brownian_strength;     /* BROWNIAN_STRENGTH (uniform +-strength per axis) */
    uint64_t seed;                /* Philox key of the Brownian jitter */
    int warmup_pbd;               /* PBD_BASE_PASSES used by fos_sim_init */
    /* OU velocity jitter after the PBD sweeps (run.py:855-867), a second jitter
     * channel next to the Brownian one; 0 = off.  Needs FosState.v_jit. */
    int ou_jitter;                /* JITTER_ENABLED */
    double jitter_rms;            /* JITTER_RMS: RMS drift per second, in mean radii */
    double jitter_tau;            /* JITTER_TAU: OU time scale (s) */
    double dt;                    /* DT: time step of the OU update (s) */
    double max_drift_fraction;    /* MAX_DRIFT_FRACTION: step cap, in GAP_FRACTION*(2r) */
    int jfa_warm_step;            /* first step of a warm-started JFA (jfa_frame == 2) */
} FosFrameParams;

/* Caller-owned per-particle state (run.py's fields). */
typedef struct FosState {
    int n;
    float* pos;                 /* [n][3] */
    float* rad;                 /* [n] */
    float* rad_target;          /* [n] */
    float* local_max_depth;     /* [n] */
    float* delta_r;             /* [n] */
    int32_t* cell_count;        /* [GRID_RES^3] */
    int32_t* cell_start;        /* [GRID_RES^3] */
    int32_t* cell_indices;      /* [n] */
    float* v_jit;               /* [n][3] OU jitter velocity (run.py:151); may be NULL
                                   unless FosFrameParams.ou_jitter */
} FosState;

void fos_frame_params_default(FosFrameParams* fp);
/* initialize_simulation's device part (run.py:320-382): wrap positions, run
 * warmup_pbd passes, zero fsc/fsc_ema/face_ids/prev scores, set rad_target =
 * rad and reset the device frame index to frame0 and the settle counter. */
int fos_sim_init(FosCtx* ctx, const FosState* st, const FosFrameParams* fp, int frame0,
                 fos_stream_t s);
/* jfa_frame: 0 no JFA, 1 the exact JFA, 2 the warm-started JFA (fos_jfa_warm
 * with fp->jfa_warm_step). */
int fos_frame(FosCtx* ctx, const FosState* st, const FosFrameParams* fp, int jfa_frame,
              fos_stream_t s);
/* Same frame replayed from a CUDA graph captured on first use per
 * (state, params, jfa_frame); recaptured when any of them changes. */
int fos_frame_graph(FosCtx* ctx, const FosState* st, const FosFrameParams* fp, int jfa_frame,
                    fos_stream_t s);
/* fos_frame with a CUDA event after every stage (no graph; synchronises).
 * stage_ms[FOS_FRAME_STAGES] receives milliseconds per stage: 0 hash-grid
 * builds, 1 max overlap, 2 settle nudge, 3 pressure sweeps, 4 Brownian, 5 PBD
 * sweeps, 6 JFA init + passes, 7 majority filter + faces, 8 finalize + EMA,
 * 9 targets + frame end, 10 OU jitter. */
#define FOS_FRAME_STAGES 11
int fos_frame_profile(FosCtx* ctx, const FosState* st, const FosFrameParams* fp, int jfa_frame,
                      float* stage_ms, fos_stream_t s);
/* Tracing: the dynamics part of a plain frame (the persistent cooperative
 * kernel) with a %globaltimer stamp, in ns, at kernel entry and after every
 * grid barrier (block 0's view).  Allocates a scratch buffer and
 * synchronises; for profiling, not for the frame loop.  *count gets the
 * number of stamps written (<= cap - 2); ns_host[cap - 2] holds the bitwise
 * NOT of the earliest block's start and ns_host[cap - 1] the latest block's
 * end (cap >= 3). */
int fos_frame_trace(FosCtx* ctx, const FosState* st, const FosFrameParams* fp, long long* ns_host,
                    int cap, int* count, fos_stream_t s);
/* The frame in two parts, for hosts that decide on the JFA after the
 * dynamics, as run.py's temporal skip does (run.py:905-1018):
 * fos_frame_dynamics runs steps 1-7 and the OU jitter; fos_frame_measure
 * runs step 8 when jfa_frame, then ends the frame.  The two in sequence equal
 * fos_frame. */
int fos_frame_dynamics(FosCtx* ctx, const FosState* st, const FosFrameParams* fp,
                       fos_stream_t s);
int fos_frame_measure(FosCtx* ctx, const FosState* st, const FosFrameParams* fp, int jfa_frame,
                      fos_stream_t s);
/* Activity signals of the temporal skip (run.py:913-976) for the current
 * state against the previous frame's positions and radii (either may be
 * NULL: the signal is then -1).  Synchronises. */
typedef struct FosSkipSignals {
    int n;
    int out_of_band;      /* particles with fsc < f_low or fsc > f_high */
    int zero_fsc;         /* particles with fsc == 0 */
    int pad;
    double r_mean;        /* mean radius: exact sum, rounded once to float32 */
    double sigma_dr;      /* population std of |rad - rad_prev| (double) */
    double vmax_dt;       /* max |pos - pos_prev| with the periodic fold, float32 */
    double fsc_mean;      /* mean fsc (exact sum) */
} FosSkipSignals;
int fos_skip_signals(FosCtx* ctx, const FosState* st, const float* pos_prev,
                     const float* rad_prev, int f_low, int f_high, FosSkipSignals* out,
                     fos_stream_t s);
/* Device frame index and settle counter: set (a checkpoint resume; also
 * clears the device error word) and read (synchronises). */
int fos_sim_set_counters(FosCtx* ctx, int frame, int settle, fos_stream_t s);
int fos_sim_counters(FosCtx* ctx, int* frame, int* settle, fos_stream_t s);

/* ------------------------------------------------------------ dirty tiles
 * mark_dirty_tiles (jfa.py:966-1008) on the current resolution's tiles of
 * 16^3 voxels (tiles_per_axis = ceil(res / 16)), tile_dirty [t][t][t] uint8:
 * a particle whose position moved more than pos_threshold * VOXEL_SIZE, whose
 * radius changed more than rad_threshold * VOXEL_SIZE, or whose tile changed
 * since (pos_prev, rad_prev) marks its tile and the halo around it.
 * clear_dirty_tiles and update_tile_cache are a memset and a copy. */
int fos_dirty_mark(FosCtx* ctx, const float* pos, const float* rad, const float* pos_prev,
                   const float* rad_prev, int n, double pos_threshold, double rad_threshold,
                   int halo, uint8_t* tile_dirty, fos_stream_t s);
/* count_dirty_tiles (jfa.py:1011-1024).  Synchronises. */
int fos_dirty_count(FosCtx* ctx, const uint8_t* tile_dirty, int* count, fos_stream_t s);

/* ------------------------------------------------------------ topology
 * Gabriel-graph / k-NN topological degree over the hash grid (topology.py),
 * an FSC-independent neighbour count.  The grid arguments are the CSR cell
 * arrays of the last rebuild (each cell's particles ascending).  Candidate
 * lists are [n][cap] int32 (MAX_TOPO_NEIGHBORS = 28 in the reference).
 * build_topo_candidates (topology.py:68-135): the first `cap` j > i within
 * max_radius_multiple * (r_i + r_j) in serial scan order; truncated[i] = 1
 * when more qualify. */
int fos_topo_candidates(FosCtx* ctx, const float* pos, const float* rad, const int32_t* cell_start,
                        const int32_t* cell_count, const int32_t* cell_indices, int n,
                        double max_radius_multiple, int cap, int32_t* topo_pairs,
                        int32_t* pair_count, int32_t* truncated, fos_stream_t s);
/* gabriel_test_topological_degree (topology.py:140-262): deg is zeroed, then
 * every kept candidate pair whose open diameter sphere holds no witness adds
 * 1 to both ends.  stride = TOPO_PAIR_SUBSAMPLING_STRIDE (pairs kept when
 * the frame hash is divisible by it), early_exit with deg_high =
 * TOPO_EARLY_EXIT_HIGH_DEGREE / TOPO_DEG_HIGH against deg_ema, cell_size =
 * CELL_SIZE (witness stencil radius). */
int fos_topo_gabriel(FosCtx* ctx, const float* pos, const int32_t* cell_start,
                     const int32_t* cell_count, const int32_t* cell_indices, int n, int frame,
                     double cell_size, int stride, int early_exit, double deg_high, int cap,
                     const int32_t* topo_pairs, const int32_t* pair_count, const float* deg_ema,
                     int32_t* deg, fos_stream_t s);
/* gabriel_update_batched (topology.py:335-446): particles i with
 * i % num_batches == batch rebuild their subsampled candidates and add their
 * Gabriel edges to deg (not zeroed).  pair_count keeps the reference's
 * uncapped count; only the `cap` stored candidates are tested. */
int fos_topo_batched(FosCtx* ctx, const float* pos, const float* rad, const int32_t* cell_start,
                     const int32_t* cell_count, const int32_t* cell_indices, int n, int batch,
                     int num_batches, int subsample_q, int frame, double max_radius_multiple,
                     double cell_size, int cap, int32_t* topo_pairs, int32_t* pair_count,
                     int32_t* truncated, int32_t* deg, fos_stream_t s);
/* knn_topo_degree (topology.py:458-505): neighbours within
 * (max_radius_multiple * r_i)^2, capped at k. */
int fos_topo_knn(FosCtx* ctx, const float* pos, const float* rad, const int32_t* cell_start,
                 const int32_t* cell_count, const int32_t* cell_indices, int n, int k,
                 double max_radius_multiple, int32_t* deg, fos_stream_t s);
/* update_topo_ema / commit_topo_to_ema (topology.py:265-283, 448-455):
 * ema = alpha * deg + (1 - alpha) * ema. */
int fos_topo_ema(FosCtx* ctx, const int32_t* deg, float* deg_ema, float alpha, int n,
                 fos_stream_t s);
/* update_radii_topological (topology.py:286-322). */
int fos_topo_update_radii(FosCtx* ctx, float* rad, const float* deg_effective, float deg_low,
                          float deg_high, float gain_grow, float gain_shrink, float r_min,
                          float r_max, int n, fos_stream_t s);

/* ------------------------------------------------------------ FSC surrogate
 * No counterpart in the reference: run.py reuses the last JFA's fsc on the
 * frames between JFA runs (run.py:1230-1261).  A learned per-pair model gives
 * a fresh FSC estimate on those frames instead.
 *
 * Candidate pairs {a, b} have |d| < cutoff * (r_a + r_b) (periodic minimum
 * image).  Each pair is kept once, by its owner i (the other particle is j):
 * for a < b the owner is a when a + b is odd and b when it is even, so every
 * particle owns about half of its pairs whatever its index.  Each pair gets
 * FOS_SUR_FEATURES FP32 features, with d = x_j - x_i:
 *   0       |d| / (r_i + r_j)
 *   1       r_i / r_j
 *   2       signed offset of the power bisector from the midpoint, over
 *           r_i + r_j: (r_i^2 - r_j^2) / (2 |d| (r_i + r_j)), evaluated as
 *           (r_i - r_j) / ((2 * x0) * (r_i + r_j)) (0 when x0 == 0)
 *   3..13   11-bin histogram (bins of width cutoff/11 in normalised distance)
 *           of both particles' other candidates, counts summed over i and j;
 *   14      1 when i and j were neighbours at the last JFA frame (j in i's
 *           neighbour list or i in j's), else 0;
 *   15      fsc_i + fsc_j of the last JFA frame.
 * The model is an MLP 16 -> 64 -> ReLU -> 64 -> ReLU -> 1 -> sigmoid giving
 * the probability that the pair shares a face.  A particle's FSC estimate is
 * the sum of its pairs' probabilities.  Inference uses BF16 weights and
 * activations with FP32 accumulation on the tensor cores; training keeps FP32
 * master weights and runs Adam.
 *
 * FP32 parameter layout (FOS_SUR_NPARAM floats):
 *   W1[64][16] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3
 * with W[out][in]. */
#define FOS_SUR_FEATURES 16
#define FOS_SUR_HIDDEN 64
#define FOS_SUR_BINS 11
#define FOS_SUR_PAIR_CAP 96 /* pairs kept per owner particle */
#define FOS_SUR_NPARAM (64 * 16 + 64 + 64 * 64 + 64 + 64 + 1)

typedef struct FosSurrogate FosSurrogate;

typedef struct FosSurrogateStats {
    int pairs;          /* candidate pairs of the last pair build */
    int overflow;       /* particles that owned more than FOS_SUR_PAIR_CAP pairs */
    int judged;         /* particles compared on the last judged JFA frame */
    int exact;          /* ... with rint(surrogate FSC) == JFA fsc */
    int within1;        /* ... with |rint(surrogate FSC) - JFA fsc| <= 1 */
    int stale_exact;    /* ... whose previous JFA fsc equals this JFA fsc */
    int stale_within1;
    double abs_err;     /* sum over particles of |surrogate FSC - JFA fsc| */
    double stale_abs_err;
} FosSurrogateStats;

/* How a surrogate frame turns the model's estimate s_i into the FSC fed to
 * the controller:
 *   FOS_SUR_ABSOLUTE  f_i = s_i;
 *   FOS_SUR_ANCHORED  f_i = max(0, fsc_i(last JFA) + s_i - s_i(last JFA)),
 *                     the last JFA's exact count moved by the change the
 *                     model sees since then (its bias cancels).  Until the
 *                     context has seen one judged JFA frame it behaves as
 *                     ABSOLUTE. */
#define FOS_SUR_ABSOLUTE 0
#define FOS_SUR_ANCHORED 1
int fos_surrogate_set_mode(FosCtx* ctx, int mode);
/* The inference kernel on ctx: FOS_SUR_TCGEN05 (the default) runs 128-pair
 * tiles on the 5th-generation tensor cores (tcgen05.mma into TMEM, read back
 * with tcgen05.ld); FOS_SUR_MMA_SYNC runs warp-level mma.sync m16n8k16 tiles
 * of 16 pairs.  Both round inputs and hidden activations to BF16 and
 * accumulate in FP32; the FP32 sums run in different orders, so the
 * probabilities agree to a few ulps, not bit for bit. */
#define FOS_SUR_MMA_SYNC 0
#define FOS_SUR_TCGEN05 1
int fos_surrogate_set_inference(FosCtx* ctx, int kind);

/* A model on `device` with candidate cutoff `cutoff` (in units of r_i + r_j).
 * Weights start at zero; set them with fos_surrogate_set_weights. */
int fos_surrogate_create(int device, float cutoff, FosSurrogate** out);
int fos_surrogate_destroy(FosSurrogate* m);
/* Host arrays: params[FOS_SUR_NPARAM] (layout above), mu/sd[FOS_SUR_FEATURES]
 * (the features are standardised as (x - mu) / sd before the first layer).
 * Resets the Adam moments and step. */
int fos_surrogate_set_weights(FosSurrogate* m, const float* params, const float* mu,
                              const float* sd);
int fos_surrogate_get_weights(FosSurrogate* m, float* params, float* mu, float* sd);
float fos_surrogate_cutoff(const FosSurrogate* m);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the mean binary cross
 * entropy of the `batch` rows X[rows[k]] (device arrays: X [*][16] raw
 * features, y [*] labels in {0,1}, rows [batch], every entry a valid row).
 * FP32 forward/backward, deterministic.  loss: device float receiving the
 * batch loss, or NULL. */
int fos_surrogate_train_step(FosSurrogate* m, const float* X, const float* y, const int32_t* rows,
                             int batch, float lr, float* loss, fos_stream_t s);
/* The same forward/backward without the update: grad[FOS_SUR_NPARAM] (device)
 * receives d(loss)/d(params). */
int fos_surrogate_gradient(FosSurrogate* m, const float* X, const float* y, const int32_t* rows,
                           int batch, float* grad, float* loss, fos_stream_t s);
/* Tensor-core inference on given raw features X [P][16] (device): prob[P]. */
int fos_surrogate_forward(FosSurrogate* m, const float* X, int P, float* prob, fos_stream_t s);

/* Candidate pairs of the n particles on ctx, found on the hash grid
 * (cell_start/count/indices of the same positions; the search reach follows
 * cutoff * (r_i + r_max)).  r_max bounds every radius.  Asynchronous. */
int fos_surrogate_pairs(FosCtx* ctx, const FosSurrogate* m, const float* pos, const float* rad,
                        int n, float r_max, const int32_t* cell_start, const int32_t* cell_count,
                        const int32_t* cell_indices, fos_stream_t s);
/* Pair count and overflow count of the last pair build (synchronises). */
int fos_surrogate_pair_count(FosCtx* ctx, int* pairs, int* overflow, fos_stream_t s);
/* Training export of the last pair build, in pair order (owner i
 * ascending, then search order): X [P][16] raw features, y [P] = 1 when j is
 * in i's JFA neighbour list on ctx (the last finalize), pair_i/pair_j [P].
 * Features 14-15 come from mem_nl [n][32] (16-byte aligned), mem_used [n] and mem_fsc [n] (an
 * earlier JFA frame's neighbour lists, used counts and fsc, so that the
 * label is not among the inputs); NULL takes the context's current ones, as
 * inference does.  Any output may be NULL.  Asynchronous; size the outputs
 * with fos_surrogate_pair_count. */
int fos_surrogate_export(FosCtx* ctx, const float* rad, float* X, float* y, int32_t* pair_i,
                         int32_t* pair_j, const int32_t* mem_nl, const int32_t* mem_used,
                         const int32_t* mem_fsc, fos_stream_t s);
/* Inference over the last pair build: fsc_float[n] = sum of pair
 * probabilities, fsc_int[n] = rint(fsc_float), pair_prob[P] in export order
 * (each may be NULL).  Without pair_prob: no host sync, graph-capturable. */
int fos_surrogate_predict(FosCtx* ctx, const FosSurrogate* m, const float* rad, float* fsc_float,
                          int32_t* fsc_int, float* pair_prob, fos_stream_t s);
/* Counters of the last pair build and of the last judged JFA frame
 * (synchronises). */
int fos_surrogate_stats(FosCtx* ctx, FosSurrogateStats* out, fos_stream_t s);
/* A frame whose FSC between JFA runs comes from the surrogate.  Plain
 * dynamics as fos_frame; then
 *  - non-JFA frame: candidate pairs + inference on the new positions, the
 *    mode's FSC f (fos_surrogate_set_mode), fsc_ema <- alpha * f +
 *    (1 - alpha) * fsc_ema (EMA_ALPHA, same first-value rule as
 *    update_fsc_ema), and set_fsc_targets on rint(f) behind the same
 *    warm-start gate;
 *  - JFA frame: the surrogate's f for the same positions, then the exact
 *    run_jfa + gate + set_fsc_targets, then the judge counters (f vs the JFA
 *    fsc, and the previous JFA fsc vs this one) and the anchor update.
 * No host sync; the _graph form replays a captured CUDA graph. */
int fos_frame_surrogate(FosCtx* ctx, const FosState* st, const FosFrameParams* fp,
                        const FosSurrogate* m, int jfa_frame, fos_stream_t s);
int fos_frame_surrogate_graph(FosCtx* ctx, const FosState* st, const FosFrameParams* fp,
                              const FosSurrogate* m, int jfa_frame, fos_stream_t s);

/* ------------------------------------------------------- batched ensembles
 * No counterpart in the reference, which runs one foam per process.  Many
 * independent periodic foams, of uneven particle counts, JFA resolutions and
 * hash grids, advance together.  All foams share one device frame index and
 * take their JFA frames together, and every stage of a frame is ONE launch
 * over all foams:
 *   - the dynamics are one persistent cooperative kernel;
 *   - the JFA passes, filter and face extraction are one launch per stage;
 *   - the finalize is one cooperative kernel.
 * Each foam's result is bit-identical to the same foam run alone through
 * fos_frame with the same parameters.
 *
 * Layout: the foams' particles are packed (foam f owns the global indices
 * [part_off[f], part_off[f+1]) in the order given).  JFA labels, face_ids and
 * neighbor_list hold GLOBAL particle indices; subtract part_off[f] for a
 * foam's own numbering.  Every foam's voxel grid starts at a multiple of 1024
 * voxels in the packed label arrays, and every foam's hash grid at its own
 * offset in the packed cell table.
 *
 * Limits: one domain_size for all foams; early_exit must be 0 (every foam runs
 * all its passes); max_eq_nei <= 16. */
typedef struct FosEnsembleFoam {
    int n;              /* particles */
    int jfa_res;        /* JFA_RES of this foam */
    int grid_res;       /* GRID_RES (hash cells per axis) of this foam */
    int f_low, f_high;  /* FSC band */
    double r_min, r_max;
    uint64_t seed;      /* Philox key of its Brownian jitter */
} FosEnsembleFoam;

/* Launch shapes the autotuner chooses between (results do not depend on them). */
typedef struct FosEnsembleTuning {
    int pass_block;          /* threads per block of the JFA pass: 128, 256 or 512 */
    int voxel_block;         /* majority filter / face extraction: 128, 256 or 512 */
    int coop_threads;        /* dynamics kernel threads per block: 512 or 1024 */
    int coop_blocks_per_sm;  /* dynamics kernel blocks per SM: 1 or 2 (if resident) */
} FosEnsembleTuning;

/* Device pointers of the packed state (n_total particles). */
typedef struct FosEnsembleView {
    int nfoams, n_total;
    float* pos;                /* [n_total][3] */
    float* rad;                /* [n_total] */
    float* rad_target;
    float* local_max_depth;
    float* delta_r;
    int32_t* fsc;              /* [n_total] */
    float* fsc_ema;            /* [n_total] */
    int32_t* face_ids;         /* [n_total][32], global indices */
    int32_t* face_counts;      /* [n_total][32] */
    int32_t* neighbor_list;    /* [n_total][32], global indices */
    int32_t* labels_a;         /* packed owner grids (pass buffers A and B) */
    int32_t* labels_b;
    const int32_t* foam_of;    /* [n_total] foam of each particle */
} FosEnsembleView;

typedef struct FosEnsemble FosEnsemble;

/* p and fp hold the parameters all foams share (their per-foam fields --
 * grid_res, f_low/f_high, r_min/r_max, seed -- are taken from foams[]). */
int fos_ensemble_create(const FosParams* p, const FosFrameParams* fp,
                        const FosEnsembleFoam* foams, int nfoams, int device, FosEnsemble** out);
int fos_ensemble_destroy(FosEnsemble* e);
int fos_ensemble_view(FosEnsemble* e, FosEnsembleView* out);
/* Host arrays of nfoams + 1 entries: particle, voxel and hash-cell offsets. */
int fos_ensemble_offsets(FosEnsemble* e, int* part_off, long long* vox_off, int* cell_off);
/* fos_sim_init for every foam: zeroed fields, rad_target = rad, positions
 * wrapped, warmup_pbd PBD passes (one cooperative launch), frame index frame0. */
int fos_ensemble_init(FosEnsemble* e, int frame0, fos_stream_t s);
/* One frame of every foam (fos_frame's order); jfa_frame for all foams. */
int fos_ensemble_frame(FosEnsemble* e, int jfa_frame, fos_stream_t s);
/* The same frame replayed from a CUDA graph (one per frame kind and tuning). */
int fos_ensemble_frame_graph(FosEnsemble* e, int jfa_frame, fos_stream_t s);
int fos_ensemble_set_tuning(FosEnsemble* e, const FosEnsembleTuning* t);
int fos_ensemble_get_tuning(FosEnsemble* e, FosEnsembleTuning* t);
/* Record passes with four voxels a thread along x where a foam's R allows it
 * (on, the default; the pass block of the tuning then does not apply), or
 * one voxel a thread (off).  DOMAIN_SIZE 1 only; the labels are the same
 * either way.  No reference counterpart. */
int fos_ensemble_set_multi_voxel(FosEnsemble* e, int on);
/* fos_frame_surrogate for every foam of the ensemble (no reference
 * counterpart): the dynamics, then on a non-JFA frame the surrogate's FSC
 * (candidate pairs on each foam's own hash grid, inference, the mode's FSC),
 * its EMA and the targets; on a JFA frame the surrogate's estimate for the
 * same positions, the JFA with its targets, then the per-cell judging.  Each
 * foam's results equal the same foam's under fos_frame_surrogate. */
int fos_ensemble_frame_surrogate(FosEnsemble* e, const FosSurrogate* m, int jfa_frame,
                                 fos_stream_t s);
/* fos_surrogate_set_mode / fos_surrogate_stats over all foams of the ensemble. */
int fos_ensemble_surrogate_mode(FosEnsemble* e, int mode);
int fos_ensemble_surrogate_stats(FosEnsemble* e, FosSurrogateStats* out, fos_stream_t s);
/* Times every candidate shape of each tuned stage on the current state (the
 * JFA stages on this state's positions, the dynamics from a snapshot that is
 * restored afterwards), keeps the fastest per stage and applies it.
 * report_ms (optional, report_cap entries) receives, per candidate, the
 * stage's mean milliseconds in the order: pass_block 128/256/512,
 * voxel_block 128/256/512, coop (threads, blocks/SM) (512,1) (512,2)
 * (1024,1) (1024,2), a non-resident shape reporting -1.  Synchronises. */
int fos_ensemble_autotune(FosEnsemble* e, int reps, FosEnsembleTuning* best, float* report_ms,
                          int report_cap, fos_stream_t s);
/* Frame index (synchronises). */
int fos_ensemble_frame_index(FosEnsemble* e, int* frame, fos_stream_t s);
/* Tracing (no reference counterpart): the dynamics kernel of one plain frame
 * of every foam with a %globaltimer stamp, in ns, at kernel entry and after
 * every grid barrier (block 0's view), as fos_frame_trace.  Advances the
 * positions and radii as that kernel does, not the frame index; allocates a
 * scratch buffer and synchronises.  *count gets the number of stamps (<= cap
 * - 2); ns_host[cap - 2] holds the bitwise NOT of the earliest block's start
 * and ns_host[cap - 1] the latest block's end (cap >= 3). */
int fos_ensemble_trace(FosEnsemble* e, long long* ns_host, int cap, int* count, fos_stream_t s);
long long fos_ensemble_launch_count(FosEnsemble* e);

/* Number of this library's kernel launches issued so far on ctx (host count). */
long long fos_launch_count(FosCtx* ctx);
/* Device error word (synchronises) and a static string for a status code. */
int fos_device_error(FosCtx* ctx, int* word, fos_stream_t s);
/* Clear the device error word (stream-ordered); the context is usable again
 * once a failed launch has ended.  No reference counterpart: the reference
 * raises Taichi exceptions and has only an unused JFA_WATCHDOG_INTERVAL
 * (config.py:174). */
int fos_device_error_clear(FosCtx* ctx, fos_stream_t s);
/* For tests of the failure path, no reference counterpart.  With
 * leave_at_barrier = k >= 2, every later cooperative launch on ctx (the
 * frame's dynamics kernel, the finalize fixed point, the ensemble kernel)
 * makes its last block leave at its k-th grid barrier without arriving, and
 * bounds every wait from the second barrier on by about 1 ms instead of 1 s:
 * the other blocks record FOS_E_TIMEOUT in the error word and end.  Nothing
 * faults and nothing hangs.  0 turns the plan off (the default). */
int fos_test_barrier_plan(FosCtx* ctx, int leave_at_barrier, fos_stream_t s);
/* JFA passes (jfa_step_ping*, jfa.py:523-623) with the candidate record rows
 * staged in shared memory by tensor-memory-accelerator copies (on) or read
 * from global memory (off, the default: staging measured about 1.45x slower).
 * Staging applies to DOMAIN_SIZE 1 and power-of-two resolutions 32..256 under
 * the reference's tie rule; the labels are the same either way.  No
 * reference counterpart. */
int fos_set_jfa_staging(FosCtx* ctx, int on);
/* JFA record passes with four voxels a thread along x, sharing the candidate
 * rows of their common x-planes, or one voxel a thread.  mode 0: one voxel a
 * thread; 1 (the default): four where R^3 / 4 threads still fill the GPU
 * (R >= 128 on a B200); 2: four (two at the first step) at every R >= 16.
 * Applies to DOMAIN_SIZE 1 and power-of-two R under the reference's tie
 * rule; the labels are the same in every mode.  No reference counterpart. */
int fos_set_jfa_multi_voxel(FosCtx* ctx, int mode);
const char* fos_status_string(int status);
/* Thread-local text of the last error raised by any entry point. */
const char* fos_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* FOS_H */
