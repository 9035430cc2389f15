// frame.cu -- headless frame driver in run.py's order, graph capture, stats.
//
// Reference: run.py:699-1261 (the per-frame call sequence), jfa.py:1149-1195
// (run_jfa stats), jfa.py:1337-1426 (validate_jfa).
#include <math.h>
#include <string.h>

#include "phases.cuh"

// launchers defined in grid.cu / dynamics.cu
int fos_grid_build_from(FosCtx* c, const float* src, float* dst, int n, int32_t* cell_count,
                        int32_t* cell_start, int32_t* cell_indices, const float* rad,
                        cudaStream_t s);
int fos_launch_pbd(FosCtx* c, float* pout, const int32_t* cs, const int32_t* cc,
                   const int32_t* ci, int n, cudaStream_t s);
int fos_launch_max_overlap(FosCtx* c, const int32_t* cs, const int32_t* cc, const int32_t* ci,
                           float* lmd, int n, unsigned int* gmax_bits, cudaStream_t s);
int fos_launch_pressure(FosCtx* c, int n, int frame, const int* frame_ptr, float* rad,
                        float* delta_r, const int32_t* face_ids, const int32_t* fsc, float k,
                        float P, float cap, int max_nei, float rmin, float rmax, int sweeps,
                        cudaStream_t s);
int fos_launch_brownian(FosCtx* c, float* pos, int n, float strength, float domain, uint64_t seed,
                        int frame, const int* frame_ptr, FosDevState* tick, cudaStream_t s);
int fos_launch_set_targets(FosCtx* c, const float* rad, float* rt, const int32_t* fsc,
                           const float* ema, int n, int f_low, int f_high, float growth, float rmin,
                           float rmax, FosDevState* gate, int warm_frames, double zero_thresh,
                           int adjust_frames, cudaStream_t s);
int fos_launch_nudge(FosCtx* c, float* rad, const float* rt, const float* lmd, int n, float alpha,
                     float max_step, float rmin, float rmax, float back, const unsigned int* back_bits,
                     int mode, const FosDevState* gate, cudaStream_t s);
int fos_launch_wrap(FosCtx* c, float* pos, int n, cudaStream_t s);
int fos_launch_ou_frame(FosCtx* c, float* pos, float* vjit, const float* rad, int n,
                        const FosFrameParams* fp, cudaStream_t s);

extern "C" void fos_frame_params_default(FosFrameParams* fp) {
    if (!fp) return;
    memset(fp, 0, sizeof(*fp));
    fp->pbd_iters = 4;               // PBD_BASE_PASSES (config.py:342)
    fp->pressure_iters = 1;          // one equilibrate_pressure call per frame (run.py:755)
    fp->f_low = 8;                   // FSC_LOW (config.py:90)
    fp->f_high = 20;                 // FSC_HIGH (config.py:91)
    fp->growth_pct = 0.10;           // GROWTH_PCT
    fp->max_step_pct = 0.12;         // MAX_STEP_PCT
    fp->adjustment_frames = 15;      // ADJUSTMENT_FRAMES
    fp->bp_mode = 2;                 // BACKPRESSURE_MODE "local"
    fp->warmstart_frames = 30;       // WARMSTART_FRAMES
    fp->zero_rate_thresh = 0.10;     // FSC_ZERO_RATE_THRESH
    fp->r_min = 0.002;               // R_MIN_MANUAL
    fp->r_max = 0.010;               // R_MAX_MANUAL
    fp->pressure_k = 0.10;
    fp->pressure_exp = 3.0;
    fp->pressure_pair_cap = 0.02;
    fp->max_eq_nei = 10;
    fp->brownian_strength = 0.0002;  // BROWNIAN_STRENGTH
    fp->seed = 0;
    fp->warmup_pbd = 4;              // PBD_BASE_PASSES
    fp->ou_jitter = 0;               // JITTER_ENABLED is True in config.py:493; off here
    fp->jitter_rms = 0.10;           // JITTER_RMS (config.py:494)
    fp->jitter_tau = 1.0;            // JITTER_TAU (config.py:496)
    fp->dt = 0.016;                  // DT (config.py:400)
    fp->max_drift_fraction = 0.20;   // MAX_DRIFT_FRACTION (config.py:498)
    fp->jfa_warm_step = 4;           // first step of a warm-started JFA (jfa_frame == 2)
}

__global__ void k_frame_set(FosDevState* ds, int frame, int settle) {
    ds->frame = frame;
    ds->settle = settle;
    ds->error = 0;
}

__global__ void k_frame_end(FosDevState* ds) { ds->frame += 1; }

static int check_state(FosCtx* c, const FosState* st, const FosFrameParams* fp) {
    FOS_REQUIRE(c && st && fp, FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(st->n >= 1 && st->n <= c->max_n, FOS_E_CAPACITY, "state n outside [1, max_n]");
    FOS_REQUIRE(st->pos && st->rad && st->rad_target && st->local_max_depth && st->delta_r &&
                    st->cell_count && st->cell_start && st->cell_indices,
                FOS_E_ARG, "NULL state buffer");
    FOS_REQUIRE(fp->pbd_iters >= 0 && fp->pressure_iters >= 0, FOS_E_ARG, "negative iterations");
    FOS_REQUIRE(!fp->ou_jitter || st->v_jit, FOS_E_ARG, "ou_jitter needs FosState.v_jit");
    FOS_REQUIRE(fp->jfa_warm_step >= 0, FOS_E_ARG, "jfa_warm_step must be >= 0");
    FOS_REQUIRE(!fp->ou_jitter || (fp->dt > 0.0 && fp->jitter_tau >= 0.0), FOS_E_ARG,
                "ou_jitter needs dt > 0 and jitter_tau >= 0");
    return FOS_OK;
}

extern "C" int fos_sim_init(FosCtx* c, const FosState* st, const FosFrameParams* fp, int frame0,
                            fos_stream_t s) {
    int rc = check_state(c, st, fp);
    if (rc) return rc;
    int n = st->n;
    size_t NS = (size_t)n * FOS_S;
    // zero-initialised Taichi fields (jfa.py:120-204, run.py:129-195)
    FOS_CUDA(cudaMemsetAsync(c->fsc, 0, (size_t)n * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->used, 0, (size_t)n * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->ema, 0, (size_t)n * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->face_ids, 0, NS * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->face_counts, 0, NS * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->prev, 0, NS * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->nl, 0xFF, NS * 4, s));
    FOS_CUDA(cudaMemsetAsync(st->local_max_depth, 0, (size_t)n * 4, s));
    FOS_CUDA(cudaMemsetAsync(st->delta_r, 0, (size_t)n * 4, s));
    FOS_CUDA(cudaMemcpyAsync(st->rad_target, st->rad, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    // init_jitter_velocities (run.py:346)
    if (st->v_jit) FOS_CUDA(cudaMemsetAsync(st->v_jit, 0, (size_t)n * 12, s));
    k_frame_set<<<1, 1, 0, s>>>(c->ds, frame0, 0);
    FOS_LAUNCHED(c);
    // wrap_seeded_positions (run.py:233-237) + warmup_pbd (run.py:293-318)
    rc = fos_launch_wrap(c, st->pos, n, s);
    if (rc) return rc;
    for (int k = 0; k < fp->warmup_pbd; ++k) {
        rc = fos_grid_build_from(c, st->pos, st->pos, n, st->cell_count, st->cell_start,
                                 st->cell_indices, st->rad, s);
        if (rc) return rc;
        rc = fos_launch_pbd(c, c->pos_tmp, st->cell_start, st->cell_count, st->cell_indices, n, s);
        if (rc) return rc;
        FOS_CUDA(cudaMemcpyAsync(st->pos, c->pos_tmp, (size_t)n * 12, cudaMemcpyDeviceToDevice, s));
    }
    return FOS_OK;
}

static float alpha_for_frames(int frames) {  // run.py:440-452
    return (float)(1.0 - pow(0.05, 1.0 / (double)(frames > 1 ? frames : 1)));
}

// Optional per-stage event timing of a frame (fos_frame_profile).
struct FrameProf {
    cudaEvent_t ev[64];
    int stage[64];
    int k = 0;
    cudaStream_t s;
    void mark(int stage_id) {
        if (k < 64) {
            cudaEventRecord(ev[k], s);
            stage[k] = stage_id;
            ++k;
        }
    }
};

// part: bit 0 = dynamics (steps 1-7 and the OU jitter), bit 1 = measurement
// (step 8 on a JFA frame) and the end of the frame.
enum { FRAME_DYNAMICS = 1, FRAME_MEASURE = 2, FRAME_ALL = 3 };
static int frame_impl(FosCtx* c, const FosState* st, const FosFrameParams* fp, int jfa_frame,
                      cudaStream_t s, FrameProf* prof, const FosSurrogate* sur = nullptr,
                      int part = FRAME_ALL);

extern "C" int fos_frame(FosCtx* c, const FosState* st, const FosFrameParams* fp, int jfa_frame,
                         fos_stream_t s) {
    return frame_impl(c, st, fp, jfa_frame, s, nullptr);
}

extern "C" int fos_frame_dynamics(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                                  fos_stream_t s) {
    return frame_impl(c, st, fp, 0, s, nullptr, nullptr, FRAME_DYNAMICS);
}

extern "C" int fos_frame_measure(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                                 int jfa_frame, fos_stream_t s) {
    return frame_impl(c, st, fp, jfa_frame, s, nullptr, nullptr, FRAME_MEASURE);
}

extern "C" int fos_frame_surrogate(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                                   const FosSurrogate* m, int jfa_frame, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr && m != nullptr, FOS_E_ARG, "ctx or surrogate model is NULL");
    int rc = fos_sur_prepare(c);
    if (rc) return rc;
    return frame_impl(c, st, fp, jfa_frame, s, nullptr, m);
}

extern "C" int fos_frame_profile(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                                 int jfa_frame, float* stage_ms, fos_stream_t s) {
    FOS_REQUIRE(stage_ms != nullptr, FOS_E_ARG, "stage_ms is NULL");
    FrameProf prof;
    prof.s = s;
    for (int i = 0; i < 64; ++i) FOS_CUDA(cudaEventCreate(&prof.ev[i]));
    prof.mark(-1);
    int rc = frame_impl(c, st, fp, jfa_frame, s, &prof);
    if (rc == FOS_OK) {
        FOS_CUDA(cudaStreamSynchronize(s));
        for (int i = 0; i < FOS_FRAME_STAGES; ++i) stage_ms[i] = 0.f;
        for (int i = 1; i < prof.k; ++i) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, prof.ev[i - 1], prof.ev[i]);
            int st_id = prof.stage[i];
            if (st_id >= 0 && st_id < FOS_FRAME_STAGES) stage_ms[st_id] += ms;
        }
    }
    for (int i = 0; i < 64; ++i) cudaEventDestroy(prof.ev[i]);
    return rc;
}

static int frame_impl(FosCtx* c, const FosState* st, const FosFrameParams* fp, int jfa_frame,
                      cudaStream_t s, FrameProf* prof, const FosSurrogate* sur, int part) {
    int rc = check_state(c, st, fp);
    if (rc) return rc;
    FOS_REQUIRE(jfa_frame >= 0 && jfa_frame <= 2, FOS_E_ARG, "jfa_frame must be 0, 1 or 2");
    const int n = st->n;
#define MARK(id) \
    if (prof) prof->mark(id)
    const int* dframe = &c->ds->frame;
    bool coop_ends = false;
    if (!(part & FRAME_DYNAMICS)) {
        // measurement part only
    } else if (c->use_coop && !prof && fp->max_eq_nei <= 16 && !(fp->ou_jitter && fp->pbd_iters == 0) &&
        fos_coop_supported(c)) {
        // (1)-(7) as one persistent cooperative kernel (frame_coop.cu); a plain
        // frame ends there, and the kernel advances the frame counter itself
        coop_ends = (part & FRAME_MEASURE) && !jfa_frame && !sur;
        rc = fos_frame_coop_dynamics(c, st, fp, s, nullptr, 0, coop_ends ? 1 : 0);
        if (rc) return rc;
    } else {
        // (1) rebuild_grid (run.py:704)
        rc = fos_grid_build_from(c, st->pos, st->pos, n, st->cell_count, st->cell_start,
                                 st->cell_indices, st->rad, s);
        if (rc) return rc;
        MARK(0);
        // (2) compute_max_overlap (run.py:709, 737 in the defined argument order)
        rc = fos_launch_max_overlap(c, st->cell_start, st->cell_count, st->cell_indices,
                                    st->local_max_depth, n, &c->ds->omax_bits, s);
        if (rc) return rc;
        MARK(1);
        // (3) nudge_radii_adaptive_ema while settle_frames_left > 0 (run.py:744-750)
        rc = fos_launch_nudge(c, st->rad, st->rad_target, st->local_max_depth, n,
                              alpha_for_frames(fp->adjustment_frames), (float)fp->max_step_pct,
                              (float)fp->r_min, (float)fp->r_max, 1.0f, &c->ds->omax_bits, fp->bp_mode,
                              c->ds, s);
        if (rc) return rc;
        MARK(2);
        // (4) equilibrate_pressure x pressure_iters on the last JFA's face_ids/fsc (run.py:755-771)
        rc = fos_launch_pressure(c, n, 0, dframe, st->rad, st->delta_r, c->face_ids, c->fsc,
                                 (float)fp->pressure_k, (float)fp->pressure_exp,
                                 (float)fp->pressure_pair_cap, fp->max_eq_nei, (float)fp->r_min,
                                 (float)fp->r_max, fp->pressure_iters, s);
        if (rc) return rc;
        MARK(3);
        // (5) apply_brownian_motion (run.py:807-813); also settle_frames_left -= 1
        rc = fos_launch_brownian(c, st->pos, n, (float)fp->brownian_strength, c->L, fp->seed, 0,
                                 dframe, c->ds, s);
        if (rc) return rc;
        MARK(4);
        // (6) PBD passes, each on a fresh grid (run.py:829-846); (7) final rebuild (run.py:874)
        const float* src = st->pos;
        for (int k = 0; k < fp->pbd_iters; ++k) {
            rc = fos_grid_build_from(c, src, st->pos, n, st->cell_count, st->cell_start,
                                     st->cell_indices, st->rad, s);
            if (rc) return rc;
            MARK(0);
            rc = fos_launch_pbd(c, c->pos_tmp, st->cell_start, st->cell_count, st->cell_indices, n, s);
            if (rc) return rc;
            MARK(5);
            src = c->pos_tmp;
        }
        // (6B) OU jitter: apply_brownian + integrate_jitter (run.py:855-867)
        if (fp->ou_jitter) {
            rc = fos_launch_ou_frame(c, (float*)src, st->v_jit, st->rad, n, fp, s);
            if (rc) return rc;
            MARK(10);
        }
        rc = fos_grid_build_from(c, src, st->pos, n, st->cell_count, st->cell_start, st->cell_indices,
                                 nullptr, s);
        if (rc) return rc;
        MARK(0);
    }
    if (!(part & FRAME_MEASURE)) return FOS_OK;
    // surrogate frames: the learned FSC between JFA runs; on a JFA frame the
    // surrogate's estimate for the same positions, judged after the JFA
    if (sur && !jfa_frame) {
        rc = fos_sur_frame_between(c, sur, st, fp, s);
        if (rc) return rc;
    }
    if (sur && jfa_frame) {
        rc = fos_sur_frame_before_jfa(c, sur, st, fp, s);
        if (rc) return rc;
    }
    // (8) measurement frame: run_jfa, warm-start gate, set_fsc_targets, settle reset
    if (jfa_frame) {
        if (jfa_frame == 2) {
            rc = fos_jfa_warm(c, st->pos, st->rad, n, fp->jfa_warm_step, s);
            if (rc) return rc;
        } else {
            rc = fos_jfa_init(c, st->pos, st->rad, n, s);
            if (rc) return rc;
            rc = fos_jfa_passes(c, n, s);
            if (rc) return rc;
        }
        MARK(6);
        rc = fos_jfa_majority_filter(c, s);
        if (rc) return rc;
        rc = fos_jfa_accumulate_faces(c, n, s);
        if (rc) return rc;
        MARK(7);
        rc = fos_jfa_finalize_ema(c, st->rad, n, s);
        if (rc) return rc;
        MARK(8);
        rc = fos_launch_set_targets(c, st->rad, st->rad_target, c->fsc, c->ema, n, fp->f_low,
                                    fp->f_high, (float)fp->growth_pct, (float)fp->r_min,
                                    (float)fp->r_max, c->ds, fp->warmstart_frames,
                                    fp->zero_rate_thresh, fp->adjustment_frames, s);
        if (rc) return rc;
        if (sur) {
            rc = fos_sur_frame_judge(c, n, s);
            if (rc) return rc;
        }
    }
    if (!coop_ends) {
        k_frame_end<<<1, 1, 0, s>>>(c->ds);
        FOS_LAUNCHED(c);
    }
    MARK(9);
#undef MARK
    return FOS_OK;
}

// ------------------------------------------------------------ temporal skip
// Activity signals of run.py's temporal skip (run.py:913-951), one pass over
// the particles.  Each block writes its partial sums to its own slot; one
// thread adds the slots in block order, so the result does not depend on
// scheduling.
struct SkipPart {
    long long rad_fx;     // sum of radii, 2^-40 fixed point (exact)
    long long fsc_sum;
    double dr_sum, dr_sq;  // sum of |dr| and |dr|^2
    unsigned int vmax_bits;
    int oob, zero, pad;
};

__global__ void __launch_bounds__(256) k_skip_partial(const float* __restrict__ pos,
                                                      const float* __restrict__ rad,
                                                      const float* __restrict__ pos_prev,
                                                      const float* __restrict__ rad_prev,
                                                      const int32_t* __restrict__ fsc, int n,
                                                      int f_low, int f_high, float L, float halfL,
                                                      SkipPart* part) {
    long long rq = 0, fq = 0;
    double ds = 0.0, dq = 0.0;
    unsigned int vb = 0u;
    int oob = 0, zero = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float r = __ldg(&rad[i]);
        rq += rad_fixed(r);
        const int f = __ldg(&fsc[i]);
        fq += f;
        oob += (f < f_low || f > f_high) ? 1 : 0;
        zero += f == 0 ? 1 : 0;
        if (rad_prev) {
            const double a = (double)fabsf(fsub(r, __ldg(&rad_prev[i])));
            ds += a;
            dq += a * a;
        }
        if (pos_prev) {
            // pos_delta with the periodic fold of run.py:933-935, then its norm
            float d2 = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float d = fsub(__ldg(&pos[3 * i + k]), __ldg(&pos_prev[3 * i + k]));
                if (fabsf(d) > halfL) d = fsub(d, d > 0.f ? L : -L);
                d2 = k == 0 ? fmul(d, d) : fadd(d2, fmul(d, d));
            }
            const unsigned int b = __float_as_uint(__fsqrt_rn(d2));
            vb = b > vb ? b : vb;
        }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        rq += __shfl_xor_sync(0xffffffffu, rq, o);
        fq += __shfl_xor_sync(0xffffffffu, fq, o);
        ds += __shfl_xor_sync(0xffffffffu, ds, o);
        dq += __shfl_xor_sync(0xffffffffu, dq, o);
        oob += __shfl_xor_sync(0xffffffffu, oob, o);
        zero += __shfl_xor_sync(0xffffffffu, zero, o);
        unsigned int ob = __shfl_xor_sync(0xffffffffu, vb, o);
        vb = ob > vb ? ob : vb;
    }
    __shared__ SkipPart sw[8];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) sw[w] = SkipPart{rq, fq, ds, dq, vb, oob, zero, 0};
    __syncthreads();
    if (threadIdx.x == 0) {
        SkipPart t = sw[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            t.rad_fx += sw[k].rad_fx;
            t.fsc_sum += sw[k].fsc_sum;
            t.dr_sum += sw[k].dr_sum;
            t.dr_sq += sw[k].dr_sq;
            t.vmax_bits = sw[k].vmax_bits > t.vmax_bits ? sw[k].vmax_bits : t.vmax_bits;
            t.oob += sw[k].oob;
            t.zero += sw[k].zero;
        }
        part[blockIdx.x] = t;
    }
}

__global__ void k_skip_final(const SkipPart* part, int blocks, int n, int have_rad_prev,
                             int have_pos_prev, FosSkipSignals* out) {
    SkipPart t = part[0];
    for (int k = 1; k < blocks; ++k) {
        t.rad_fx += part[k].rad_fx;
        t.fsc_sum += part[k].fsc_sum;
        t.dr_sum += part[k].dr_sum;
        t.dr_sq += part[k].dr_sq;
        t.vmax_bits = part[k].vmax_bits > t.vmax_bits ? part[k].vmax_bits : t.vmax_bits;
        t.oob += part[k].oob;
        t.zero += part[k].zero;
    }
    const double dn = (double)(n > 1 ? n : 1);
    out->n = n;
    out->r_mean = (double)mean_from_fixed((unsigned long long)t.rad_fx, n);
    if (have_rad_prev) {
        const double m = t.dr_sum / dn;
        const double var = t.dr_sq / dn - m * m;
        out->sigma_dr = var > 0.0 ? sqrt(var) : 0.0;
    } else {
        out->sigma_dr = -1.0;
    }
    out->vmax_dt = have_pos_prev ? (double)__uint_as_float(t.vmax_bits) : -1.0;
    out->fsc_mean = (double)t.fsc_sum / dn;
    out->out_of_band = t.oob;
    out->zero_fsc = t.zero;
}

extern "C" int fos_skip_signals(FosCtx* c, const FosState* st, const float* pos_prev,
                                const float* rad_prev, int f_low, int f_high, FosSkipSignals* out,
                                fos_stream_t s) {
    FOS_REQUIRE(c && st && out && st->pos && st->rad, FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(st->n >= 1 && st->n <= c->max_n, FOS_E_CAPACITY, "state n outside [1, max_n]");
    const int n = st->n;
    int blocks = fos_blocks(n, 256);
    if (blocks > FOS_SKIP_BLOCKS) blocks = FOS_SKIP_BLOCKS;
    SkipPart* part = (SkipPart*)c->skip_part;
    k_skip_partial<<<blocks, 256, 0, s>>>(st->pos, st->rad, pos_prev, rad_prev, c->fsc, n, f_low,
                                          f_high, c->L, c->halfL, part);
    FOS_LAUNCHED(c);
    FosSkipSignals* dout = (FosSkipSignals*)(part + FOS_SKIP_BLOCKS);
    k_skip_final<<<1, 1, 0, s>>>(part, blocks, n, rad_prev != nullptr, pos_prev != nullptr, dout);
    FOS_LAUNCHED(c);
    FosSkipSignals* h = (FosSkipSignals*)c->pinned;
    FOS_CUDA(cudaMemcpyAsync(h, dout, sizeof(FosSkipSignals), cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaStreamSynchronize(s));
    *out = *h;
    return FOS_OK;
}

static int frame_graph_impl(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                            const FosSurrogate* sur, int jfa_frame, cudaStream_t s);

extern "C" int fos_frame_graph(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                               int jfa_frame, fos_stream_t s) {
    return frame_graph_impl(c, st, fp, nullptr, jfa_frame, s);
}

extern "C" int fos_frame_surrogate_graph(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                                         const FosSurrogate* m, int jfa_frame, fos_stream_t s) {
    FOS_REQUIRE(m != nullptr, FOS_E_ARG, "surrogate model is NULL");
    return frame_graph_impl(c, st, fp, m, jfa_frame, s);
}

static int frame_graph_impl(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                            const FosSurrogate* sur, int jfa_frame, cudaStream_t s) {
    int rc = check_state(c, st, fp);
    if (rc) return rc;
    if (sur) {
        rc = fos_sur_prepare(c);  // allocation stays outside the capture
        if (rc) return rc;
    }
    FOS_REQUIRE(jfa_frame >= 0 && jfa_frame <= 2, FOS_E_ARG, "jfa_frame must be 0, 1 or 2");
    int g = jfa_frame + (sur ? 3 : 0);
    FosGraphKey key;
    memset(&key, 0, sizeof(key));
    key.st = *st;
    key.fp = *fp;
    key.sur = sur;
    key.sur_mode = sur ? c->sur_mode : 0;
    key.jfa = g;
    key.res = c->res;
    key.p = c->p;
    if (!c->gvalid[g] || memcmp(&key, &c->gkey[g], sizeof(key)) != 0) {
        if (c->gexec[g]) {
            cudaGraphExecDestroy(c->gexec[g]);
            c->gexec[g] = nullptr;
        }
        cudaStream_t cap;
        FOS_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        long long before = c->launches;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            cudaStreamDestroy(cap);
            return fos_cuda_fail(e, "cudaStreamBeginCapture", __FILE__, __LINE__);
        }
        rc = frame_impl(c, st, fp, jfa_frame, cap, nullptr, sur);
        cudaGraph_t graph = nullptr;
        e = cudaStreamEndCapture(cap, &graph);
        cudaStreamDestroy(cap);
        long long captured = c->launches - before;
        c->launches = before;
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return fos_cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        e = cudaGraphInstantiate(&c->gexec[g], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fos_cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__);
        c->gkey[g] = key;
        c->gvalid[g] = true;
        c->glaunch[g] = captured;
    }
    FOS_CUDA(cudaGraphLaunch(c->gexec[g], s));
    c->launches += c->glaunch[g];
    return FOS_OK;
}

extern "C" int fos_sim_set_counters(FosCtx* c, int frame, int settle, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(frame >= 0 && settle >= 0, FOS_E_ARG, "negative counter");
    k_frame_set<<<1, 1, 0, s>>>(c->ds, frame, settle);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_sim_counters(FosCtx* c, int* frame, int* settle, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    int* h = (int*)c->pinned;
    FOS_CUDA(cudaMemcpyAsync(h, c->ds, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaStreamSynchronize(s));
    if (frame) *frame = h[0];
    if (settle) *settle = h[1];
    return FOS_OK;
}

// ------------------------------------------------------------------ stats
// One pass over particles for compute_pair_symmetry, compute_overflow_count,
// compute_fsc_stats and the first pass of compute_score_stats
// (jfa.py:1204-1330); sums in double, min/max exact.
struct JfaStatAcc {
    double sum_fsc, sum_ema, sum_score, sum_sq;
    long long p_dir, count_scores;
    int overflow, min_fsc, max_fsc, pad;
};

__global__ void k_jfa_stats1(int n, const int32_t* __restrict__ used, const int32_t* __restrict__ fsc,
                             const float* __restrict__ ema, const int32_t* __restrict__ face_ids,
                             const int32_t* __restrict__ face_counts, const float* __restrict__ rad,
                             float vs, float face_scale, JfaStatAcc* acc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int u = used[i];
    atomicAdd((unsigned long long*)&acc->p_dir, (unsigned long long)u);
    if (u >= FOS_S) atomicAdd(&acc->overflow, 1);
    int f = fsc[i];
    atomicAdd(&acc->sum_fsc, (double)f);
    atomicAdd(&acc->sum_ema, (double)ema[i]);
    atomicMin(&acc->min_fsc, f);
    atomicMax(&acc->max_fsc, f);
    // compute_score_stats scans face slots 0..used-1 (jfa.py:1273-1290)
    for (int s = 0; s < u && s < FOS_S; ++s) {
        int j = face_ids[(size_t)i * FOS_S + s];
        if (j >= 0 && j < n) {
            int v = face_counts[(size_t)i * FOS_S + s];
            if (v > 0) {
                float rm = fmul(0.5f, fadd(rad[i], rad[j]));
                float q = fdiv(fmul(2.0f, rm), vs);
                float e = fmul(face_scale, fmul(q, q));
                if (e > 0.0f) {
                    atomicAdd(&acc->sum_score, (double)fdiv((float)v, e));
                    atomicAdd((unsigned long long*)&acc->count_scores, 1ull);
                }
            }
        }
    }
}

__global__ void k_jfa_stats2(int n, const int32_t* __restrict__ used,
                             const int32_t* __restrict__ face_ids,
                             const int32_t* __restrict__ face_counts, const float* __restrict__ rad,
                             float vs, float face_scale, JfaStatAcc* acc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double mean = acc->count_scores > 0 ? acc->sum_score / (double)acc->count_scores : 0.0;
    int u = used[i];
    for (int s = 0; s < u && s < FOS_S; ++s) {
        int j = face_ids[(size_t)i * FOS_S + s];
        if (j >= 0 && j < n) {
            int v = face_counts[(size_t)i * FOS_S + s];
            if (v > 0) {
                float rm = fmul(0.5f, fadd(rad[i], rad[j]));
                float q = fdiv(fmul(2.0f, rm), vs);
                float e = fmul(face_scale, fmul(q, q));
                if (e > 0.0f) {
                    double d = (double)fdiv((float)v, e) - mean;
                    atomicAdd(&acc->sum_sq, d * d);
                }
            }
        }
    }
}

extern "C" int fos_jfa_stats(FosCtx* c, int n, const float* rad, FosJfaStats* out, fos_stream_t s) {
    FOS_REQUIRE(c && out && (n == 0 || rad), FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(n >= 0 && n <= c->max_n, FOS_E_CAPACITY, "n outside [0, max_n]");
    JfaStatAcc* acc = (JfaStatAcc*)c->stats_f;  // 64 floats = 256 bytes of scratch
    JfaStatAcc init;
    memset(&init, 0, sizeof(init));
    init.min_fsc = 999999;  // compute_fsc_stats initial min/max (jfa.py:1246-1247)
    init.max_fsc = -1;
    JfaStatAcc* h = (JfaStatAcc*)c->pinned;
    *h = init;
    FOS_CUDA(cudaMemcpyAsync(acc, h, sizeof(init), cudaMemcpyHostToDevice, s));
    if (n > 0) {
        k_jfa_stats1<<<fos_blocks(n, 256), 256, 0, s>>>(n, c->used, c->fsc, c->ema, c->face_ids,
                                                        c->face_counts, rad, c->vs, c->face_scale,
                                                        acc);
        FOS_LAUNCHED(c);
        k_jfa_stats2<<<fos_blocks(n, 256), 256, 0, s>>>(n, c->used, c->face_ids, c->face_counts,
                                                        rad, c->vs, c->face_scale, acc);
        FOS_LAUNCHED(c);
    }
    char* hb = (char*)c->pinned;
    FOS_CUDA(cudaMemcpyAsync(hb, acc, sizeof(JfaStatAcc), cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaMemcpyAsync(hb + 256, c->ds, sizeof(FosDevState), cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaStreamSynchronize(s));
    JfaStatAcc a;
    memcpy(&a, hb, sizeof(a));
    FosDevState d;
    memcpy(&d, hb + 256, sizeof(d));
    memset(out, 0, sizeof(*out));
    out->num_passes = d.passes_done;
    out->early_exit = d.early_exited;
    for (int p = 0; p < FOS_MAX_PASSES; ++p) out->changes[p] = (long long)d.changes[p];
    out->jfa_res = c->res;
    out->voxel_size = c->vs;
    double nn = (double)(n > 0 ? n : 1);
    out->mean_score = a.count_scores > 0 ? (float)(a.sum_score / (double)a.count_scores) : 0.f;
    out->std_score = a.count_scores > 0 ? (float)sqrt(a.sum_sq / (double)a.count_scores) : 0.f;
    out->p_dir = (int)a.p_dir;
    out->p_und_accepted = (int)(a.p_dir / 2);
    out->overflow_count = a.overflow;
    out->overflow_pct = (float)(100.0 * a.overflow / nn);
    out->mean_fsc = (float)(a.sum_fsc / nn);
    out->min_fsc = a.min_fsc;
    out->max_fsc = a.max_fsc;
    out->mean_fsc_ema = (float)(a.sum_ema / nn);
    out->finalize_iterations = d.fin_iters;
    out->face_pairs = d.pair_count;
    out->max_row_candidates = d.max_rowcnt;
    out->zero_fsc_count = d.zero_fsc;
    return d.error ? fos_fail(d.error, "device error word set during the last JFA run") : FOS_OK;
}

// check_symmetry / check_overflow / check_self_loops (jfa.py:1337-1397)
__global__ void k_validate(int n, const int32_t* __restrict__ nl, const int32_t* __restrict__ used,
                           int* out3) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int asym = 0, self = 0;
    for (int s = 0; s < FOS_S; ++s) {
        int j = nl[(size_t)i * FOS_S + s];
        if (j == i) self++;
        if (j >= 0 && j < n) {
            bool found = false;
            for (int k = 0; k < FOS_S && !found; ++k) found = nl[(size_t)j * FOS_S + k] == i;
            if (!found) asym++;
        }
    }
    if (asym) atomicAdd(&out3[0], asym);
    if (used[i] >= FOS_S) atomicAdd(&out3[1], 1);
    if (self) atomicAdd(&out3[2], self);
}

extern "C" int fos_jfa_validate(FosCtx* c, int n, FosValidate* out, fos_stream_t s) {
    FOS_REQUIRE(c && out, FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(n >= 0 && n <= c->max_n, FOS_E_CAPACITY, "n outside [0, max_n]");
    int* d = c->stats_i + 32;
    FOS_CUDA(cudaMemsetAsync(d, 0, 3 * sizeof(int), s));
    if (n > 0) {
        k_validate<<<fos_blocks(n, 128), 128, 0, s>>>(n, c->nl, c->used, d);
        FOS_LAUNCHED(c);
    }
    int* h = (int*)c->pinned;
    FOS_CUDA(cudaMemcpyAsync(h, d, 3 * sizeof(int), cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaStreamSynchronize(s));
    out->asymmetric_pairs = h[0];
    out->overflow_count = h[1];
    out->self_loops = h[2];
    out->passed = (h[1] == 0 && h[2] == 0) ? 1 : 0;
    return FOS_OK;
}
