// dynamics.cu -- PBD overlap projection, max overlap, Jacobi pressure
// diffusion, Brownian jitter and the FSC radius controller as standalone
// kernels (the per-element arithmetic lives in phases.cuh).
//
// Reference: dynamics.py.  All neighbour work is a gather over the sorted
// hash-grid cells (27-cell stencil, cells in (dx, dy, dz) order, dz fastest,
// particles ascending inside a cell), in the reference's accumulation order.
#include <string.h>

#include "phases.cuh"

// project_overlaps (dynamics.py:77-171) as one Jacobi sweep, one warp per
// particle (sorted position kk); see pbd_warp.
__global__ void __launch_bounds__(256) k_pbd(const float4* __restrict__ sp,
                                             const int32_t* __restrict__ ci,
                                             float* __restrict__ pout, int n, GridGeom g,
                                             const int32_t* __restrict__ cs,
                                             const int32_t* __restrict__ cc, float gap1, float mdf,
                                             float dmul) {
    int kk = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (kk >= n) return;  // warp-uniform
    pbd_warp<LdRO>(kk, threadIdx.x & 31, sp, ci, pout, g, cs, cc, gap1, mdf, dmul);
}

// compute_local_max_overlaps + reduce_max_depth (dynamics.py:304-372).
__global__ void __launch_bounds__(256) k_max_overlap(const float4* __restrict__ sp,
                                                     const int32_t* __restrict__ ci, int n,
                                                     GridGeom g, const int32_t* __restrict__ cs,
                                                     const int32_t* __restrict__ cc, float eps,
                                                     float* __restrict__ lmd,
                                                     unsigned int* gmax_bits) {
    int kk = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    unsigned int b = 0u;
    if (kk < n) b = maxov_warp<LdRO>(kk, threadIdx.x & 31, sp, ci, g, cs, cc, eps, lmd);
    block_max_atomic(b, gmax_bits);
}

// equilibrate_pressure (dynamics.py:1454-1557), one Jacobi sweep, GS lanes
// per particle.  With pmax != NULL the sweep also reports max |dr| and the
// count of |dr| > 1e-12 (block-reduced, one atomic pair per block).
template <int GS>
__global__ void __launch_bounds__(256) k_pressure(PressureArgs a, const int* frame_ptr,
                                                  const float* __restrict__ rin,
                                                  float* __restrict__ rout,
                                                  float* __restrict__ delta_r, unsigned int* pmax,
                                                  int* pchanged) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int lane = threadIdx.x & 31;
    if (frame_ptr) a.frame = *frame_ptr;
    int i = (int)(tid / GS);
    float d = pressure_group<GS, LdRO>(i, lane, a, rin, rout, delta_r);
    if (pmax) {
        float ad = fabsf(d);
        int ch = (i < a.n && (lane & (GS - 1)) == 0) && ad > 1e-12f;
        int cnt = __syncthreads_count(ch);
        unsigned int bm = __reduce_max_sync(0xffffffffu, ch ? __float_as_uint(ad) : 0u);
        block_max_atomic(bm, pmax);
        if (threadIdx.x == 0 && cnt) atomicAdd(pchanged, cnt);
    }
}

// apply_brownian_motion (dynamics.py:1596-1634).  With tick != NULL, thread 0
// also decrements the device settle counter (run.py:750), which the frame's
// nudge already read.
__global__ void k_brownian(float* pos, int n, float strength, float domain, float halfL,
                           uint32_t k0, uint32_t k1, int frame_arg, const int* frame_ptr,
                           FosDevState* tick) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (tick && i == 0 && tick->settle > 0) tick->settle -= 1;
    if (i >= n) return;
    unsigned int frame = (unsigned int)(frame_ptr ? *frame_ptr : frame_arg);
    brownian_one<LdRO>(i, (unsigned int)i, pos, strength, domain, halfL, k0, k1, frame);
}

// Sum of the radii as 2^-40 fixed-point integers (compute_mean_radius,
// dynamics.py:675-689): warp sums, one 64-bit atomic per warp.
__global__ void __launch_bounds__(256) k_rad_sum(const float* __restrict__ rad, int n,
                                                 unsigned long long* sum) {
    long long q = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        q += rad_fixed(__ldg(&rad[i]));
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    if ((threadIdx.x & 31) == 0 && q) atomicAdd(sum, (unsigned long long)q);
}

__global__ void k_mean_from_sum(const unsigned long long* sum, int n, float* mean) {
    *mean = mean_from_fixed(*sum, n);
}

// apply_brownian (dynamics.py:607-646), mean radius from a device float.
__global__ void k_ou_velocity(float* vjit, const float* __restrict__ rad, const float* mean, int n,
                              OuParams o, unsigned int frame) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float kick = ou_kick(o, *mean);
    float3 v = make_float3(vjit[3 * i + 0], vjit[3 * i + 1], vjit[3 * i + 2]);
    v = ou_velocity((unsigned int)i, v, __ldg(&rad[i]), kick, o, frame);
    vjit[3 * i + 0] = v.x;
    vjit[3 * i + 1] = v.y;
    vjit[3 * i + 2] = v.z;
}

// integrate_jitter (dynamics.py:649-660)
__global__ void k_ou_move(float* pos, const float* __restrict__ vjit, int n, OuParams o) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 p = make_float3(pos[3 * i + 0], pos[3 * i + 1], pos[3 * i + 2]);
    float3 v = make_float3(__ldg(&vjit[3 * i + 0]), __ldg(&vjit[3 * i + 1]),
                           __ldg(&vjit[3 * i + 2]));
    p = ou_move(p, v, o);
    pos[3 * i + 0] = p.x;
    pos[3 * i + 1] = p.y;
    pos[3 * i + 2] = p.z;
}

// Frame step 6B (run.py:855-867): apply_brownian + integrate_jitter fused,
// the mean radius from the fixed-point sum and the frame index from the
// device counter.
__global__ void k_ou_frame(float* pos, float* vjit, const float* __restrict__ rad, int n,
                           const unsigned long long* sum, const int* frame_ptr, OuParams o) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float kick = ou_kick(o, mean_from_fixed(*sum, n));
    float3 p = make_float3(pos[3 * i + 0], pos[3 * i + 1], pos[3 * i + 2]);
    p = ou_one(i, (unsigned int)i, p, vjit, __ldg(&rad[i]), kick, o, (unsigned int)*frame_ptr);
    pos[3 * i + 0] = p.x;
    pos[3 * i + 1] = p.y;
    pos[3 * i + 2] = p.z;
}

// set_fsc_targets (dynamics.py:1242-1320).  With gate != NULL it runs only
// when the warm-start gate (run.py:1184-1197) is open -- frame >=
// warm_frames and zero-FSC fraction <= zero_thresh -- and then also resets
// the settle counter to adjust_frames (run.py:1231).
__global__ void k_set_targets(const float* __restrict__ rad, float* __restrict__ rt,
                              const int32_t* __restrict__ fsc, const float* __restrict__ ema,
                              int n, int f_low, int f_high, float growth, float rmin, float rmax,
                              float db, FosDevState* gate, int warm_frames, double zero_thresh,
                              int adjust_frames) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (gate) {
        double f0 = (double)gate->zero_fsc / (double)(n > 0 ? n : 1);
        bool warm = (gate->frame < warm_frames) || (f0 > zero_thresh);
        if (warm) return;
        if (i == 0) gate->settle = adjust_frames;  // settle is not read by this kernel
    }
    if (i >= n) return;
    rt[i] = target_one(rad[i], ema[i], fsc[i], f_low, f_high, growth, rmin, rmax, db);
}

// nudge_radii_adaptive_ema (dynamics.py:1366-1427).  back_global is taken
// from back_bits (the device max overlap, run.py:454-470) when non-NULL.  With
// gate != NULL it is a no-op unless the settle counter is > 0.
__global__ void k_nudge(float* rad, const float* __restrict__ rt, const float* __restrict__ lmd,
                        int n, float alpha, float max_step, float rmin, float rmax, float back_arg,
                        const unsigned int* back_bits, double contact_tol_d, int mode,
                        float contact_tol, const FosDevState* gate) {
    if (gate && gate->settle <= 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float back = back_arg;
    if (back_bits && mode == 1) back = back_global_from_bits(*back_bits, contact_tol_d);
    rad[i] = nudge_one(rad[i], rt[i], lmd[i], alpha, max_step, rmin, rmax, back, mode,
                       contact_tol);
}

// compute_controller_stats (dynamics.py:1322-1363); sums in double.
__global__ void k_controller_stats(const float* __restrict__ rad, const float* __restrict__ rt,
                                   const float* __restrict__ ema, int n, int f_low, int f_high,
                                   int* counts, double* sum, unsigned int* maxbits) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float f = ema[i];
    float dr = fsub(rt[i], rad[i]);
    if (f < (float)f_low) atomicAdd(&counts[0], 1);
    else if (f > (float)f_high) atomicAdd(&counts[1], 1);
    else atomicAdd(&counts[2], 1);
    atomicAdd(sum, (double)dr);
    atomicMax(maxbits, __float_as_uint(fabsf(dr)));
}

__global__ void k_minmax(const float* __restrict__ v, int n, unsigned int* mn, unsigned int* mx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned int b = float_order_key(v[i]);
    atomicMin(mn, b);
    atomicMax(mx, b);
}

__global__ void k_wrap_positions(float* pos, int n, float L, float invL) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * n) return;
    pos[i] = grid_wrap(pos[i], L, invL);
}

// ------------------------------------------------------------ host side
static int check_dyn(FosCtx* c, int n) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(n >= 0 && n <= c->max_n, FOS_E_CAPACITY, "n outside [0, max_n]");
    return FOS_OK;
}

int fos_grid_gather_sorted(FosCtx* c, const int32_t* idx, const float* pos, const float* rad,
                           int n, cudaStream_t s);

// PBD sweep over the cell-ordered copy ctx->sorted (must match cs/cc/ci).
int fos_launch_pbd(FosCtx* c, float* pout, const int32_t* cs, const int32_t* cc,
                   const int32_t* ci, int n, cudaStream_t s) {
    if (n == 0) return FOS_OK;
    GridGeom g{c->G, c->L, c->invL, c->halfL};
    k_pbd<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(c->sorted, ci, pout, n, g, cs, cc, c->gap1,
                                                    c->mdf, c->dmul);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// Max overlap over the cell-ordered copy ctx->sorted (must match cs/cc/ci).
int fos_launch_max_overlap(FosCtx* c, const int32_t* cs, const int32_t* cc, const int32_t* ci,
                           float* lmd, int n, unsigned int* gmax_bits, cudaStream_t s) {
    FOS_CUDA(cudaMemsetAsync(gmax_bits, 0, 4, s));
    if (n == 0) return FOS_OK;
    GridGeom g{c->G, c->L, c->invL, c->halfL};
    k_max_overlap<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(c->sorted, ci, n, g, cs, cc, c->eps, lmd,
                                                            gmax_bits);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// `sweeps` pressure sweeps ping-ponging rad <-> rad_tmp; the result ends in rad.
int fos_launch_pressure(FosCtx* c, int n, int frame, const int* frame_ptr, float* rad,
                        float* delta_r, const int32_t* face_ids, const int32_t* fsc, float k,
                        float P, float cap, int max_nei, float rmin, float rmax, int sweeps,
                        cudaStream_t s) {
    if (n == 0 || sweeps <= 0) return FOS_OK;
    // stats (max |dr|, changed count) are those of the last sweep, as one
    // equilibrate_pressure call returns them; earlier sweeps skip them.
    unsigned int* pmax = &c->ds->maxabs_dr_bits;
    int* pch = &c->ds->changed;
    FOS_CUDA(cudaMemsetAsync(pch, 0, 2 * sizeof(int), s));  // changed, maxabs_dr_bits
    for (int w = 0; w < sweeps; ++w) {
        const float* rin = (w & 1) ? c->rad_tmp : rad;
        float* rout = (w & 1) ? rad : c->rad_tmp;
        bool last = (w == sweeps - 1);
        PressureArgs a{n, frame, max_nei, k, P, cap, rmin, rmax, face_ids, fsc, 0};
        if (max_nei <= 16)
            k_pressure<16><<<fos_blocks(16LL * n, 256), 256, 0, s>>>(
                a, frame_ptr, rin, rout, delta_r, last ? pmax : nullptr, last ? pch : nullptr);
        else
            k_pressure<32><<<fos_blocks(32LL * n, 256), 256, 0, s>>>(
                a, frame_ptr, rin, rout, delta_r, last ? pmax : nullptr, last ? pch : nullptr);
        FOS_LAUNCHED(c);
    }
    if (sweeps & 1)
        FOS_CUDA(cudaMemcpyAsync(rad, c->rad_tmp, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    return FOS_OK;
}

int fos_launch_brownian(FosCtx* c, float* pos, int n, float strength, float domain, uint64_t seed,
                        int frame, const int* frame_ptr, FosDevState* tick, cudaStream_t s) {
    float halfL = (float)(0.5 * (double)domain);
    k_brownian<<<fos_blocks(n > 0 ? n : 1, 256), 256, 0, s>>>(pos, n, strength, domain, halfL,
                                                              (uint32_t)seed, (uint32_t)(seed >> 32),
                                                              frame, frame_ptr, tick);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

static int launch_rad_sum(FosCtx* c, const float* rad, int n, cudaStream_t s) {
    FOS_CUDA(cudaMemsetAsync(&c->ds->rad_sum, 0, sizeof(unsigned long long), s));
    int blocks = fos_blocks(n > 0 ? n : 1, 256);
    if (blocks > 2 * c->num_sms) blocks = 2 * c->num_sms;
    k_rad_sum<<<blocks, 256, 0, s>>>(rad, n, &c->ds->rad_sum);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// Frame step 6B: mean radius, then the fused OU update of every particle.
int fos_launch_ou_frame(FosCtx* c, float* pos, float* vjit, const float* rad, int n,
                        const FosFrameParams* fp, cudaStream_t s) {
    if (n == 0) return FOS_OK;
    int rc = launch_rad_sum(c, rad, n, s);
    if (rc) return rc;
    OuParams o = ou_params(fp->jitter_rms, fp->jitter_tau, fp->max_drift_fraction,
                           c->p.gap_fraction, (float)fp->dt, c->L, c->invL, fp->seed);
    k_ou_frame<<<fos_blocks(n, 256), 256, 0, s>>>(pos, vjit, rad, n, &c->ds->rad_sum,
                                                  &c->ds->frame, o);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

int fos_launch_set_targets(FosCtx* c, const float* rad, float* rt, const int32_t* fsc,
                           const float* ema, int n, int f_low, int f_high, float growth, float rmin,
                           float rmax, FosDevState* gate, int warm_frames, double zero_thresh,
                           int adjust_frames, cudaStream_t s) {
    k_set_targets<<<fos_blocks(n > 0 ? n : 1, 256), 256, 0, s>>>(
        rad, rt, fsc, ema, n, f_low, f_high, growth, rmin, rmax, c->deadband, gate, warm_frames,
        zero_thresh, adjust_frames);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

int fos_launch_nudge(FosCtx* c, float* rad, const float* rt, const float* lmd, int n, float alpha,
                     float max_step, float rmin, float rmax, float back, const unsigned int* back_bits,
                     int mode, const FosDevState* gate, cudaStream_t s) {
    if (n == 0) return FOS_OK;
    k_nudge<<<fos_blocks(n, 256), 256, 0, s>>>(rad, rt, lmd, n, alpha, max_step, rmin, rmax, back,
                                               back_bits, c->p.contact_tol, mode, c->contact_tol,
                                               gate);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

int fos_launch_wrap(FosCtx* c, float* pos, int n, cudaStream_t s) {
    if (n == 0) return FOS_OK;
    k_wrap_positions<<<fos_blocks(3LL * n, 256), 256, 0, s>>>(pos, n, c->L, c->invL);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_project_overlaps(FosCtx* c, float* pos, const float* rad, const int32_t* cs,
                                    const int32_t* cc, const int32_t* ci, int n, fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (pos && rad && cs && cc && ci), FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    rc = fos_grid_gather_sorted(c, ci, pos, rad, n, s);
    if (rc) return rc;
    rc = fos_launch_pbd(c, c->pos_tmp, cs, cc, ci, n, s);
    if (rc) return rc;
    FOS_CUDA(cudaMemcpyAsync(pos, c->pos_tmp, (size_t)n * 12, cudaMemcpyDeviceToDevice, s));
    return FOS_OK;
}

extern "C" int fos_compute_max_overlap(FosCtx* c, const float* pos, const float* rad,
                                       const int32_t* cs, const int32_t* cc, const int32_t* ci,
                                       float* lmd, int n, float* max_dev, float* max_host,
                                       fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (pos && rad && cs && cc && ci && lmd), FOS_E_ARG, "NULL argument");
    unsigned int* bits = &c->ds->omax_bits;
    rc = fos_grid_gather_sorted(c, ci, pos, rad, n, s);
    if (rc) return rc;
    rc = fos_launch_max_overlap(c, cs, cc, ci, lmd, n, bits, s);
    if (rc) return rc;
    if (max_dev) FOS_CUDA(cudaMemcpyAsync(max_dev, bits, 4, cudaMemcpyDeviceToDevice, s));
    if (max_host) {
        float* h = (float*)c->pinned;
        FOS_CUDA(cudaMemcpyAsync(h, bits, 4, cudaMemcpyDeviceToHost, s));
        FOS_CUDA(cudaStreamSynchronize(s));
        *max_host = *h;
    }
    return FOS_OK;
}

extern "C" int fos_equilibrate_pressure(FosCtx* c, int n, int frame, float* rad, float* delta_r,
                                        const int32_t* face_ids, const int32_t* fsc, float k,
                                        float p_exp, float pair_cap, int max_nei, float r_min,
                                        float r_max, int sweeps, float* max_abs_dr_host,
                                        int* changed_host, fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (rad && delta_r && face_ids && fsc), FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(sweeps >= 0, FOS_E_ARG, "sweeps must be >= 0");
    rc = fos_launch_pressure(c, n, frame, nullptr, rad, delta_r, face_ids, fsc, k, p_exp, pair_cap,
                             max_nei, r_min, r_max, sweeps, s);
    if (rc) return rc;
    if (max_abs_dr_host || changed_host) {
        int* h = (int*)c->pinned;
        FOS_CUDA(cudaMemcpyAsync(h, &c->ds->changed, 8, cudaMemcpyDeviceToHost, s));
        FOS_CUDA(cudaStreamSynchronize(s));
        // FosDevState: changed then maxabs_dr_bits, adjacent
        if (changed_host) *changed_host = (n == 0 || sweeps == 0) ? 0 : h[0];
        if (max_abs_dr_host) {
            unsigned int b = (unsigned int)h[1];
            float f;
            memcpy(&f, &b, 4);
            *max_abs_dr_host = (n == 0 || sweeps == 0) ? 0.f : f;
        }
    }
    return FOS_OK;
}

extern "C" int fos_apply_brownian(FosCtx* c, float* pos, int n, float strength, float domain_size,
                                  uint64_t seed, uint32_t frame, fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || pos, FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    return fos_launch_brownian(c, pos, n, strength, domain_size, seed, (int)frame, nullptr, nullptr,
                               s);
}

extern "C" int fos_init_jitter_velocities(FosCtx* c, float* v_jit, int n, fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || v_jit, FOS_E_ARG, "NULL argument");
    if (n) FOS_CUDA(cudaMemsetAsync(v_jit, 0, (size_t)n * 12, s));
    return FOS_OK;
}

extern "C" int fos_compute_mean_radius(FosCtx* c, const float* rad, int n, float* mean_radius,
                                       fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(mean_radius && (n == 0 || rad), FOS_E_ARG, "NULL argument");
    rc = launch_rad_sum(c, rad, n, s);
    if (rc) return rc;
    k_mean_from_sum<<<1, 1, 0, s>>>(&c->ds->rad_sum, n, mean_radius);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_apply_jitter(FosCtx* c, float* v_jit, const float* rad, const float* mean_radius,
                                int n, float dt, double jitter_rms, double jitter_tau,
                                double max_drift_fraction, double gap_fraction, uint64_t seed,
                                uint32_t frame, fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (v_jit && rad && mean_radius), FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    OuParams o = ou_params(jitter_rms, jitter_tau, max_drift_fraction, gap_fraction, dt, c->L,
                           c->invL, seed);
    k_ou_velocity<<<fos_blocks(n, 256), 256, 0, s>>>(v_jit, rad, mean_radius, n, o, frame);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_integrate_jitter(FosCtx* c, float* pos, const float* v_jit, int n, float dt,
                                    fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (pos && v_jit), FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    OuParams o = ou_params(0.0, 1.0, 0.0, 0.0, dt, c->L, c->invL, 0);
    k_ou_move<<<fos_blocks(n, 256), 256, 0, s>>>(pos, v_jit, n, o);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_set_fsc_targets(FosCtx* c, const float* rad, float* rad_target,
                                   const int32_t* fsc, const float* fsc_ema, int n, int f_low,
                                   int f_high, float growth_pct, float r_min, float r_max,
                                   fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (rad && rad_target && fsc && fsc_ema), FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    return fos_launch_set_targets(c, rad, rad_target, fsc, fsc_ema, n, f_low, f_high, growth_pct,
                                  r_min, r_max, nullptr, 0, 0.0, 0, s);
}

extern "C" int fos_nudge_radii(FosCtx* c, float* rad, const float* rad_target,
                               const float* local_max_depth, int n, float alpha,
                               float max_step_pct, float r_min, float r_max, float back_global,
                               int mode, fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (rad && rad_target && local_max_depth), FOS_E_ARG, "NULL argument");
    return fos_launch_nudge(c, rad, rad_target, local_max_depth, n, alpha, max_step_pct, r_min,
                            r_max, back_global, nullptr, mode, nullptr, s);
}

extern "C" int fos_controller_stats(FosCtx* c, const float* rad, const float* rad_target,
                                    const float* fsc_ema, int n, int f_low, int f_high, int* grow,
                                    int* shrink, int* idle, float* mean_dr, float* max_dr,
                                    fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (rad && rad_target && fsc_ema), FOS_E_ARG, "NULL argument");
    int* counts = c->stats_i + 8;
    double* sum = (double*)(c->stats_f + 16);
    unsigned int* mx = (unsigned int*)(c->stats_i + 12);
    FOS_CUDA(cudaMemsetAsync(c->stats_i + 8, 0, 8 * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->stats_f + 16, 0, 8, s));
    if (n > 0) {
        k_controller_stats<<<fos_blocks(n, 256), 256, 0, s>>>(rad, rad_target, fsc_ema, n, f_low,
                                                              f_high, counts, sum, mx);
        FOS_LAUNCHED(c);
    }
    char* h = (char*)c->pinned;
    FOS_CUDA(cudaMemcpyAsync(h, c->stats_i + 8, 8 * 4, cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaMemcpyAsync(h + 64, c->stats_f + 16, 8, cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaStreamSynchronize(s));
    int* hi = (int*)h;
    if (grow) *grow = hi[0];
    if (shrink) *shrink = hi[1];
    if (idle) *idle = hi[2];
    double sm;
    memcpy(&sm, h + 64, 8);
    if (mean_dr) *mean_dr = (float)(sm / (double)(n > 1 ? n : 1));
    if (max_dr) {
        unsigned int b = (unsigned int)hi[4];
        float f;
        memcpy(&f, &b, 4);
        *max_dr = f;
    }
    return FOS_OK;
}

extern "C" int fos_pressure_stats(FosCtx* c, int n, const float* rad, float* rmin, float* rmax,
                                  fos_stream_t s) {
    int rc = check_dyn(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || rad, FOS_E_ARG, "NULL argument");
    unsigned int* mm = (unsigned int*)(c->stats_i + 20);
    unsigned int init[2] = {0xFFFFFFFFu, 0u};
    unsigned int* hp = (unsigned int*)c->pinned;
    hp[0] = init[0];
    hp[1] = init[1];
    FOS_CUDA(cudaMemcpyAsync(mm, hp, 8, cudaMemcpyHostToDevice, s));
    if (n > 0) {
        k_minmax<<<fos_blocks(n, 256), 256, 0, s>>>(rad, n, mm, mm + 1);
        FOS_LAUNCHED(c);
    }
    FOS_CUDA(cudaMemcpyAsync(hp + 4, mm, 8, cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaStreamSynchronize(s));
    auto unkey = [](unsigned int k) {
        unsigned int u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
        float f;
        memcpy(&f, &u, 4);
        return f;
    };
    // compute_pressure_stats starts from 1e9 / -1e9
    if (rmin) *rmin = n > 0 ? unkey(hp[4]) : 1e9f;
    if (rmax) *rmax = n > 0 ? unkey(hp[5]) : -1e9f;
    return FOS_OK;
}
