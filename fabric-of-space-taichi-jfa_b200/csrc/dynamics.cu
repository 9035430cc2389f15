// dynamics.cu -- PBD overlap projection, max overlap, Jacobi pressure
// diffusion, Brownian jitter and the FSC radius controller.
//
// Reference: dynamics.py.  All neighbour work is a gather over the sorted
// hash-grid cells (27-cell stencil, cells in (dx, dy, dz) order, dz fastest,
// particles ascending inside a cell), in the reference's accumulation order.
#include <string.h>

#include "fos_internal.cuh"

// Home cell as project_overlaps / compute_local_max_overlaps compute it
// (dynamics.py:101-103): int(((wrapP(p) + HALF_L) * INV_L) * GRID_RES), no
// epsilon and no wrap before the +-1 offsets.
__device__ __forceinline__ int home_coord(float p, float L, float invL, float halfL, int G) {
    float w = grid_wrap(p, L, invL);
    float q = fmul(fadd(w, halfL), invL);
    return (int)fmul(q, (float)G);
}

// project_overlaps (dynamics.py:77-171) as one Jacobi sweep: read pos_in,
// write pos_out (the reference updates in place with atomics, so its result
// depends on scheduling; the Jacobi form is the deterministic restatement).
__global__ void __launch_bounds__(128) k_pbd(const float* __restrict__ pin, float* __restrict__ pout,
                                             const float* __restrict__ rad, int n, int G, float L,
                                             float invL, float halfL,
                                             const int32_t* __restrict__ cs,
                                             const int32_t* __restrict__ cc,
                                             const int32_t* __restrict__ ci, float gap1, float mdf,
                                             float dmul) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float px = pin[3 * i + 0], py = pin[3 * i + 1], pz = pin[3 * i + 2];
    float ri = rad[i];
    int hx = home_coord(px, L, invL, halfL, G);
    int hy = home_coord(py, L, invL, halfL, G);
    int hz = home_coord(pz, L, invL, halfL, G);
    float cx = 0.f, cy = 0.f, cz = 0.f;
    float md = fmul(mdf, ri);
    for (int dx = -1; dx <= 1; ++dx) {
        int nx = wrap_mod(hx + dx, G);
        for (int dy = -1; dy <= 1; ++dy) {
            int ny = wrap_mod(hy + dy, G);
            for (int dz = -1; dz <= 1; ++dz) {
                int nz = wrap_mod(hz + dz, G);
                int cid = (nx * G + ny) * G + nz;
                int st = cs[cid], ct = cc[cid];
                for (int k = st; k < st + ct; ++k) {
                    int j = ci[k];
                    if (j == i) continue;
                    float ddx = grid_wrap(fsub(pin[3 * j + 0], px), L, invL);
                    float ddy = grid_wrap(fsub(pin[3 * j + 1], py), L, invL);
                    float ddz = grid_wrap(fsub(pin[3 * j + 2], pz), L, invL);
                    float d2 = fadd(fadd(fadd(fmul(ddx, ddx), fmul(ddy, ddy)), fmul(ddz, ddz)), 1e-12f);
                    float dist = __fsqrt_rn(d2);
                    float tsep = fmul(fadd(ri, rad[j]), gap1);
                    if (dist < tsep) {
                        float ov = fsub(tsep, dist);
                        float ux = fdiv(ddx, dist), uy = fdiv(ddy, dist), uz = fdiv(ddz, dist);
                        float mag = fminf(fmul(ov, 0.5f), md);
                        float vx = fmul(-ux, mag), vy = fmul(-uy, mag), vz = fmul(-uz, mag);
                        vx = fmaxf(-md, fminf(md, vx));
                        vy = fmaxf(-md, fminf(md, vy));
                        vz = fmaxf(-md, fminf(md, vz));
                        cx = fadd(cx, vx);
                        cy = fadd(cy, vy);
                        cz = fadd(cz, vz);
                    }
                }
            }
        }
    }
    float mt = fmul(fmul(mdf, ri), dmul);
    float cm = __fsqrt_rn(fadd(fadd(fmul(cx, cx), fmul(cy, cy)), fmul(cz, cz)));
    if (cm > mt) {
        float sc = fdiv(mt, cm);
        cx = fmul(cx, sc);
        cy = fmul(cy, sc);
        cz = fmul(cz, sc);
    }
    pout[3 * i + 0] = grid_wrap(fadd(px, cx), L, invL);
    pout[3 * i + 1] = grid_wrap(fadd(py, cy), L, invL);
    pout[3 * i + 2] = grid_wrap(fadd(pz, cz), L, invL);
}

// compute_local_max_overlaps + reduce_max_depth (dynamics.py:304-372).
__global__ void __launch_bounds__(128) k_max_overlap(const float* __restrict__ pos,
                                                     const float* __restrict__ rad, int n, int G,
                                                     float L, float invL, float halfL,
                                                     const int32_t* __restrict__ cs,
                                                     const int32_t* __restrict__ cc,
                                                     const int32_t* __restrict__ ci, float eps,
                                                     float* __restrict__ lmd,
                                                     unsigned int* gmax_bits) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float lm = 0.f;
    if (i < n) {
        float px = pos[3 * i + 0], py = pos[3 * i + 1], pz = pos[3 * i + 2];
        float ri = rad[i];
        int hx = home_coord(px, L, invL, halfL, G);
        int hy = home_coord(py, L, invL, halfL, G);
        int hz = home_coord(pz, L, invL, halfL, G);
        for (int dx = -1; dx <= 1; ++dx) {
            int nx = wrap_mod(hx + dx, G);
            for (int dy = -1; dy <= 1; ++dy) {
                int ny = wrap_mod(hy + dy, G);
                for (int dz = -1; dz <= 1; ++dz) {
                    int nz = wrap_mod(hz + dz, G);
                    int cid = (nx * G + ny) * G + nz;
                    int st = cs[cid], ct = cc[cid];
                    for (int k = st; k < st + ct; ++k) {
                        int j = ci[k];
                        if (!(i < j)) continue;
                        float ddx = grid_wrap(fsub(pos[3 * j + 0], px), L, invL);
                        float ddy = grid_wrap(fsub(pos[3 * j + 1], py), L, invL);
                        float ddz = grid_wrap(fsub(pos[3 * j + 2], pz), L, invL);
                        float dist = __fsqrt_rn(
                            fadd(fadd(fadd(fmul(ddx, ddx), fmul(ddy, ddy)), fmul(ddz, ddz)), eps));
                        float td = fadd(ri, rad[j]);
                        if (dist < td) lm = fmaxf(lm, fsub(td, dist));
                    }
                }
            }
        }
        lmd[i] = lm;
    }
    // warp max, then one atomic per warp (non-negative floats order as uints)
    unsigned int b = __float_as_uint(lm);
    b = __reduce_max_sync(0xffffffffu, b);
    if ((threadIdx.x & 31) == 0 && b) atomicMax(gmax_bits, b);
}

// hash_func (dynamics.py:1436-1451) in wrapping int32 arithmetic.
__device__ __forceinline__ int hash_func(int i, int frame) {
    unsigned int t = (unsigned int)i + 12345u * (unsigned int)frame;
    return (int)((1103515245u * t + 12345u) & 0x7fffffffu);
}

// equilibrate_pressure (dynamics.py:1454-1557), one Jacobi sweep: reads
// rad_in, writes rad_out and delta_r.  Stats of this sweep go to slot
// `slot` of pmax/pchanged; the other slot is cleared for the next sweep.
__global__ void __launch_bounds__(256) k_pressure(int n, int frame_arg, const int* frame_ptr,
                                                  const float* __restrict__ rin,
                                                  float* __restrict__ rout,
                                                  float* __restrict__ delta_r,
                                                  const int32_t* __restrict__ face_ids,
                                                  const int32_t* __restrict__ fsc, float k,
                                                  float P, float cap, int max_nei, float rmin,
                                                  float rmax, unsigned int* pmax, int* pchanged,
                                                  int slot) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        pmax[slot ^ 1] = 0u;
        pchanged[slot ^ 1] = 0;
    }
    float d = 0.f;
    if (i < n) {
        int frame = frame_ptr ? *frame_ptr : frame_arg;
        float ri = rin[i];
        float Vi = powf(ri, P);
        int fc = fsc[i];
        if (fc > 0) {
            int an = fc < max_nei ? fc : max_nei;
            int st = hash_func(i, frame) % fc;
            float invP = fdiv(1.0f, P);
            for (int kk = 0; kk < an; ++kk) {
                int ni = (st + kk) % fc;
                int j = face_ids[(size_t)i * FOS_S + ni];
                if (j < 0 || j >= n || j == i) continue;
                float Vj = powf(rin[j], P);
                float dvr = fmul(k, fsub(Vi, Vj));
                float vmin = fminf(Vi, Vj);
                float dv = fmaxf(fmul(-cap, vmin), fminf(fmul(cap, vmin), dvr));
                float vn = fsub(Vi, dv);
                d = fadd(d, fsub(powf(vn, invP), ri));
            }
        }
        delta_r[i] = d;
        rout[i] = fmaxf(rmin, fminf(rmax, fadd(ri, d)));
    }
    float ad = fabsf(d);
    int ch = (i < n) && ad > 1e-12f;
    unsigned int m = __ballot_sync(0xffffffffu, ch);
    unsigned int b = __reduce_max_sync(0xffffffffu, ch ? __float_as_uint(ad) : 0u);
    if ((threadIdx.x & 31) == 0 && m) {
        atomicAdd(&pchanged[slot], __popc(m));
        atomicMax(&pmax[slot], b);
    }
}

// apply_brownian_motion (dynamics.py:1596-1634).  ti.random() is replaced by
// Philox-4x32-10 with counter (i, frame, 'BROW', 0) and key = seed; each axis
// draws u = (x >> 8) * 2^-24.  With tick != NULL, thread 0 also decrements the
// device settle counter (run.py:750), which the frame's nudge already read.
__global__ void k_brownian(float* pos, int n, float strength, float domain, float halfL,
                           uint32_t k0, uint32_t k1, int frame_arg, const int* frame_ptr,
                           FosDevState* tick) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (tick && i == 0 && tick->settle > 0) tick->settle -= 1;
    if (i >= n) return;
    unsigned int frame = (unsigned int)(frame_ptr ? *frame_ptr : frame_arg);
    uint4 r = philox4x32_10(make_uint4((unsigned int)i, frame, 0x42524f57u, 0u), k0, k1);
    unsigned int rr[3] = {r.x, r.y, r.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float u = fmul((float)(rr[d] >> 8), 0x1p-24f);
        float dd = fmul(fmul(fsub(u, 0.5f), 2.0f), strength);
        float p = fadd(pos[3 * i + d], dd);
        if (p < -halfL) p = fadd(p, domain);
        else if (p >= halfL) p = fsub(p, domain);
        pos[3 * i + d] = p;
    }
}

// smoothstep (dynamics.py:1226-1240)
__device__ __forceinline__ float smoothstep(float e0, float e1, float x) {
    float t = fminf(1.0f, fmaxf(0.0f, fdiv(fsub(x, e0), fsub(e1, e0))));
    return fmul(fmul(t, t), fsub(3.0f, fmul(2.0f, t)));
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
    const float hg = 1.0f, idle = 0.003f;
    float r0 = rad[i];
    float e = ema[i];
    float f = e > 0.0f ? e : (float)fsc[i];
    float lo = (float)f_low, hi = (float)f_high;
    float out;
    if (f < fsub(lo, hg)) {
        out = fminf(fmul(r0, fadd(1.0f, fmul(growth, 1.0f))), rmax);
    } else if (f < lo) {
        float gain = fsub(1.0f, smoothstep(fsub(fsub(lo, hg), db), lo, f));
        out = fminf(fmul(r0, fadd(1.0f, fmul(growth, gain))), rmax);
    } else if (f > fadd(hi, hg)) {
        out = fmaxf(fmul(r0, fsub(1.0f, fmul(growth, 1.0f))), rmin);
    } else if (f > hi) {
        float gain = smoothstep(hi, fadd(fadd(hi, hg), db), f);
        out = fmaxf(fmul(r0, fsub(1.0f, fmul(growth, gain))), rmin);
    } else {
        float bc = fmul(0.5f, fadd(lo, hi));
        if (f < bc) out = fminf(fmul(r0, fadd(1.0f, fmul(growth, idle))), rmax);
        else out = fmaxf(fmul(r0, fsub(1.0f, fmul(growth, idle))), rmin);
    }
    rt[i] = out;
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
    if (back_bits && mode == 1) {
        double om = (double)__uint_as_float(*back_bits);
        double raw = contact_tol_d > 0 ? (contact_tol_d - om) / contact_tol_d : 1.0;
        back = contact_tol_d > 0 ? (float)fmax(0.25, fmin(1.0, raw)) : 1.0f;
    }
    float r0 = rad[i];
    float r_t = fminf(rmax, fmaxf(rmin, rt[i]));
    float d = fmul(alpha, fsub(r_t, r0));
    float b = 1.0f;
    if (mode == 1) b = back;
    else if (mode == 2) {
        b = fdiv(fsub(contact_tol, lmd[i]), contact_tol);
        b = fminf(1.0f, fmaxf(0.25f, b));
    }
    d = fmul(d, b);
    float cap = fmul(max_step, r0);
    if (d > cap) d = cap;
    if (d < -cap) d = -cap;
    rad[i] = fminf(rmax, fmaxf(rmin, fadd(r0, d)));
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

int fos_launch_pbd(FosCtx* c, const float* pin, float* pout, const float* rad,
                   const int32_t* cs, const int32_t* cc, const int32_t* ci, int n, cudaStream_t s) {
    if (n == 0) return FOS_OK;
    k_pbd<<<fos_blocks(n, 128), 128, 0, s>>>(pin, pout, rad, n, c->G, c->L, c->invL, c->halfL, cs,
                                             cc, ci, c->gap1, c->mdf, c->dmul);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

int fos_launch_max_overlap(FosCtx* c, const float* pos, const float* rad, const int32_t* cs,
                           const int32_t* cc, const int32_t* ci, float* lmd, int n,
                           unsigned int* gmax_bits, cudaStream_t s) {
    FOS_CUDA(cudaMemsetAsync(gmax_bits, 0, 4, s));
    if (n == 0) return FOS_OK;
    k_max_overlap<<<fos_blocks(n, 128), 128, 0, s>>>(pos, rad, n, c->G, c->L, c->invL, c->halfL, cs,
                                                     cc, ci, c->eps, lmd, gmax_bits);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// `sweeps` pressure sweeps ping-ponging rad <-> rad_tmp; the result ends in rad.
int fos_launch_pressure(FosCtx* c, int n, int frame, const int* frame_ptr, float* rad,
                        float* delta_r, const int32_t* face_ids, const int32_t* fsc, float k,
                        float P, float cap, int max_nei, float rmin, float rmax, int sweeps,
                        cudaStream_t s) {
    if (n == 0 || sweeps <= 0) return FOS_OK;
    unsigned int* pmax = &c->ds->maxabs_dr_bits;
    int* pch = &c->ds->changed;
    // two stat slots live in stats_i / stats_f scratch: [0..1] max bits, [2..3] counts
    unsigned int* sm = (unsigned int*)c->stats_i;
    int* sc = c->stats_i + 2;
    FOS_CUDA(cudaMemsetAsync(c->stats_i, 0, 4 * sizeof(int), s));
    for (int w = 0; w < sweeps; ++w) {
        const float* rin = (w & 1) ? c->rad_tmp : rad;
        float* rout = (w & 1) ? rad : c->rad_tmp;
        k_pressure<<<fos_blocks(n, 256), 256, 0, s>>>(n, frame, frame_ptr, rin, rout, delta_r,
                                                      face_ids, fsc, k, P, cap, max_nei, rmin,
                                                      rmax, sm, sc, w & 1);
        FOS_LAUNCHED(c);
    }
    if (sweeps & 1)
        FOS_CUDA(cudaMemcpyAsync(rad, c->rad_tmp, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    int last = (sweeps - 1) & 1;
    FOS_CUDA(cudaMemcpyAsync(pmax, sm + last, 4, cudaMemcpyDeviceToDevice, s));
    FOS_CUDA(cudaMemcpyAsync(pch, sc + last, 4, cudaMemcpyDeviceToDevice, s));
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
    rc = fos_launch_pbd(c, pos, c->pos_tmp, rad, cs, cc, ci, n, s);
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
    rc = fos_launch_max_overlap(c, pos, rad, cs, cc, ci, lmd, n, bits, s);
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
