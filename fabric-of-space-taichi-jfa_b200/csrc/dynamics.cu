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

// ------------------------------------------------------------------
// Warp-cooperative enumeration of a particle's 27-cell neighbourhood.
// Lane l < 27 owns cell l of the stencil in the reference's (dx, dy, dz)
// order (dz fastest); an inclusive warp scan of the cell counts numbers the
// candidates 0..total-1 in exactly the order of the reference's nested loops
// (cells in stencil order, particles ascending inside a cell).  Candidate t
// is located by a binary search over the scanned counts.
struct Stencil {
    int st, excl, incl, total;
};

__device__ __forceinline__ Stencil stencil_ranges(float px, float py, float pz, float L, float invL,
                                                  float halfL, int G,
                                                  const int32_t* __restrict__ cs,
                                                  const int32_t* __restrict__ cc, int lane) {
    int hx = home_coord(px, L, invL, halfL, G);
    int hy = home_coord(py, L, invL, halfL, G);
    int hz = home_coord(pz, L, invL, halfL, G);
    int st = 0, ct = 0;
    if (lane < 27) {
        int nx = wrap_mod(hx + lane / 9 - 1, G);
        int ny = wrap_mod(hy + (lane / 3) % 3 - 1, G);
        int nz = wrap_mod(hz + lane % 3 - 1, G);
        int cid = (nx * G + ny) * G + nz;
        st = cs[cid];
        ct = cc[cid];
    }
    int incl = ct;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    Stencil r;
    r.st = st;
    r.incl = incl;
    r.excl = incl - ct;
    r.total = __shfl_sync(0xffffffffu, incl, 31);
    return r;
}

// Sorted-array position of candidate t (t < total).
__device__ __forceinline__ int stencil_locate(const Stencil& r, int t) {
    int c = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
        int v = __shfl_sync(0xffffffffu, r.incl, c + step - 1);
        if (v <= t) c += step;
    }
    int src = c & 31;
    int st = __shfl_sync(0xffffffffu, r.st, src);
    int ex = __shfl_sync(0xffffffffu, r.excl, src);
    return st + (t - ex);
}

// project_overlaps (dynamics.py:77-171) as one Jacobi sweep: every particle
// reads the pre-sweep positions (the cell-ordered copy sp, which holds pos and
// rad) and writes pout (the reference updates in place with atomics, so its
// result depends on scheduling; the Jacobi form is the deterministic
// restatement).  One warp per particle: lanes evaluate 32 candidates at a
// time, and the corrections of overlapping pairs are added in candidate
// order, so the FP32 sum is the reference loop's sum bit for bit.
__global__ void __launch_bounds__(256) k_pbd(const float4* __restrict__ sp,
                                             const int32_t* __restrict__ ci,
                                             float* __restrict__ pout, int n, int G, float L,
                                             float invL, float halfL,
                                             const int32_t* __restrict__ cs,
                                             const int32_t* __restrict__ cc, float gap1, float mdf,
                                             float dmul) {
    int kk = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    int lane = threadIdx.x & 31;
    if (kk >= n) return;  // warp-uniform
    float4 me = sp[kk];
    float px = me.x, py = me.y, pz = me.z, ri = me.w;
    Stencil r = stencil_ranges(px, py, pz, L, invL, halfL, G, cs, cc, lane);
    float md = fmul(mdf, ri);
    float cx = 0.f, cy = 0.f, cz = 0.f;
    for (int base = 0; base < r.total; base += 32) {
        int t = base + lane;
        int k = stencil_locate(r, t < r.total ? t : r.total - 1);
        bool hit = false;
        float vx = 0.f, vy = 0.f, vz = 0.f;
        if (t < r.total && k != kk) {
            float4 q = sp[k];
            float ddx = grid_wrap(fsub(q.x, px), L, invL);
            float ddy = grid_wrap(fsub(q.y, py), L, invL);
            float ddz = grid_wrap(fsub(q.z, pz), L, invL);
            float d2 = fadd(fadd(fadd(fmul(ddx, ddx), fmul(ddy, ddy)), fmul(ddz, ddz)), 1e-12f);
            float dist = __fsqrt_rn(d2);
            float tsep = fmul(fadd(ri, q.w), gap1);
            if (dist < tsep) {
                hit = true;
                float ov = fsub(tsep, dist);
                float ux = fdiv(ddx, dist), uy = fdiv(ddy, dist), uz = fdiv(ddz, dist);
                float mag = fminf(fmul(ov, 0.5f), md);
                vx = fmaxf(-md, fminf(md, fmul(-ux, mag)));
                vy = fmaxf(-md, fminf(md, fmul(-uy, mag)));
                vz = fmaxf(-md, fminf(md, fmul(-uz, mag)));
            }
        }
        unsigned int m = __ballot_sync(0xffffffffu, hit);
        while (m) {
            int b = __ffs(m) - 1;
            m &= m - 1;
            cx = fadd(cx, __shfl_sync(0xffffffffu, vx, b));
            cy = fadd(cy, __shfl_sync(0xffffffffu, vy, b));
            cz = fadd(cz, __shfl_sync(0xffffffffu, vz, b));
        }
    }
    if (lane == 0) {
        float mt = fmul(fmul(mdf, ri), dmul);
        float cm = __fsqrt_rn(fadd(fadd(fmul(cx, cx), fmul(cy, cy)), fmul(cz, cz)));
        if (cm > mt) {
            float sc = fdiv(mt, cm);
            cx = fmul(cx, sc);
            cy = fmul(cy, sc);
            cz = fmul(cz, sc);
        }
        int i = ci[kk];
        pout[3 * i + 0] = grid_wrap(fadd(px, cx), L, invL);
        pout[3 * i + 1] = grid_wrap(fadd(py, cy), L, invL);
        pout[3 * i + 2] = grid_wrap(fadd(pz, cz), L, invL);
    }
}

// compute_local_max_overlaps + reduce_max_depth (dynamics.py:304-372), one
// warp per particle over the same candidate enumeration (pairs i < j only).
__global__ void __launch_bounds__(256) k_max_overlap(const float4* __restrict__ sp,
                                                     const int32_t* __restrict__ ci, int n, int G,
                                                     float L, float invL, float halfL,
                                                     const int32_t* __restrict__ cs,
                                                     const int32_t* __restrict__ cc, float eps,
                                                     float* __restrict__ lmd,
                                                     unsigned int* gmax_bits) {
    int kk = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    int lane = threadIdx.x & 31;
    if (kk >= n) return;  // warp-uniform
    float4 me = sp[kk];
    int i = ci[kk];
    Stencil r = stencil_ranges(me.x, me.y, me.z, L, invL, halfL, G, cs, cc, lane);
    float lm = 0.f;
    for (int base = 0; base < r.total; base += 32) {
        int t = base + lane;
        int k = stencil_locate(r, t < r.total ? t : r.total - 1);
        if (t < r.total) {
            int j = ci[k];
            if (i < j) {
                float4 q = sp[k];
                float ddx = grid_wrap(fsub(q.x, me.x), L, invL);
                float ddy = grid_wrap(fsub(q.y, me.y), L, invL);
                float ddz = grid_wrap(fsub(q.z, me.z), L, invL);
                float dist = __fsqrt_rn(
                    fadd(fadd(fadd(fmul(ddx, ddx), fmul(ddy, ddy)), fmul(ddz, ddz)), eps));
                float td = fadd(me.w, q.w);
                if (dist < td) lm = fmaxf(lm, fsub(td, dist));
            }
        }
    }
    // max is exact in any order; non-negative floats order as their bits
    unsigned int b = __reduce_max_sync(0xffffffffu, __float_as_uint(lm));
    if (lane == 0) {
        lmd[i] = __uint_as_float(b);
        if (b) atomicMax(gmax_bits, b);
    }
}

// hash_func (dynamics.py:1436-1451) in wrapping int32 arithmetic.
__device__ __forceinline__ int hash_func(int i, int frame) {
    unsigned int t = (unsigned int)i + 12345u * (unsigned int)frame;
    return (int)((1103515245u * t + 12345u) & 0x7fffffffu);
}

// equilibrate_pressure (dynamics.py:1454-1557), one Jacobi sweep: reads
// rad_in, writes rad_out and delta_r.  GS lanes per particle: lane t handles
// the t-th budgeted neighbour of the hashed rotation, and the radius deltas
// are summed in neighbour order (the reference's serial accumulation order).
// Stats of this sweep go to slot `slot` of pmax/pchanged; the other slot is
// cleared for the next sweep.
template <int GS>
__global__ void __launch_bounds__(256) k_pressure(int n, int frame_arg, const int* frame_ptr,
                                                  const float* __restrict__ rin,
                                                  float* __restrict__ rout,
                                                  float* __restrict__ delta_r,
                                                  const int32_t* __restrict__ face_ids,
                                                  const int32_t* __restrict__ fsc, float k,
                                                  float P, float cap, int max_nei, float rmin,
                                                  float rmax, unsigned int* pmax, int* pchanged,
                                                  int slot) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        pmax[slot ^ 1] = 0u;
        pchanged[slot ^ 1] = 0;
    }
    int lane = threadIdx.x & 31;
    int gl = lane & (GS - 1);
    unsigned int gmask = GS == 32 ? 0xffffffffu : (0xffffu << (lane & 16));
    int i = (int)(tid / GS);
    bool live = i < n;
    int frame = frame_ptr ? *frame_ptr : frame_arg;
    float ri = live ? rin[i] : 0.f;
    int fc = live ? fsc[i] : 0;
    float d = 0.f;
    if (fc > 0) {
        int an = fc < max_nei ? fc : max_nei;
        int st = hash_func(i, frame) % fc;
        float Vi = powf(ri, P);
        float invP = fdiv(1.0f, P);
        for (int base = 0; base < an; base += GS) {
            int kk = base + gl;
            bool hit = false;
            float term = 0.f;
            if (kk < an) {
                int ni = (st + kk) % fc;
                int j = face_ids[(size_t)i * FOS_S + ni];
                if (!(j < 0 || j >= n || j == i)) {
                    float Vj = powf(rin[j], P);
                    float dvr = fmul(k, fsub(Vi, Vj));
                    float vmin = fminf(Vi, Vj);
                    float dv = fmaxf(fmul(-cap, vmin), fminf(fmul(cap, vmin), dvr));
                    term = fsub(powf(fsub(Vi, dv), invP), ri);
                    hit = true;
                }
            }
            unsigned int m = __ballot_sync(gmask, hit) & gmask;
            m >>= (GS == 32 ? 0 : (lane & 16));
            while (m) {
                int b = __ffs(m) - 1;
                m &= m - 1;
                d = fadd(d, __shfl_sync(gmask, term, b, GS));
            }
        }
    }
    if (live && gl == 0) {
        delta_r[i] = d;
        rout[i] = fmaxf(rmin, fminf(rmax, fadd(ri, d)));
    }
    float ad = fabsf(d);
    int ch = (live && gl == 0) && ad > 1e-12f;
    unsigned int wm = __ballot_sync(0xffffffffu, ch);
    unsigned int bm = __reduce_max_sync(0xffffffffu, ch ? __float_as_uint(ad) : 0u);
    if (lane == 0 && wm) {
        atomicAdd(&pchanged[slot], __popc(wm));
        atomicMax(&pmax[slot], bm);
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

int fos_grid_gather_sorted(FosCtx* c, const int32_t* idx, const float* pos, const float* rad,
                           int n, cudaStream_t s);

// PBD sweep over the cell-ordered copy ctx->sorted (must match cs/cc/ci).
int fos_launch_pbd(FosCtx* c, float* pout, const int32_t* cs, const int32_t* cc,
                   const int32_t* ci, int n, cudaStream_t s) {
    if (n == 0) return FOS_OK;
    k_pbd<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(c->sorted, ci, pout, n, c->G, c->L, c->invL,
                                                    c->halfL, cs, cc, c->gap1, c->mdf, c->dmul);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// Max overlap over the cell-ordered copy ctx->sorted (must match cs/cc/ci).
int fos_launch_max_overlap(FosCtx* c, const int32_t* cs, const int32_t* cc, const int32_t* ci,
                           float* lmd, int n, unsigned int* gmax_bits, cudaStream_t s) {
    FOS_CUDA(cudaMemsetAsync(gmax_bits, 0, 4, s));
    if (n == 0) return FOS_OK;
    k_max_overlap<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(c->sorted, ci, n, c->G, c->L, c->invL,
                                                            c->halfL, cs, cc, c->eps, lmd,
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
    unsigned int* pmax = &c->ds->maxabs_dr_bits;
    int* pch = &c->ds->changed;
    // two stat slots live in stats_i / stats_f scratch: [0..1] max bits, [2..3] counts
    unsigned int* sm = (unsigned int*)c->stats_i;
    int* sc = c->stats_i + 2;
    FOS_CUDA(cudaMemsetAsync(c->stats_i, 0, 4 * sizeof(int), s));
    for (int w = 0; w < sweeps; ++w) {
        const float* rin = (w & 1) ? c->rad_tmp : rad;
        float* rout = (w & 1) ? rad : c->rad_tmp;
        if (max_nei <= 16)
            k_pressure<16><<<fos_blocks(16LL * n, 256), 256, 0, s>>>(
                n, frame, frame_ptr, rin, rout, delta_r, face_ids, fsc, k, P, cap, max_nei, rmin,
                rmax, sm, sc, w & 1);
        else
            k_pressure<32><<<fos_blocks(32LL * n, 256), 256, 0, s>>>(
                n, frame, frame_ptr, rin, rout, delta_r, face_ids, fsc, k, P, cap, max_nei, rmin,
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
