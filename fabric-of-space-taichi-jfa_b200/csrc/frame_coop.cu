// frame_coop.cu -- the dynamics part of one frame as ONE persistent
// cooperative kernel.
//
// A plain frame of the reference (run.py:699-874) is a chain of ~70 dependent
// stages: 10 hash-grid rebuilds, the max-overlap reduction, the settle nudge,
// M pressure sweeps, Brownian jitter and K PBD sweeps.  At 10k particles
// each stage is a few microseconds of work, so separate launches are bound by
// launch latency.  Here every stage is a phase of a single launch whose
// blocks are all co-resident (cooperative launch), separated by bounded grid
// barriers; each phase calls the same per-element device functions as the
// standalone kernels (phases.cuh), so the results are identical.
//
// Grid rebuilds inside the kernel (grid.py:145-309 / run.py:476-504): the
// histogram of a rebuild runs inside the phase that produced the positions
// and drops each particle into a fixed-capacity cell row; the frame's own
// stages read those rows as they are (coop_p1_dst, coop_layout below).  A row
// that overflows sends its rebuild to the CSR form (coop_csr, coop.cuh); the
// final rebuild, whose cell arrays the caller sees, is always the CSR form.
#include <string.h>

#include "coop.cuh"

struct CoopArgs {
    int n, G3, chunk, pbd_iters, sweeps, bp_mode, small_grid;
    GridGeom g;
    float* pos;
    float* pos_tmp;
    float* rad;
    float* rad_tmp;
    const float* rad_target;
    float* lmd;
    float* delta_r;
    int32_t* cc;
    int32_t* cs;
    int32_t* ci;
    int32_t* cellof;
    int32_t* rank;
    int32_t* ci_tmp;
    int32_t* cnt;               // 3 x G3 count buffers (rebuild r uses buffer r % 3)
    int32_t* rows_ci[2];        // fixed-capacity rows of rebuild r: set r & 1 (NULL: CSR only)
    float4* rows_sp[2];
    int32_t* slot_of;
    float* vol0;                // [n] r^P ping-pong of the pressure sweeps
    float* vol1;
    unsigned long long* ptag;   // non-NULL: barrier-free pressure sweeps on tagged words
    int32_t* pnbr;              // [16 n] the frame's pressure neighbours (sweeps with barriers)
    int32_t* part;
    int32_t* bsum;
    float4* sp;
    FosDevState* ds;
    float gap1, mdf, dmul, eps, contact_tol;
    double contact_tol_d;
    float alpha, max_step, rmin, rmax;
    PressureArgs pa;
    float strength, domain, halfL;
    uint32_t k0, k1;
    int ou;                     // OU jitter fused into the last PBD sweep (pbd_iters >= 1)
    float* vjit;
    OuParams ou_p;
    unsigned long long* trace;  // optional: %globaltimer after every phase (block 0); the
    int trace_cap;              // last two slots: ~(earliest block start), latest block end
    int end_frame;              // advance the frame counter at the end (k_frame_end)
};

// Tagged pressure words: (tag << 32) | float bits, written and read whole, so
// a reader that sees the tag it waits for also sees that sweep's value.
__device__ __forceinline__ void st_tagged(unsigned long long* p, unsigned int tag, float v) {
    const unsigned long long w = ((unsigned long long)tag << 32) | __float_as_uint(v);
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}

__device__ __forceinline__ unsigned long long ld_tagged(const unsigned long long* p) {
    unsigned long long w;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
    return w;
}

// Lanes per particle of the barrier-free pressure sweeps (a power of two
// dividing 16: each lane takes 16 / COOP_PLANES neighbours).
#ifndef COOP_PLANES
#define COOP_PLANES 8
#endif
// Rounds of 8-lane groups in flight in the pressure sweeps with grid barriers
// (n > threads / 8): their loads are all issued before the first sum.
#ifndef COOP_PRESS_ROUNDS
#define COOP_PRESS_ROUNDS 2
#endif
// Pause between two polls of a word that is not ready yet, in ns (fewer L2
// requests from waiting warps).
#ifndef COOP_POLL_NS
#define COOP_POLL_NS 0
#endif

// Every lane waits for the words base[j[h]] (where need[h]) to carry `tag`
// and gets their values in v[h]; the whole warp polls together, so the warp's
// groups never diverge.  Bounded like the grid barrier: after ~1 s, or once
// the error word is set, it records FOS_E_TIMEOUT, clears ok and returns
// (the next grid barrier then ends the kernel).
template <int H>
__device__ __forceinline__ void wait_tagged_n(const unsigned long long* base, const int* j,
                                              bool* need, unsigned int tag, FosDevState* ds,
                                              bool& ok, float* v) {
    const long long t0 = clock64();
    unsigned int polls = 0;
    for (;;) {
        bool any = false;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            if (need[h]) {
                const unsigned long long w = ld_tagged(&base[j[h]]);
                if ((unsigned int)(w >> 32) == tag) {
                    v[h] = __uint_as_float((unsigned int)w);
                    need[h] = false;
                }
            }
            any |= need[h];
        }
        if (!__any_sync(0xffffffffu, any) || !ok) return;
        if (COOP_POLL_NS > 0) __nanosleep(COOP_POLL_NS);
        if ((++polls & 31u) == 0u &&
            __any_sync(0xffffffffu, *((volatile int*)&ds->error) != 0 ||
                                        clock64() - t0 > FOS_BAR_CYCLE_LIMIT)) {
            atomicCAS(&ds->error, 0, (int)FOS_E_TIMEOUT);
            ok = false;
            return;
        }
    }
}

// Rebuild r of a frame (r = 0 before max overlap, 1..pbd_iters before each PBD
// sweep, pbd_iters + 1 the final CSR one) drops its particles into count
// buffer r % 3, row set r & 1 and overflow flag r % 3 of the barrier word; its
// P1 runs in the phase before its first reader, which gets the flags from the
// barrier between them.  The rows stay in arrival order: max overlap does
// not depend on the order, and the PBD sweeps put their hits in index order
// themselves (pbd_warp_rows), so no phase sorts the rows.
__device__ __forceinline__ P1Dst coop_p1_dst(const CoopArgs& a, int r) {
    return P1Dst{a.cnt + (size_t)(r % 3) * a.G3, a.rows_ci[r & 1], a.rows_sp[r & 1], a.slot_of,
                 &a.ds->bar_count, 1u << (FOS_BAR_FLAG_SHIFT + r % 3)};
}

// Rebuild index as a deferred P1 target.
struct RebuildIdx {
    int r;
};
__device__ __forceinline__ P1Dst p1_target(const CoopArgs& a, RebuildIdx t) {
    return coop_p1_dst(a, t.r);
}

// Layout of rebuild r for the phase that reads it (flags: from the barrier
// after its P1): the rows when none overflowed, else the CSR form, whose
// phases run first.  Also clears count buffer and overflow flag (r + 2) % 3
// for rebuild r + 2, whose P1 comes one phase later (their last reader, of
// rebuild r - 1, is done).
__device__ __forceinline__ bool coop_layout(const CoopArgs& a, const UniGeo& geo, int r,
                                            unsigned int flags, int& tk, unsigned int& ep,
                                            CoopLayout& lay, bool& rows) {
    const int T = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t* zc = a.cnt + (size_t)((r + 2) % 3) * a.G3;
    for (int c = tid; c < a.G3; c += T) zc[c] = 0;
    if (tid == 0) atomicAnd(&a.ds->bar_count, ~(1u << (FOS_BAR_FLAG_SHIFT + (r + 2) % 3)));
    const bool ovf = (flags >> (r % 3)) & 1u;
    const int32_t* cnt = a.cnt + (size_t)(r % 3) * a.G3;
    rows = a.rows_ci[0] != nullptr && !ovf;
    if (rows) {
        lay = CoopLayout{a.rows_ci[r & 1], a.rows_sp[r & 1], nullptr, cnt, COOP_CAP};
        return true;
    }
    lay = CoopLayout{a.ci, a.sp, a.cs, a.cc, 0};
    return coop_csr(a, geo, cnt, a.pos, a.rad, false, tk, ep);
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, COOP_BLOCKS_PER_SM) k_frame_coop(CoopArgs a) {
    const int T = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int W = T >> 5;
    // warp index for one-warp-per-particle loops: consecutive warps on
    // consecutive blocks, so a last partial round spreads over every SM
    const int wid = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
    // rounds of work with block-uniform trip counts (block reductions inside)
    const int warp_rounds = (a.n + W - 1) / W;
    int tk = 0;
    unsigned int ep = 0;
    if (a.trace && threadIdx.x == 0) atomicMax(&a.trace[a.trace_cap - 2], ~global_ns());
    trace_mark(a, tk);

    // (1) rebuild_grid (run.py:704): rebuild 0's P1, then its layout
    const UniGeo geo{a.g.G, a.g.L, a.g.invL, a.g.halfL};
    CoopLayout lay;
    bool rows = false;
    {
        const P1Dst t = coop_p1_dst(a, 0);
        unsigned int rmx = 0u;  // the largest radius (positive floats order as their bits)
        for (int i = spread_tid(); i < a.n; i += T) {
            const float r_i = __ldcg(&a.rad[i]);
            rmx = max(rmx, __float_as_uint(r_i));
            coop_p1_val(a, geo, i,
                        make_float3(__ldcg(&a.pos[3 * i + 0]), __ldcg(&a.pos[3 * i + 1]),
                                    __ldcg(&a.pos[3 * i + 2])),
                        r_i, a.pos, t);
        }
        block_max_atomic(__reduce_max_sync(0xffffffffu, rmx), &a.ds->rmax0_bits);
    }
    unsigned int gfl = 0u;  // overflow flags from the barrier after the last P1
    const unsigned int* const fw0[1] = {&a.ds->rmax0_bits};
    unsigned int fv0[1];
    if (!grid_barrier(a.ds, ep, &gfl, fw0, 1, fv0)) return;
    trace_mark(a, tk);
    const float cell_w = a.g.L / (float)a.g.G;
    // (2) compute_max_overlap (run.py:709): particle i's slot comes from
    // slot_of, prefetched one round ahead (the rows' slots come from P1; the
    // CSR form rewrites slot_of, and the first prefetch is then repeated).
    int kk0 = wid < a.n ? __ldcg(&a.slot_of[wid]) : 0;
    if (!coop_layout(a, geo, 0, gfl, tk, ep, lay, rows)) return;
    // max overlap visits only the cells that can hold a positive depth (rows only)
    const float rmax0 = rows && a.g.G >= 5 ? __uint_as_float(fv0[0]) : 0.f;
    if (!rows) kk0 = wid < a.n ? __ldcg(&a.slot_of[wid]) : 0;
    {
        unsigned int wmax = 0u;
        int kk_next = kk0;
        for (int r = 0; r < warp_rounds; ++r) {
            const int i = r * W + wid;
            const int kk = kk_next;
            kk_next = i + W < a.n ? __ldcg(&a.slot_of[i + W]) : 0;
            if (i < a.n) {
                unsigned int b = maxov_warp<LdL1>(kk, lane, lay.sp, lay.ci, a.g, lay.cs, lay.cc,
                                                  a.eps, a.lmd, lay.cap, 0, rmax0, cell_w);
                wmax = b > wmax ? b : wmax;
            }
        }
        block_max_atomic(wmax, &a.ds->omax_bits);
    }
    // settle, the deepest overlap, the frame number and the launch epoch,
    // fetched once per block
    const unsigned int* const fw[4] = {(const unsigned int*)&a.ds->settle, &a.ds->omax_bits,
                                       (const unsigned int*)&a.ds->frame, &a.ds->coop_epoch};
    unsigned int fv[4];
    if (!grid_barrier(a.ds, ep, nullptr, fw, 4, fv)) return;
    trace_mark(a, tk);
    const bool nudge = (int)fv[0] > 0;
    const float bg = back_global_from_bits(fv[1], a.contact_tol_d);
    PressureArgs pa = a.pa;
    pa.frame = (int)fv[2];
    if (a.ptag) {
        // (3) + (4) without grid barriers (n * COOP_PLANES <= T,
        // 1 <= sweeps <= FOS_PTAG_SWEEPS): each group of COOP_PLANES lanes
        // nudges its particle and runs every pressure sweep on it.  The power
        // r^P that starts sweep w is published as the word ptag[w * n + i]
        // tagged (epoch << 7) | (w + 1), and a sweep waits for its neighbours'
        // words of the same sweep, so it reads exactly the values a barrier
        // between the sweeps would give.  Every sweep has its own words: a
        // particle may run ahead of the particles that read it.
        constexpr int NL = COOP_PLANES, H = 16 / COOP_PLANES;
        const int i = (((threadIdx.x >> 5) * gridDim.x + blockIdx.x) * (32 / NL)) + (lane / NL);
        const int gl = lane & (NL - 1);
        const bool live = i < a.n;
        const unsigned int tbase = fv[3] << 7;
        float ri = 0.f;
        if (live) {
            ri = __ldcg(&a.rad[i]);
            if (nudge)
                ri = nudge_one(ri, __ldcg(&a.rad_target[i]), __ldcg(&a.lmd[i]), a.alpha,
                               a.max_step, a.rmin, a.rmax, bg, a.bp_mode, a.contact_tol);
        }
        float Vi = live ? pow_P(ri, pa.P) : 0.f;
        if (live && gl == 0) {
            if (nudge) a.rad[i] = ri;
            st_tagged(&a.ptag[i], tbase | 1u, Vi);
        }
        const PressureNbrN<NL> nb = pressure_nbr_n<NL, LdL2>(i, lane, pa);
        bool ok = true;
        float d = 0.f;
        for (int w = 0; w < a.sweeps; ++w) {
            const unsigned int tag = tbase | (unsigned int)(w + 1);
            d = 0.f;
            float vj[H];
            bool need[H];
#pragma unroll
            for (int h = 0; h < H; ++h) {
                vj[h] = 0.f;
                need[h] = nb.fc > 0 && nb.ok[h];
            }
            wait_tagged_n<H>(a.ptag + (size_t)w * a.n, nb.j, need, tag, a.ds, ok, vj);
            if (nb.fc > 0) d = pressure_sum_n<NL>(pa, nb, lane, ri, Vi, vj);
            ri = fmaxf(pa.rmin, fminf(pa.rmax, fadd(ri, d)));
            if (w + 1 < a.sweeps) {
                Vi = pow_P(ri, pa.P);
                if (live && gl == 0) st_tagged(&a.ptag[(size_t)(w + 1) * a.n + i], tag + 1u, Vi);
            }
        }
        if (live && gl == 0) {
            a.delta_r[i] = d;
            a.rad[i] = ri;
        }
        // the last sweep's stats
        const float ad = fabsf(d);
        const int ch = (live && gl == 0) && ad > 1e-12f;
        const int cnt = __syncthreads_count(ch);
        const unsigned int bm = __reduce_max_sync(0xffffffffu, ch ? __float_as_uint(ad) : 0u);
        block_max_atomic(bm, &a.ds->maxabs_dr_bits);
        if (threadIdx.x == 0 && cnt) atomicAdd(&a.ds->changed, cnt);
        if (!grid_barrier(a.ds, ep)) return;
        trace_mark(a, tk);
    } else {
    // 8-lane groups, two neighbours per lane: every particle in one round
    const int groups_per_round = T / 8;
    const int p_rounds = (a.n + groups_per_round - 1) / groups_per_round;
    // with one round (n <= T/8) each lane keeps its neighbours in registers
    // for all sweeps, and the particles are spread over every block, so every
    // SM issues the same share of the sweep
    const bool keep_nbr = p_rounds == 1;
    // with more rounds the nudge phase writes each particle's neighbours to a
    // table (pressure_nbr_fill) and a sweep takes two rounds at a time
    const bool table = a.pnbr != nullptr && !keep_nbr;
    // (3) nudge_radii_adaptive_ema while settle_frames_left > 0 (run.py:744-750);
    // each final radius's power r^P seeds the pressure sweeps
    {
        for (int i = spread_tid(); i < a.n; i += T) {
            float r = __ldcg(&a.rad[i]);
            if (nudge) {
                r = nudge_one(r, __ldcg(&a.rad_target[i]), __ldcg(&a.lmd[i]), a.alpha,
                              a.max_step, a.rmin, a.rmax, bg, a.bp_mode, a.contact_tol);
                a.rad[i] = r;
            }
            if (a.sweeps > 0) a.vol0[i] = pow_P(r, a.pa.P);
            if (table && a.sweeps > 0) pressure_nbr_fill<LdL2>(i, pa, a.pnbr);
        }
    }
    if (!grid_barrier(a.ds, ep)) return;
    trace_mark(a, tk);
    // (4) pressure sweeps (run.py:755-771); the last sweep reports its stats
    // four consecutive particles per warp (one sector of each per-particle
    // array), consecutive warps of particles on consecutive blocks
    const int i_one =
        (int)((((threadIdx.x >> 5) * gridDim.x + blockIdx.x) << 2) + ((threadIdx.x >> 3) & 3));
    const PressureNbr nb0 = pressure_nbr8x2<LdL2>(i_one, lane, pa);
    for (int w = 0; w < a.sweeps; ++w) {
        const float* rin = (w & 1) ? a.rad_tmp : a.rad;
        float* rout = (w & 1) ? a.rad : a.rad_tmp;
        const float* vin = (w & 1) ? a.vol1 : a.vol0;
        float* vout = (w & 1) ? a.vol0 : a.vol1;
        bool last = (w == a.sweeps - 1);
        if (table) {
            // COOP_PRESS_ROUNDS rounds at a time: every group's loads before
            // the first sum
            constexpr int NR = COOP_PRESS_ROUNDS;
            for (int r = 0; r < p_rounds; r += NR) {
                int ii[NR];
                PressureIn pin[NR];
#pragma unroll
                for (int h = 0; h < NR; ++h) {
                    ii[h] = (r + h) * groups_per_round + tid / 8;
                    pin[h] = pressure_in8x2n<PRESS_LD>(ii[h], lane, a.n, a.pnbr, rin, vin);
                }
                float* vo = last ? nullptr : vout;
                float dd[NR];
#pragma unroll
                for (int h = 0; h < NR; ++h)
                    dd[h] = pressure_out8x2n(ii[h], lane, a.n, pa, pin[h], pa.rmin, pa.rmax, rout,
                                             vo, a.delta_r);
                if (last) {
#pragma unroll
                    for (int h = 0; h < NR; ++h) {
                        const float ad = fabsf(dd[h]);
                        const int ch = (ii[h] < a.n && (lane & 7) == 0) && ad > 1e-12f;
                        const int cnt = __syncthreads_count(ch);
                        const unsigned int bm =
                            __reduce_max_sync(0xffffffffu, ch ? __float_as_uint(ad) : 0u);
                        block_max_atomic(bm, &a.ds->maxabs_dr_bits);
                        if (threadIdx.x == 0 && cnt) atomicAdd(&a.ds->changed, cnt);
                    }
                }
            }
            if (!grid_barrier(a.ds, ep)) return;
            trace_mark(a, tk);
            continue;
        }
        for (int r = 0; r < p_rounds; ++r) {
            const int i = keep_nbr ? i_one : r * groups_per_round + tid / 8;
            const PressureNbr nb = keep_nbr ? nb0 : pressure_nbr8x2<LdL2>(i, lane, pa);
            float d = pressure_sweep8x2v<LdL2>(i, lane, pa, nb, rin, vin, rout,
                                               last ? nullptr : vout, a.delta_r);
            if (last) {
                float ad = fabsf(d);
                int ch = (i < a.n && (lane & 7) == 0) && ad > 1e-12f;
                int cnt = __syncthreads_count(ch);
                unsigned int bm = __reduce_max_sync(0xffffffffu, ch ? __float_as_uint(ad) : 0u);
                block_max_atomic(bm, &a.ds->maxabs_dr_bits);
                if (threadIdx.x == 0 && cnt) atomicAdd(&a.ds->changed, cnt);
            }
        }
        if (!grid_barrier(a.ds, ep)) return;
        trace_mark(a, tk);
    }
    }
    // (5) apply_brownian_motion (run.py:807-813); the odd-sweep result is copied
    // back into rad, and settle_frames_left -= 1 (run.py:750).  Each new
    // position enters the next rebuild's histogram right away (its P1).
    // With the OU jitter on, the final radii are also summed here for its
    // mean radius (run.py:860-861).
    {
        unsigned int frame = (unsigned int)pa.frame;
        long long rq = 0;
        unsigned int rmx = 0u;  // the largest radius (positive floats order as their bits)
        for (int i = spread_tid(); i < a.n; i += T) {
            if ((a.sweeps & 1) && !a.ptag) a.rad[i] = __ldcg(&a.rad_tmp[i]);
            const float r_i = __ldcg(&a.rad[i]);
            if (a.ou) rq += rad_fixed(r_i);
            rmx = max(rmx, __float_as_uint(r_i));
            brownian_one<LdL2>(i, (unsigned int)i, a.pos, a.strength, a.domain, a.halfL, a.k0,
                               a.k1, frame);
            coop_p1_one(a, geo, i, a.pos, a.rad, a.pos, coop_p1_dst(a, 1));
        }
        if (a.ou) {
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) rq += __shfl_xor_sync(0xffffffffu, rq, o);
            if (lane == 0 && rq) atomicAdd(&a.ds->rad_sum, (unsigned long long)rq);
        }
        block_max_atomic(__reduce_max_sync(0xffffffffu, rmx), &a.ds->rmax_bits);
        if (tid == 0 && a.ds->settle > 0) a.ds->settle -= 1;
    }
    const unsigned int* const fwr[1] = {&a.ds->rmax_bits};
    unsigned int fvr[1];
    if (!grid_barrier(a.ds, ep, &gfl, fwr, 1, fvr)) return;
    trace_mark(a, tk);
    // The PBD sweeps' stencils skip the cells that cannot hold an overlap
    // (radii are fixed during the sweeps; see stencil_ranges_near).  A radius
    // that is not a positive number leaves the full stencil.
    const float rmax_all = a.g.G >= 5 ? __uint_as_float(fvr[0]) : 0.f;
    // (6) PBD passes, each on a fresh grid (run.py:829-846); (7) rebuild (run.py:874)
    // Every rebuild here has its P1 done by the phase that produced the
    // positions (Brownian, then each PBD sweep's lane 0).
    // The OU jitter step (run.py:855-867) runs inside the last sweep's P1.
    for (int k = 0; k < a.pbd_iters; ++k) {
        kk0 = wid < a.n ? __ldcg(&a.slot_of[wid]) : 0;  // as in (2)
        if (!coop_layout(a, geo, k + 1, gfl, tk, ep, lay, rows)) return;
        if (!rows) kk0 = wid < a.n ? __ldcg(&a.slot_of[wid]) : 0;
        const RebuildIdx next{k + 2};
        OuStep ous;
        const bool ou_here = a.ou && k == a.pbd_iters - 1;
        if (ou_here) {
            const unsigned long long sum = *((volatile unsigned long long*)&a.ds->rad_sum);
            ous = OuStep{a.vjit, a.rad, a.ou_p, ou_kick(a.ou_p, mean_from_fixed(sum, a.n)),
                         (unsigned int)pa.frame, 0};
        }
        P1Defer p1;
        int kk_next = kk0;
        for (int r = 0; r < warp_rounds; ++r) {
            const int i = r * W + wid;
            const int kk = kk_next;
            kk_next = i + W < a.n ? __ldcg(&a.slot_of[i + W]) : 0;
            if (i < a.n) {  // warp-uniform
                float4 nv = make_float4(0.f, 0.f, 0.f, 0.f);
                const int pi =
                    rows ? pbd_warp_rows<LdL1>(kk, lane, lay.sp, lay.ci, a.pos_tmp, a.g, lay.cc,
                                               COOP_CAP, a.gap1, a.mdf, a.dmul, &nv, rmax_all,
                                               cell_w)
                         : pbd_warp<LdL1>(kk, lane, lay.sp, lay.ci, a.pos_tmp, a.g, lay.cs,
                                          lay.cc, a.gap1, a.mdf, a.dmul, &nv, lay.cap);
                p1.put(a, geo, lane, pi, nv, a.pos, next, ou_here ? &ous : nullptr);
            }
        }
        p1.flush(a, geo, a.pos, next, ou_here ? &ous : nullptr);
        if (!grid_barrier(a.ds, ep, &gfl)) return;
        trace_mark(a, tk);
    }
    if (!coop_csr(a, geo, a.cnt + (size_t)((a.pbd_iters + 1) % 3) * a.G3, a.pos, nullptr, true,
                  tk, ep))
        return;
    // every block has read the frame counter (it was fetched after max overlap)
    if (a.end_frame && blockIdx.x == 0 && threadIdx.x == 0) a.ds->frame += 1;
    if (a.trace) {
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(&a.trace[a.trace_cap - 1], global_ns());
    }
}

// Per-launch state of the cooperative frame, and count buffers 0 and 1 of
// its rebuilds cleared (the frame clears buffer 2 itself).
__global__ void k_coop_prep(FosDevState* ds, int32_t* cnt01, int m) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    for (int k = t; k < m; k += gridDim.x * blockDim.x) cnt01[k] = 0;
    if (t == 0) {
        ds->coop_epoch += 1u;
        ds->rmax_bits = 0u;
        ds->rmax0_bits = 0u;
        ds->grid_ovf = 0;
        ds->rad_sum = 0ull;
        ds->omax_bits = 0u;
        ds->maxabs_dr_bits = 0u;
        ds->changed = 0;
        ds->bar_count = 0u;
    }
}

// Host side ---------------------------------------------------------------
// Threads per block of the dynamics kernel when every particle has its own
// 8-lane group in one round (the barrier-free pressure sweeps): fewer threads
// with more registers each (80 against 64) for the latency-bound small frame.  Measured on the 10,000-particle foam: 153.1 against 155.7 us
// a plain frame; at 200,000 particles 1,024 threads stay faster (1.47 against
// 1.67 ms), so larger frames keep COOP_THREADS.
#define COOP_THREADS_SMALL 768

static int coop_grid_size(FosCtx* c) {
    if (c->coop_blocks >= 0) return c->coop_blocks;
    int per_sm = 0, per_sm_small = 0;
    if (cudaFuncSetAttribute(k_frame_coop<COOP_THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (COOP_SMALL_G3 + 1) * 4) != cudaSuccess ||
        cudaFuncSetAttribute(k_frame_coop<COOP_THREADS_SMALL>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (COOP_SMALL_G3 + 1) * 4) != cudaSuccess)
        return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_frame_coop<COOP_THREADS>,
                                                      COOP_THREADS,
                                                      (COOP_SMALL_G3 + 1) * 4) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_small,
                                                      k_frame_coop<COOP_THREADS_SMALL>,
                                                      COOP_THREADS_SMALL,
                                                      (COOP_SMALL_G3 + 1) * 4) != cudaSuccess)
        return -1;
    if (per_sm_small < per_sm) per_sm = per_sm_small;  // both shapes take the same grid
    if (per_sm > COOP_BLOCKS_PER_SM) per_sm = COOP_BLOCKS_PER_SM;  // fewest barrier arrivals
    int blocks = per_sm * c->num_sms;
    if (blocks > 1024) blocks = 1024;
    c->coop_blocks = blocks;
    return blocks;
}

bool fos_coop_supported(FosCtx* c) {
    int dev = c->device, ok = 0;
    cudaDeviceGetAttribute(&ok, cudaDevAttrCooperativeLaunch, dev);
    return ok && coop_grid_size(c) > 0;
}

int fos_frame_coop_dynamics(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                            cudaStream_t s, unsigned long long* trace, int trace_cap,
                            int end_frame) {
    int blocks = coop_grid_size(c);
    FOS_REQUIRE(blocks > 0, FOS_E_CUDA, "cooperative frame kernel cannot be resident");
    const int n = st->n;
    const int G3 = c->G * c->G * c->G;
    CoopArgs a;
    memset(&a, 0, sizeof(a));
    a.n = n;
    a.G3 = G3;
    a.chunk = (G3 + blocks - 1) / blocks;
    a.small_grid = G3 <= COOP_SMALL_G3 ? 1 : 0;
    a.pbd_iters = fp->pbd_iters;
    a.sweeps = fp->pressure_iters;
    a.bp_mode = fp->bp_mode;
    a.g = GridGeom{c->G, c->L, c->invL, c->halfL};
    a.pos = st->pos;
    a.pos_tmp = c->pos_tmp;
    a.rad = st->rad;
    a.rad_tmp = c->rad_tmp;
    a.rad_target = st->rad_target;
    a.lmd = st->local_max_depth;
    a.delta_r = st->delta_r;
    a.cc = st->cell_count;
    a.cs = st->cell_start;
    a.ci = st->cell_indices;
    a.cellof = c->cellof;
    a.rank = c->rank;
    a.ci_tmp = c->ci_tmp;
    a.cnt = c->coop_cnt;
    if (c->coop_fixed) {  // the two row sets
        a.rows_ci[0] = c->coop_cfix;
        a.rows_ci[1] = c->coop_idsort;
        a.rows_sp[0] = c->coop_spst;
        a.rows_sp[1] = c->coop_spfix;
    }
    a.slot_of = c->coop_slot;
    a.vol0 = c->pvol;
    a.vol1 = c->pvol + c->max_n;
    // barrier-free pressure sweeps: every particle in one 8-lane group, on
    // the smaller blocks when they still hold every group
    const bool ptag_ok = c->ptag && n <= c->ptag_n && fp->pressure_iters >= 1 &&
                         fp->pressure_iters <= FOS_PTAG_SWEEPS;
    int threads = COOP_THREADS;
    if (ptag_ok && (long long)n * COOP_PLANES <= (long long)blocks * COOP_THREADS_SMALL)
        threads = COOP_THREADS_SMALL;
    if (ptag_ok && (long long)n * COOP_PLANES <= (long long)blocks * threads)
        a.ptag = c->ptag;
    else
        a.pnbr = c->pnbr;
    a.part = c->coop_part;
    a.bsum = c->coop_bsum;
    a.sp = c->sorted;
    a.ds = c->ds;
    a.gap1 = c->gap1;
    a.mdf = c->mdf;
    a.dmul = c->dmul;
    a.eps = c->eps;
    a.contact_tol = c->contact_tol;
    a.contact_tol_d = c->p.contact_tol;
    a.alpha = (float)(1.0 - pow(0.05, 1.0 / (double)(fp->adjustment_frames > 1 ? fp->adjustment_frames : 1)));
    a.max_step = (float)fp->max_step_pct;
    a.rmin = (float)fp->r_min;
    a.rmax = (float)fp->r_max;
    a.pa = PressureArgs{n,
                        0,
                        fp->max_eq_nei,
                        (float)fp->pressure_k,
                        (float)fp->pressure_exp,
                        (float)fp->pressure_pair_cap,
                        (float)fp->r_min,
                        (float)fp->r_max,
                        c->face_ids,
                        c->fsc,
                        0};
    a.strength = (float)fp->brownian_strength;
    a.domain = c->L;
    a.halfL = (float)(0.5 * (double)c->L);
    a.k0 = (uint32_t)fp->seed;
    a.k1 = (uint32_t)(fp->seed >> 32);
    a.ou = fp->ou_jitter ? 1 : 0;
    a.vjit = st->v_jit;
    a.ou_p = ou_params(fp->jitter_rms, fp->jitter_tau, fp->max_drift_fraction, c->p.gap_fraction,
                       (float)fp->dt, c->L, c->invL, fp->seed);
    a.trace = trace;
    a.trace_cap = trace_cap;
    a.end_frame = end_frame;

    FOS_REQUIRE(fp->max_eq_nei <= 16, FOS_E_ARG, "cooperative frame needs max_eq_nei <= 16");
    FOS_REQUIRE(n <= (1 << 26), FOS_E_ARG, "cooperative frame supports up to 2^26 particles");
    FOS_REQUIRE(!a.ou || fp->pbd_iters >= 1, FOS_E_ARG,
                "cooperative frame runs the OU jitter inside a PBD sweep: pbd_iters >= 1");
    k_coop_prep<<<fos_blocks(2LL * G3, 256) < 64 ? fos_blocks(2LL * G3, 256) : 64, 256, 0, s>>>(
        c->ds, c->coop_cnt, 2 * G3);
    FOS_LAUNCHED(c);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = a.small_grid ? (size_t)(G3 + 1) * 4 : 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (threads == COOP_THREADS_SMALL)
        FOS_CUDA(cudaLaunchKernelEx(&cfg, k_frame_coop<COOP_THREADS_SMALL>, a));
    else
        FOS_CUDA(cudaLaunchKernelEx(&cfg, k_frame_coop<COOP_THREADS>, a));
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// Cooperative dynamics of one frame with %globaltimer stamps after every phase
// (block 0's view): stamp 0 at kernel entry, then one per grid barrier.
extern "C" int fos_frame_trace(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                               long long* ns_host, int cap, int* count, fos_stream_t s) {
    FOS_REQUIRE(c && st && fp && ns_host && count && cap >= 3, FOS_E_ARG, "NULL argument or cap < 3");
    FOS_REQUIRE(fos_coop_supported(c), FOS_E_STATE, "cooperative launch unsupported");
    unsigned long long* d = nullptr;
    FOS_CUDA(cudaMalloc(&d, (size_t)cap * 8));
    cudaMemsetAsync(d, 0, (size_t)cap * 8, s);
    int rc = fos_frame_coop_dynamics(c, st, fp, s, d, cap);
    if (rc == FOS_OK) {
        cudaError_t e = cudaMemcpyAsync(ns_host, d, (size_t)cap * 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fos_cuda_fail(e, "trace readback", __FILE__, __LINE__);
    }
    cudaFree(d);
    int k = 0;
    while (k < cap - 2 && ns_host[k] != 0) ++k;
    *count = k;
    return rc;
}
