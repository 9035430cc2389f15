// coop.cuh -- building blocks of the persistent cooperative kernels: the
// block scan, the bounded grid barrier's tracing hook, and the hash-grid
// rebuild as grid-barrier phases (grid.py:145-309 / run.py:476-504).  The
// single-foam frame kernel (frame_coop.cu) and the ensemble frame kernel
// (ensemble.cu) share them; a Geo policy maps a particle to its cell:
//   UniGeo   one periodic grid of G^3 cells;
//   the ensemble's policy, foam f's grid at its offset in the packed table.
#pragma once

#include "phases.cuh"

// block size and resident blocks per SM of the single-foam cooperative kernel
#ifndef COOP_THREADS
#define COOP_THREADS 1024
#endif
#ifndef COOP_BLOCKS_PER_SM
#define COOP_BLOCKS_PER_SM 1
#endif
#define COOP_SMALL_G3 12288  // cell tables up to this size are scanned per block in smem

struct UniGeo {
    int G;
    float L, invL, halfL;
    __device__ __forceinline__ int cell(int, float wx, float wy, float wz) const {
        return cell_of_wrapped(wx, wy, wz, invL, halfL, G);
    }
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Records a timestamp in trace[k++] from block 0, thread 0 (tracing only).
template <class Args>
__device__ __forceinline__ void trace_mark(const Args& a, int& k) {
    if (a.trace && blockIdx.x == 0 && threadIdx.x == 0 && k < a.trace_cap - 2) a.trace[k] = global_ns();
    ++k;
}

// Block-wide exclusive scan (one value per thread, blockDim <= 1024).
__device__ __forceinline__ int coop_block_scan(int v, int* total) {
    __shared__ int s_w[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        int t = lane < nw ? s_w[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) s_w[lane] = t;
    }
    __syncthreads();
    int base = w > 0 ? s_w[w - 1] : 0;
    *total = s_w[(blockDim.x >> 5) - 1];
    __syncthreads();
    return base + x - v;
}

#define COOP_CAP 32  // slots per cell of the fixed-capacity rows (one warp sorts a row)

// Thread index for per-particle loops of the persistent kernels: 32
// consecutive particles per warp (coalesced accesses), consecutive warps of
// particles on consecutive blocks, so n < gridDim.x * blockDim.x particles
// spread over every SM instead of filling the first blocks.  A bijection of
// [0, gridDim.x * blockDim.x) for blockDim.x a multiple of 32.
__device__ __forceinline__ int spread_tid() {
    return (int)((((threadIdx.x >> 5) * gridDim.x + blockIdx.x) << 5) + (threadIdx.x & 31));
}

// One rebuild's grid as its consumers (max overlap, PBD) see it.  The CSR
// form and the sorted fixed-capacity rows (coop_grid) hold each cell's
// particles in ascending index order, so a stencil walk visits candidates in
// the reference's order; the frames' arrival-order rows do not, and their PBD
// sweeps order the hits themselves (pbd_warp_rows).  slot_of[i] (an argument
// array) is particle i's slot in whichever form was built.
struct CoopLayout {
    const int32_t* ci;  // particle at slot k
    const float4* sp;   // (pos, rad) at slot k
    const int32_t* cs;  // CSR form: first slot of each cell
    const int32_t* cc;  // particles per cell
    int cap;            // fixed-capacity form (> 0): cell c's slots start at c * cap
    __device__ __forceinline__ int start(int c) const { return cap ? c * cap : __ldcg(&cs[c]); }
    __device__ __forceinline__ int count(int c) const { return __ldcg(&cc[c]); }
};

// P1 of a rebuild for one particle whose source position is v and radius r:
// wrap v into dst[i], find its cell, take an arrival rank in the count
// buffer `par` (all-zero before the first arrival) and drop the particle into
// slot rank of the cell's fixed-capacity rows: its index into cfix and its
// (wrapped position, radius) into spst, so a row sort needs no gather (a
// full row sets overflow bit par, and the rebuild then takes the CSR form).
// A phase that produces particle i's new position can run this for the next
// rebuild right away, so that rebuild needs no P1 phase or barrier of its own.
// Where a P1 drops its particle: the count buffer, the rows (cfix / spst, or
// NULL for none), the slot map (slot[i] = the particle's row slot; NULL for
// none) and the overflow bit that a full row sets in *ovf_word.
struct P1Dst {
    int32_t* cnt;
    int32_t* cfix;
    float4* spst;
    int32_t* slot;
    unsigned int* ovf_word;
    unsigned int ovf_bit;
};

// The alternating form: count buffer `par`, the one set of rows (sorted into
// a second set by the rebuild), no slot map.
template <class Args>
__device__ __forceinline__ P1Dst coop_p1_par(const Args& a, int par) {
    return P1Dst{par ? a.cnt2 : a.cnt, a.cfix, a.spst, nullptr, (unsigned int*)&a.ds->grid_ovf,
                 1u << par};
}

template <class Args, class Geo>
__device__ __forceinline__ void coop_p1_val(const Args& a, const Geo& geo, int i, float3 v,
                                            float r, float* dst, const P1Dst& t) {
    float wx = grid_wrap(v.x, geo.L, geo.invL);
    float wy = grid_wrap(v.y, geo.L, geo.invL);
    float wz = grid_wrap(v.z, geo.L, geo.invL);
    dst[3 * i + 0] = wx;
    dst[3 * i + 1] = wy;
    dst[3 * i + 2] = wz;
    int c = geo.cell(i, wx, wy, wz);
    a.cellof[i] = c;
    int k = atomicAdd(&t.cnt[c], 1);
    a.rank[i] = k;
    if (t.cfix) {
        if (k < COOP_CAP) {
            const size_t slot = (size_t)c * COOP_CAP + k;
            t.cfix[slot] = i;
            t.spst[slot] = make_float4(wx, wy, wz, r);
            if (t.slot) t.slot[i] = (int)slot;
        } else {
            atomicOr(t.ovf_word, t.ovf_bit);
        }
    }
}

template <class Args, class Geo>
__device__ __forceinline__ void coop_p1_one(const Args& a, const Geo& geo, int i, const float* src,
                                            const float* rad, float* dst, const P1Dst& t) {
    float3 v = make_float3(__ldcg(&src[3 * i + 0]), __ldcg(&src[3 * i + 1]),
                           __ldcg(&src[3 * i + 2]));
    coop_p1_val(a, geo, i, v, rad ? __ldcg(&rad[i]) : 0.f, dst, t);
}

// With ou != NULL each deferred particle first takes the frame's OU jitter
// step (apply_brownian + integrate_jitter, run.py:855-867) at its new
// position, which is what the rebuild after the last PBD sweep then sees.
struct OuStep {
    float* vjit;
    const float* rad;
    OuParams o;
    float kick;           // sigma * sqrt(dt)
    unsigned int frame;
    int ctr_base;         // Philox counter = i - ctr_base (index within the foam)
    // batched ensembles: per-foam values in place of kick, o.k0/o.k1 and
    // ctr_base, looked up through foam_of[i] (NULL for a single foam)
    const int32_t* foam_of = nullptr;
    const float* kick_f = nullptr;   // sigma * sqrt(dt) of each foam's mean radius
    const uint2* key_f = nullptr;    // each foam's Philox key (its seed)
    const int32_t* base_f = nullptr; // each foam's first particle index
};

// A P1 target given directly.
template <class Args>
__device__ __forceinline__ const P1Dst& p1_target(const Args&, const P1Dst& t) {
    return t;
}

// Tgt: a P1Dst, or any type with a p1_target(args, tgt) overload that builds
// one when the deferred particles are flushed (fewer live registers).
struct P1Defer {
    int i = -1;
    float4 v;  // new position, radius
    int q = 0;
    template <class Args, class Geo, class Tgt>
    __device__ __forceinline__ void put(const Args& a, const Geo& geo, int lane, int pi, float4 pv,
                                        float* dst, const Tgt& t, const OuStep* ou = nullptr) {
        const int slot = q & 31;
        const int si = __shfl_sync(0xffffffffu, pi, 0);
        const float sx = __shfl_sync(0xffffffffu, pv.x, 0);
        const float sy = __shfl_sync(0xffffffffu, pv.y, 0);
        const float sz = __shfl_sync(0xffffffffu, pv.z, 0);
        const float sr = __shfl_sync(0xffffffffu, pv.w, 0);
        if (lane == slot) {
            i = si;
            v = make_float4(sx, sy, sz, sr);
        }
        ++q;
        if (slot == 31) flush(a, geo, dst, t, ou);
    }
    template <class Args, class Geo, class Tgt>
    __device__ __forceinline__ void flush(const Args& a, const Geo& geo, float* dst, const Tgt& t,
                                          const OuStep* ou = nullptr) {
        if (i >= 0) {
            float3 p = make_float3(v.x, v.y, v.z);
            if (ou) {
                if (ou->foam_of) {
                    const int f = __ldg(&ou->foam_of[i]);
                    OuParams o = ou->o;
                    const uint2 k = __ldg(&ou->key_f[f]);
                    o.k0 = k.x;
                    o.k1 = k.y;
                    p = ou_one(i, (unsigned int)(i - __ldg(&ou->base_f[f])), p, ou->vjit, v.w,
                               __ldcg(&ou->kick_f[f]), o, ou->frame);
                } else {
                    p = ou_one(i, (unsigned int)(i - ou->ctr_base), p, ou->vjit, v.w, ou->kick,
                               ou->o, ou->frame);
                }
            }
            coop_p1_val(a, geo, i, p, v.w, dst, p1_target(a, t));
        }
        i = -1;
    }
};

// The CSR form of a rebuild whose P1 filled count buffer `cnt` (cellof and
// rank written): small tables (G3 <= COOP_SMALL_G3) scan the whole table in
// every block's shared memory (block 0 writes cell_count/cell_start) and
// scatter ranks, then place stably; large tables use a chunked four-phase
// form.  CSR ci/cc/cs and slot_of are written, and sp when rad is given.
// Ends with a grid barrier unless last; false if a barrier timed out.
template <class Args, class Geo>
__device__ bool coop_csr(const Args& a, const Geo& geo, const int32_t* cnt, const float* dst,
                         const float* rad, bool last, int& tk, unsigned int& ep) {
    extern __shared__ int s_tab[];  // small form: G3 + 1 exclusive starts
    const int T = gridDim.x * blockDim.x;
    if (a.small_grid) {
        // P2: the whole count table into shared memory with coalesced loads
        // (each block reads each line once), a scan per block (each thread
        // takes `per` consecutive cells), then the rank scatter
        for (int c = threadIdx.x; c < a.G3; c += blockDim.x) s_tab[c] = __ldcg(&cnt[c]);
        __syncthreads();
        const int per = (a.G3 + blockDim.x - 1) / blockDim.x;
        const int b0 = threadIdx.x * per, b1 = min(a.G3, b0 + per);
        int sum = 0;
        for (int c = b0; c < b1; ++c) sum += s_tab[c];
        int tot;
        int run = coop_block_scan(sum, &tot);
        for (int c = b0; c < b1; ++c) {
            int v = s_tab[c];
            s_tab[c] = run;
            run += v;
        }
        if (threadIdx.x == 0) s_tab[a.G3] = tot;
        __syncthreads();
        if (blockIdx.x == 0) {
            for (int c = threadIdx.x; c < a.G3; c += blockDim.x) {
                a.cs[c] = s_tab[c];
                a.cc[c] = s_tab[c + 1] - s_tab[c];
            }
        }
        for (int i = spread_tid(); i < a.n; i += T)
            a.ci_tmp[s_tab[__ldcg(&a.cellof[i])] + __ldcg(&a.rank[i])] = i;
        if (!grid_barrier(a.ds, ep)) return false;
        trace_mark(a, tk);
        // P3: stable placement from the block's copy of the starts
        for (int i = spread_tid(); i < a.n; i += T) {
            int c = __ldcg(&a.cellof[i]);
            int b = s_tab[c], e = s_tab[c + 1];
            int r = 0;
            for (int k = b; k < e; ++k) r += __ldcg(&a.ci_tmp[k]) < i;
            a.ci[b + r] = i;
            a.slot_of[i] = b + r;
            if (rad)
                a.sp[b + r] = make_float4(__ldcg(&dst[3 * i + 0]), __ldcg(&dst[3 * i + 1]),
                                          __ldcg(&dst[3 * i + 2]), __ldcg(&rad[i]));
        }
        if (!last && !grid_barrier(a.ds, ep)) return false;
        trace_mark(a, tk);
        return true;
    }
    // P2: each block scans its chunk of cells (local exclusive offsets + total)
    {
        int c0 = blockIdx.x * a.chunk;
        int carry = 0;
        for (int base = c0; base < c0 + a.chunk; base += blockDim.x) {
            int c = base + threadIdx.x;
            bool in = c < c0 + a.chunk && c < a.G3;
            int v = in ? __ldcg(&cnt[c]) : 0;
            int tot;
            int ex = coop_block_scan(v, &tot);
            if (in) {
                a.part[c] = carry + ex;
                a.cc[c] = v;
            }
            carry += tot;
        }
        if (threadIdx.x == 0) a.bsum[blockIdx.x] = carry;
    }
    if (!grid_barrier(a.ds, ep)) return false;
    trace_mark(a, tk);
    // P3: block-sum prefix, final cell starts of this block's chunk, rank scatter
    {
        __shared__ int s_pre[1024];  // gridDim.x <= 1024 (checked on the host)
        int v = threadIdx.x < gridDim.x ? __ldcg(&a.bsum[threadIdx.x]) : 0;
        int tot;
        int ex = coop_block_scan(v, &tot);
        s_pre[threadIdx.x] = ex;
        __syncthreads();
        int c0 = blockIdx.x * a.chunk;
        for (int c = c0 + threadIdx.x; c < c0 + a.chunk && c < a.G3; c += blockDim.x) {
            a.cs[c] = __ldcg(&a.part[c]) + s_pre[blockIdx.x];
        }
        for (int i = spread_tid(); i < a.n; i += T) {
            int c = __ldcg(&a.cellof[i]);
            int slot = __ldcg(&a.part[c]) + s_pre[c / a.chunk] + __ldcg(&a.rank[i]);
            a.ci_tmp[slot] = i;
        }
    }
    if (!grid_barrier(a.ds, ep)) return false;
    trace_mark(a, tk);
    // P4: stable placement: slot = cell start + #(lower-indexed particles in the cell)
    for (int i = spread_tid(); i < a.n; i += T) {
        int c = __ldcg(&a.cellof[i]);
        int b = __ldcg(&a.cs[c]), e = b + __ldcg(&a.cc[c]);
        int r = 0;
        for (int k = b; k < e; ++k) r += __ldcg(&a.ci_tmp[k]) < i;
        a.ci[b + r] = i;
        a.slot_of[i] = b + r;
        if (rad) {
            a.sp[b + r] = make_float4(__ldcg(&dst[3 * i + 0]), __ldcg(&dst[3 * i + 1]),
                                      __ldcg(&dst[3 * i + 2]), __ldcg(&rad[i]));
        }
    }
    if (!last && !grid_barrier(a.ds, ep)) return false;
    trace_mark(a, tk);
    return true;
}

// Rebuild of the hash grid from src into dst (wrapped) with count buffer
// `par` (rebuilds alternate buffers, so the next rebuild's P1 can run while
// this grid is still being read).  Ends with a grid barrier unless last;
// returns false if a barrier timed out; *out receives the layout.
//   P1        histogram + arrival rank + fixed-capacity row slot (skipped
//             when p1_done: the previous phase ran coop_p1_* for every
//             particle with the same src, dst and par);
//   fixed     when the rows did not overflow, want_csr is false and rad is
//             given: one phase, one warp per cell sorts its row by particle
//             index and writes the (pos, rad) copy;
//   CSR       otherwise (the user-visible final rebuild always): coop_csr.
// The second phase also clears the other count buffer and overflow bit for
// the rebuild after this one.
template <class Args, class Geo>
__device__ bool coop_grid(const Args& a, const Geo& geo, const float* src, float* dst,
                          const float* rad, bool last, int& tk, unsigned int& ep, bool p1_done,
                          int par, bool want_csr, CoopLayout* out) {
    const int T = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t* cnt = par ? a.cnt2 : a.cnt;
    int32_t* cnt_next = par ? a.cnt : a.cnt2;
    if (!p1_done) {
        const P1Dst t = coop_p1_par(a, par);
        for (int i = spread_tid(); i < a.n; i += T) coop_p1_one(a, geo, i, src, rad, dst, t);
        if (!grid_barrier(a.ds, ep)) return false;
        trace_mark(a, tk);
    }
    const bool ovf = ((*((volatile int*)&a.ds->grid_ovf)) >> par) & 1;
    for (int c = tid; c < a.G3; c += T) cnt_next[c] = 0;
    if (tid == 0) atomicAnd(&a.ds->grid_ovf, ~(1 << (par ^ 1)));
    if (a.cfix && !want_csr && !ovf && rad) {
        // fixed-capacity rows: sort each cell's (<= COOP_CAP) arrivals by
        // index.  A warp takes two cells per round; their counts are loaded
        // one round ahead, so a round waits for one load latency, and only
        // the occupied slots of a row are read (the slots past the count hold
        // stale entries that would mostly come from DRAM).
        const int lane = threadIdx.x & 31, W = T >> 5, wid = tid >> 5;
        int mn[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) mn[h] = wid + h * W < a.G3 ? __ldcg(&cnt[wid + h * W]) : 0;
        for (int c0 = wid; c0 < a.G3; c0 += 2 * W) {
            const int cc2[2] = {c0, c0 + W};
            int m[2], id[2];
            float4 pr[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                m[h] = mn[h];  // <= COOP_CAP; 0 past the table
                const int cn = c0 + (2 + h) * W;
                mn[h] = cn < a.G3 ? __ldcg(&cnt[cn]) : 0;
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const size_t base = (size_t)cc2[h] * COOP_CAP;
                id[h] = lane < m[h] ? __ldcg(&a.cfix[base + lane]) : 0;
                pr[h] = lane < m[h] ? __ldcg(&a.spst[base + lane]) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int key = lane < m[h] ? id[h] : 0x7fffffff;
                int r = 0;
                for (int k = 0; k < m[h]; ++k) r += __shfl_sync(0xffffffffu, key, k) < key;
                if (lane < m[h]) {
                    const size_t base = (size_t)cc2[h] * COOP_CAP;
                    a.idsort[base + r] = key;
                    a.spfix[base + r] = pr[h];
                    a.slot_of[key] = (int)(base + r);
                }
            }
        }
        if (out) *out = CoopLayout{a.idsort, a.spfix, nullptr, cnt, COOP_CAP};
        if (!last && !grid_barrier(a.ds, ep)) return false;
        trace_mark(a, tk);
        return true;
    }
    if (out) *out = CoopLayout{a.ci, a.sp, a.cs, a.cc, 0};
    return coop_csr(a, geo, cnt, dst, rad, last, tk, ep);
}

