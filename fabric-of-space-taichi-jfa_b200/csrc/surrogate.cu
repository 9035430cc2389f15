// surrogate.cu -- learned face-sharing-count surrogate.  It has no
// counterpart in the reference, which reuses the last JFA's fsc on the frames
// between JFA runs (run.py:1230-1261).
//
// Pipeline on a context (fos_surrogate_pairs, then fos_surrogate_predict):
//   k_sur_pairs    one warp per particle (hash-cell order) scans the cells
//                  within cutoff * (r_i + r_max), counts every candidate in
//                  i's 13-bin histogram and appends the pairs i owns to its
//                  fixed-capacity segment (pair {a < b} belongs to a when
//                  a + b is odd, to b when it is even);
//   k_sur_mlp_seg  one warp per group of 4 owners walks their segments 16
//                  pairs at a time: the lanes build the features of the 16
//                  pairs (standardised, BF16) in shared memory, then both
//                  hidden layers run on the tensor cores (mma.sync m16n8k16,
//                  BF16 x BF16 -> FP32); the first layer's accumulators are
//                  re-packed in registers as the second layer's A operand; the
//                  64 -> 1 layer, sigmoid and the per-particle sums
//                  (fixed-point, so the result does not depend on the order of
//                  the atomics) follow in registers;
//   k_sur_fsc      fixed-point sums -> the model's estimate s;
//   k_sur_combine  s -> the FSC f the controller sees (absolute: f = s;
//                  anchored: f = last JFA fsc + s - s at that JFA).
// Training (fos_surrogate_train_step): k_sur_train runs forward + backward
// of 64-row tiles in shared memory with FP32 CUDA-core arithmetic and keeps
// each block's gradient in registers; k_sur_adam reduces the per-block
// gradients in a fixed order (deterministic) and applies Adam.
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include "phases.cuh"

#define SUR_NB FOS_SUR_BINS
#define SUR_NF FOS_SUR_FEATURES
#define SUR_H FOS_SUR_HIDDEN
#define SUR_CAP FOS_SUR_PAIR_CAP
#define SUR_NPARAM FOS_SUR_NPARAM

#define SUR_OFF_W1 0
#define SUR_OFF_B1 (SUR_OFF_W1 + SUR_H * SUR_NF)
#define SUR_OFF_W2 (SUR_OFF_B1 + SUR_H)
#define SUR_OFF_B2 (SUR_OFF_W2 + SUR_H * SUR_H)
#define SUR_OFF_W3 (SUR_OFF_B2 + SUR_H)
#define SUR_OFF_B3 (SUR_OFF_W3 + SUR_H)
static_assert(SUR_OFF_B3 + 1 == SUR_NPARAM, "parameter layout");

#define SUR_FIX 1048576.0f  // 2^20: fixed-point scale of the per-particle sums

// ------------------------------------------------------------ model object
struct FosSurrogate {
    int device = 0;
    float cutoff = 2.5f;
    float* params = nullptr;  // [NPARAM] FP32 master weights
    float* adam_m = nullptr;  // [NPARAM]
    float* adam_v = nullptr;  // [NPARAM]
    float* part = nullptr;    // [nblk][NPARAM + 1] per-block gradients + loss
    float* norm = nullptr;    // mu[16], 1/sd[16] (FP32)
    __nv_bfloat16* wbf = nullptr;  // W1 [64][16], W2 [64][64], w3 [64] in BF16
    __nv_bfloat16* xb = nullptr;   // forward() scratch: standardised BF16 features
    size_t xb_rows = 0;
    int nblk = 0;
    int num_sms = 0;
    long long step = 0;
    float host_mu[SUR_NF], host_sd[SUR_NF];
};

// Per-context buffers of the pair search and inference.
struct FosSurBufs {
    int32_t* pj = nullptr;       // [n][CAP] partner index
    float* pnd = nullptr;        // [n][CAP] normalised distance
    int32_t* pcount = nullptr;   // [n + 1]
    int32_t* pstart = nullptr;   // [n + 1] exclusive scan; pstart[n] = P
    int32_t* hist = nullptr;     // [n][13]
    unsigned long long* acc = nullptr;  // [n] fixed-point probability sums
    float* fscf = nullptr;       // [n] the FSC f the controller sees (float)
    int32_t* fsci = nullptr;     // [n] rint(fscf)
    int32_t* prev = nullptr;     // [n] previous JFA fsc (judge baseline)
    float* raw = nullptr;        // [n] model estimate s of the last inference
    float* anchor = nullptr;     // [n] s at the last judged JFA frame
    int* anchor_valid = nullptr; // device flag: anchor holds a JFA frame's s
    unsigned long long* cnt = nullptr;  // counters, see SurCnt
    int n = 0;                   // particles of the last pair build
    float cutoff = 0.f;          // cutoff of the last pair build
};

enum SurCnt {
    SC_OVERFLOW = 0,
    SC_JUDGED,
    SC_EXACT,
    SC_WITHIN1,
    SC_STALE_EXACT,
    SC_STALE_WITHIN1,
    SC_ABS_ERR,        // fixed point 2^-20
    SC_STALE_ABS_ERR,  // integer
    SC_N
};

// ------------------------------------------------------------ pair search
// The candidates of the particle at cell-ordered slot kk (one warp): g, cs
// and cc describe the hash grid the particle lives in (a batched ensemble
// passes its foam's grid: cs / cc at the foam's cell offset, whose entries
// are slots of the packed cell-ordered arrays), r_max that grid's radius bound.
__device__ __forceinline__ void sur_pairs_warp(int kk, int lane, const float4* __restrict__ sp,
                                               const int32_t* __restrict__ ci, const GridGeom g,
                                               const int32_t* __restrict__ cs,
                                               const int32_t* __restrict__ cc, float cutoff,
                                               float r_max, int32_t* __restrict__ pj,
                                               float* __restrict__ pnd,
                                               int32_t* __restrict__ pcount,
                                               int32_t* __restrict__ hist,
                                               unsigned long long* __restrict__ counters) {
    const float4 me = sp[kk];
    const int i = ci[kk];
    const int G = g.G;
    // home cell exactly as the grid build assigns it
    const float wx = grid_wrap(me.x, g.L, g.invL), wy = grid_wrap(me.y, g.L, g.invL),
                wz = grid_wrap(me.z, g.L, g.invL);
    const int cid = cell_of_wrapped(wx, wy, wz, g.invL, g.halfL, G);
    const int hx = cid / (G * G), hy = (cid / G) % G, hz = cid % G;
    // every partner within cutoff * (r_i + r_j) <= cutoff * (r_i + r_max) lies
    // at most floor(reach_dist / cell) + 1 cells away along each axis
    const float cellw = g.L / (float)G;
    const int reach = (int)floorf(cutoff * (me.w + r_max) / cellw) + 1;
    int span = 2 * reach + 1;
    int r0 = -reach;
    if (span >= G) {  // the whole axis, each cell once
        span = G;
        r0 = 0;
    }
    const float inv_cut_bins = (float)SUR_NB / cutoff;
    int h[SUR_NB];
#pragma unroll
    for (int b = 0; b < SUR_NB; ++b) h[b] = 0;
    int cnt = 0;
    const int z0 = wrap_mod(hz + r0, G);
    const int len1 = span < G - z0 ? span : G - z0;
    // Cells beyond reach_dist = cutoff * (r_i + r_max) of the particle hold no
    // candidate: a column whose nearest point in x-y is farther is skipped,
    // and each other column's z run is trimmed to the cells its z-extent
    // reaches (bounds from the particle's offset in its home cell, less a
    // margin for float error; the run stays in the same cyclic order, so the
    // candidates are a subsequence of the untrimmed walk).  Needs span < G,
    // so that each offset is a distinct cell.
    const bool trim = span < G;
    const float margin = 1e-5f * g.L + 1e-6f;
    const float rd = cutoff * (me.w + r_max) * 1.0001f + margin;
    const float rel[3] = {wx - ((float)hx * cellw - g.halfL), wy - ((float)hy * cellw - g.halfL),
                          wz - ((float)hz * cellw - g.halfL)};
    // The span x span columns each hold a z run of one or two contiguous
    // cell ranges ("pieces").  32 pieces at a time: each lane loads one
    // piece's particle range, a warp scan lays the ranges end to end, and the
    // warp walks the concatenation 32 candidates per step, each lane locating
    // its piece by a shuffle binary search.  The candidate order is the same
    // as a piece-by-piece scan, and no lane waits on a serial chain of
    // cell_start loads.
    const int npieces = 2 * span * span;
    for (int pb = 0; pb < npieces; pb += 32) {
        const int pc = pb + lane;
        int k0 = 0, len = 0;
        if (pc < npieces) {
            const int col = pc >> 1, piece = pc & 1;
            const int ox = col / span, oy = col - (col / span) * span;
            int za = piece == 0 ? z0 : 0;
            int zl = piece == 0 ? len1 : span - len1;
            if (trim) {
                const int o2[2] = {r0 + ox, r0 + oy};
                float bxy2 = 0.f;
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const int o = o2[a];
                    float b = o == 0 ? 0.f
                                     : (o < 0 ? rel[a] + (float)(-o - 1) * cellw
                                              : (cellw - rel[a]) + (float)(o - 1) * cellw);
                    b = fmaxf(0.f, b - margin);
                    bxy2 += b * b;
                }
                if (bxy2 > rd * rd) {
                    zl = 0;
                } else {
                    const float sz = sqrtf(rd * rd - bxy2) + margin;
                    const int kneg = min(reach, max(0, (int)floorf((sz - rel[2]) / cellw) + 1));
                    const int kpos =
                        min(reach, max(0, (int)floorf((sz - (cellw - rel[2])) / cellw) + 1));
                    const int length = kneg + kpos + 1;
                    const int zs = wrap_mod(hz - kneg, G);
                    const int l1 = length < G - zs ? length : G - zs;
                    za = piece == 0 ? zs : 0;
                    zl = piece == 0 ? l1 : length - l1;
                }
            }
            if (zl > 0) {
                const int nx = wrap_mod(hx + r0 + ox, G);
                const int ny = wrap_mod(hy + r0 + oy, G);
                const int c0 = (nx * G + ny) * G + za, c1 = c0 + zl - 1;
                k0 = __ldg(&cs[c0]);
                len = __ldg(&cs[c1]) + __ldg(&cc[c1]) - k0;
            }
        }
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int excl = incl - len;
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        for (int tb = 0; tb < total; tb += 32) {
            const int t = tb + lane;
            // largest piece q with excl[q] <= t (empty pieces never win)
            int q = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int e = __shfl_sync(0xffffffffu, excl, q + step);
                if (e <= t) q += step;
            }
            const int kq = __shfl_sync(0xffffffffu, k0, q);
            const int eq = __shfl_sync(0xffffffffu, excl, q);
            const int k = kq + (t - eq);
            bool cand = false;
            float nd = 0.f;
            int j = -1;
            if (t < total && k != kk) {
                const float4 qv = sp[k];
                const float dx = grid_wrap(fsub(qv.x, me.x), g.L, g.invL);
                const float dy = grid_wrap(fsub(qv.y, me.y), g.L, g.invL);
                const float dz = grid_wrap(fsub(qv.z, me.z), g.L, g.invL);
                const float dist = sqrtf(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
                nd = fdiv(dist, fadd(me.w, qv.w));
                cand = nd < cutoff;
                if (cand) {
                    int bin = (int)fmul(nd, inv_cut_bins);
                    bin = bin < SUR_NB - 1 ? bin : SUR_NB - 1;
#pragma unroll
                    for (int b = 0; b < SUR_NB; ++b) h[b] += (bin == b) ? 1 : 0;
                    j = ci[k];
                }
            }
            // balanced ownership of the unordered pair {i, j}
            const bool keep = cand && ((i < j) == (((i + j) & 1) != 0));
            const unsigned int m = __ballot_sync(0xffffffffu, keep);
            const int slot = cnt + __popc(m & ((1u << lane) - 1u));
            if (keep && slot < SUR_CAP) {
                pj[(size_t)i * SUR_CAP + slot] = j;
                pnd[(size_t)i * SUR_CAP + slot] = nd;
            }
            cnt += __popc(m);
        }
    }
#pragma unroll
    for (int b = 0; b < SUR_NB; ++b) {
        int v = h[b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) hist[(size_t)i * SUR_NB + b] = v;
    }
    if (lane == 0) {
        pcount[i] = cnt < SUR_CAP ? cnt : SUR_CAP;
        if (cnt > SUR_CAP) atomicAdd(&counters[SC_OVERFLOW], 1ull);
    }
}

__global__ void __launch_bounds__(256) k_sur_pairs(const float4* __restrict__ sp,
                                                   const int32_t* __restrict__ ci, int n, GridGeom g,
                                                   const int32_t* __restrict__ cs,
                                                   const int32_t* __restrict__ cc, float cutoff,
                                                   float r_max, int32_t* __restrict__ pj,
                                                   float* __restrict__ pnd,
                                                   int32_t* __restrict__ pcount,
                                                   int32_t* __restrict__ hist,
                                                   unsigned long long* __restrict__ counters) {
    const int kk = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (kk >= n) return;  // warp-uniform
    sur_pairs_warp(kk, threadIdx.x & 31, sp, ci, g, cs, cc, cutoff, r_max, pj, pnd, pcount, hist,
                   counters);
}

// The same over a batched ensemble's packed grid: particle i of foam f =
// foam_of[i] searches foam f's hash grid (fG[f] cells a side, its cell
// table at fcell[f]) with foam f's radius bound frmax[f].  Pairs never cross
// foams, since each grid holds only its foam's particles.
__global__ void __launch_bounds__(256) k_sur_pairs_ens(
    const float4* __restrict__ sp, const int32_t* __restrict__ ci, int n, float L, float invL,
    float halfL, const int32_t* __restrict__ foam_of, const int32_t* __restrict__ fG,
    const int32_t* __restrict__ fcell, const float* __restrict__ frmax,
    const int32_t* __restrict__ cs, const int32_t* __restrict__ cc, float cutoff,
    int32_t* __restrict__ pj, float* __restrict__ pnd, int32_t* __restrict__ pcount,
    int32_t* __restrict__ hist, unsigned long long* __restrict__ counters) {
    const int kk = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (kk >= n) return;  // warp-uniform
    const int f = __ldg(&foam_of[__ldg(&ci[kk])]);
    const GridGeom g{__ldg(&fG[f]), L, invL, halfL};
    const int off = __ldg(&fcell[f]);
    sur_pairs_warp(kk, threadIdx.x & 31, sp, ci, g, cs + off, cc + off, cutoff, __ldg(&frmax[f]),
                   pj, pnd, pcount, hist, counters);
}

// Memory features of pair (i, j) from the last JFA frame (its neighbour
// lists nl [n][32] with used counts, and its fsc): whether the two were
// neighbours (j in i's list or i in j's), and fsc_i + fsc_j.
// The rows are read as 16-byte vectors (a row is 128 bytes, 16-byte aligned).
__device__ __forceinline__ bool sur_in_row(const int32_t* __restrict__ nl,
                                           const int32_t* __restrict__ used, int a, int b) {
    const int u = min(__ldg(&used[a]), FOS_S);
    const int4* row = reinterpret_cast<const int4*>(nl + (size_t)a * FOS_S);
    bool m = false;
    for (int q = 0; q < u; q += 4) {
        const int4 v = __ldg(&row[q >> 2]);
        m |= (v.x == b) | ((q + 1 < u) & (v.y == b)) | ((q + 2 < u) & (v.z == b)) |
             ((q + 3 < u) & (v.w == b));
    }
    return m;
}

__device__ __forceinline__ float sur_member(const int32_t* __restrict__ nl,
                                            const int32_t* __restrict__ used, int i, int j) {
    return (sur_in_row(nl, used, i, j) || sur_in_row(nl, used, j, i)) ? 1.f : 0.f;
}

// The 16 raw features of pair (i, j) at normalised distance nd; hi and hj
// are the two particles' histogram rows (SUR_NB ints each), mem and fsum
// the memory features.
__device__ __forceinline__ void sur_features(float ri, float rj, float nd, const int32_t* hi,
                                             const int32_t* hj, float inv_cut_bins, float mem,
                                             float fsum, float* x) {
    x[0] = nd;
    x[1] = fdiv(ri, rj);
    x[2] = nd > 0.f ? fdiv(fsub(ri, rj), fmul(fmul(2.0f, nd), fadd(ri, rj))) : 0.f;
    int bin = (int)fmul(nd, inv_cut_bins);
    bin = bin < SUR_NB - 1 ? bin : SUR_NB - 1;
#pragma unroll
    for (int b = 0; b < SUR_NB; ++b) {
        // the pair itself is in both histograms: leave it out
        const int v = __ldg(&hi[b]) + __ldg(&hj[b]) - (b == bin ? 2 : 0);
        x[3 + b] = (float)v;
    }
    x[3 + SUR_NB] = mem;
    x[4 + SUR_NB] = fsum;
}
static_assert(SUR_NF == SUR_NB + 5, "feature layout: 3 geometric, the bins, 2 memory");

// Training export: one warp per owner i writes its pairs' raw FP32 feature
// rows, labels (j in i's JFA neighbour list) and indices at pstart[i] + slot.
__global__ void __launch_bounds__(256) k_sur_export(int n, const int32_t* __restrict__ pj,
                                                    const float* __restrict__ pnd,
                                                    const int32_t* __restrict__ pstart,
                                                    const float* __restrict__ rad,
                                                    const int32_t* __restrict__ hist, float cutoff,
                                                    int32_t* __restrict__ fi,
                                                    int32_t* __restrict__ fj, float* __restrict__ X,
                                                    float* __restrict__ y,
                                                    const int32_t* __restrict__ nl,
                                                    const int32_t* __restrict__ mnl,
                                                    const int32_t* __restrict__ mused,
                                                    const int32_t* __restrict__ mfsc) {
    const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const int b0 = pstart[i], cnt = pstart[i + 1] - b0;
    const float ri = rad[i];
    const float inv_cut_bins = (float)SUR_NB / cutoff;
    for (int s = lane; s < cnt; s += 32) {
        const int j = pj[(size_t)i * SUR_CAP + s];
        const float nd = pnd[(size_t)i * SUR_CAP + s];
        float x[SUR_NF];
        sur_features(ri, rad[j], nd, hist + (size_t)i * SUR_NB, hist + (size_t)j * SUR_NB,
                     inv_cut_bins, sur_member(mnl, mused, i, j),
                     (float)(__ldg(&mfsc[i]) + __ldg(&mfsc[j])), x);
        const size_t row = (size_t)b0 + s;
        if (X) {
#pragma unroll
            for (int f = 0; f < SUR_NF; ++f) X[row * SUR_NF + f] = x[f];
        }
        if (y) {
            float lab = 0.f;
            for (int q = 0; q < FOS_S; ++q)
                if (nl[(size_t)i * FOS_S + q] == j) lab = 1.f;
            y[row] = lab;
        }
        if (fi) fi[row] = i;
        if (fj) fj[row] = j;
    }
}

// Raw FP32 rows -> standardised BF16 rows (fos_surrogate_forward).
__global__ void k_sur_std(int P, const float* __restrict__ X, const float* __restrict__ norm,
                          uint4* __restrict__ xb) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    unsigned int w[8];
#pragma unroll
    for (int f = 0; f < SUR_NF; f += 2) {
        const float a = (X[(size_t)p * SUR_NF + f] - norm[f]) * norm[SUR_NF + f];
        const float b = (X[(size_t)p * SUR_NF + f + 1] - norm[f + 1]) * norm[SUR_NF + f + 1];
        __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
        w[f / 2] = *reinterpret_cast<unsigned int*>(&v);
    }
    xb[(size_t)p * 2] = make_uint4(w[0], w[1], w[2], w[3]);
    xb[(size_t)p * 2 + 1] = make_uint4(w[4], w[5], w[6], w[7]);
}

// ------------------------------------------------------------ inference
__device__ __forceinline__ unsigned int pack_bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned int*>(&v);
}

// D += A * B, m16n8k16, BF16 inputs, FP32 accumulators.
__device__ __forceinline__ void mma_16816(float* d, unsigned int a0, unsigned int a1,
                                          unsigned int a2, unsigned int a3, unsigned int b0,
                                          unsigned int b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

#define SUR_W2_STRIDE 36  // 32-bit words per W2 row in shared memory (64 BF16 + pad)

// Weights of one block in shared memory, layer-1 B fragments in registers.
struct SurSmem {
    unsigned int w2[SUR_H * SUR_W2_STRIDE];
    float b1[SUR_H], b2[SUR_H], w3[SUR_H], norm[2 * SUR_NF];
};

__device__ __forceinline__ void sur_load_weights(SurSmem& sm, const __nv_bfloat16* wbf,
                                                 const float* params, const float* norm) {
    const unsigned int* w2u = reinterpret_cast<const unsigned int*>(wbf + SUR_H * SUR_NF);
    for (int t = threadIdx.x; t < SUR_H * SUR_H / 2; t += blockDim.x)
        sm.w2[(t / 32) * SUR_W2_STRIDE + (t % 32)] = w2u[t];
    for (int t = threadIdx.x; t < SUR_H; t += blockDim.x) {
        sm.b1[t] = params[SUR_OFF_B1 + t];
        sm.b2[t] = params[SUR_OFF_B2 + t];
        sm.w3[t] = __bfloat162float(wbf[SUR_H * SUR_NF + SUR_H * SUR_H + t]);
    }
    if (norm)
        for (int t = threadIdx.x; t < 2 * SUR_NF; t += blockDim.x) sm.norm[t] = norm[t];
}

// Fragment layout of m16n8k16 (lane = 4 * gid + tg): A holds rows gid and
// gid + 8 at columns 2tg, 2tg+1 (a0, a1) and 2tg+8, 2tg+9 (a2, a3); B holds
// k = 2tg, 2tg+1 (b0) and 2tg+8, 2tg+9 (b1) of column gid; C holds rows gid
// (c0, c1) and gid + 8 (c2, c3) at columns 2tg, 2tg+1.  Returns the logits
// of rows gid (z0) and gid + 8 (z1), summed over the quad.
__device__ __forceinline__ void sur_mlp_tile(const SurSmem& sm, const unsigned int (&bw1)[8][2],
                                             unsigned int a0, unsigned int a1, unsigned int a2,
                                             unsigned int a3, int gid, int tg, float& z0,
                                             float& z1) {
    unsigned int h[4][4];
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
            const int nt = 2 * ks + hf;
            float d[4] = {0.f, 0.f, 0.f, 0.f};
            mma_16816(d, a0, a1, a2, a3, bw1[nt][0], bw1[nt][1]);
            const int col = nt * 8 + 2 * tg;
            const float bb0 = sm.b1[col], bb1 = sm.b1[col + 1];
            h[ks][2 * hf + 0] = pack_bf16x2(fmaxf(d[0] + bb0, 0.f), fmaxf(d[1] + bb1, 0.f));
            h[ks][2 * hf + 1] = pack_bf16x2(fmaxf(d[2] + bb0, 0.f), fmaxf(d[3] + bb1, 0.f));
        }
    }
    z0 = 0.f;
    z1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        const unsigned int* wrow = sm.w2 + (nt * 8 + gid) * SUR_W2_STRIDE;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
            mma_16816(d, h[ks][0], h[ks][1], h[ks][2], h[ks][3], wrow[ks * 8 + tg],
                      wrow[ks * 8 + 4 + tg]);
        const int col = nt * 8 + 2 * tg;
        const float bb0 = sm.b2[col], bb1 = sm.b2[col + 1];
        const float w30 = sm.w3[col], w31 = sm.w3[col + 1];
        z0 += fmaxf(d[0] + bb0, 0.f) * w30 + fmaxf(d[1] + bb1, 0.f) * w31;
        z1 += fmaxf(d[2] + bb0, 0.f) * w30 + fmaxf(d[3] + bb1, 0.f) * w31;
    }
    z0 += __shfl_xor_sync(0xffffffffu, z0, 1);
    z0 += __shfl_xor_sync(0xffffffffu, z0, 2);
    z1 += __shfl_xor_sync(0xffffffffu, z1, 1);
    z1 += __shfl_xor_sync(0xffffffffu, z1, 2);
}

__device__ __forceinline__ void sur_load_bw1(const __nv_bfloat16* wbf, int gid, int tg,
                                             unsigned int (&bw1)[8][2]) {
    const unsigned int* w1u = reinterpret_cast<const unsigned int*>(wbf);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int nrow = nt * 8 + gid;
        bw1[nt][0] = w1u[nrow * 8 + tg];
        bw1[nt][1] = w1u[nrow * 8 + 4 + tg];
    }
}

// Inference on flat standardised BF16 rows (fos_surrogate_forward): one warp
// per 16-row tile, persistent grid.
__global__ void __launch_bounds__(256) k_sur_mlp(int P, const uint4* __restrict__ xb,
                                                 const __nv_bfloat16* __restrict__ wbf,
                                                 const float* __restrict__ params,
                                                 float* __restrict__ prob) {
    __shared__ SurSmem sm;
    sur_load_weights(sm, wbf, params, nullptr);
    __syncthreads();
    const float b3 = params[SUR_OFF_B3];
    const int lane = threadIdx.x & 31, gid = lane >> 2, tg = lane & 3;
    unsigned int bw1[8][2];
    sur_load_bw1(wbf, gid, tg, bw1);
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int tiles = (P + 15) >> 4;
    const unsigned int* xu = reinterpret_cast<const unsigned int*>(xb);
    for (int tile = wid; tile < tiles; tile += warps) {
        const int r0 = tile * 16 + gid, r1 = r0 + 8;
        const bool v0 = r0 < P, v1 = r1 < P;
        const unsigned int a0 = v0 ? xu[(size_t)r0 * 8 + tg] : 0u;
        const unsigned int a1 = v1 ? xu[(size_t)r1 * 8 + tg] : 0u;
        const unsigned int a2 = v0 ? xu[(size_t)r0 * 8 + 4 + tg] : 0u;
        const unsigned int a3 = v1 ? xu[(size_t)r1 * 8 + 4 + tg] : 0u;
        float z0, z1;
        sur_mlp_tile(sm, bw1, a0, a1, a2, a3, gid, tg, z0, z1);
        if (tg < 2) {  // lane tg 0 finishes row gid, lane tg 1 row gid + 8
            const int r = tg == 0 ? r0 : r1;
            if (r < P) prob[r] = 1.0f / (1.0f + expf(-((tg == 0 ? z0 : z1) + b3)));
        }
    }
}

#define SUR_GROUP 4  // owner particles per warp group of the fused inference
#define SUR_XS 12    // 32-bit words per BF16 feature row in shared memory (8 + pad)

// Fused features + MLP over the pair segments of the last pair build.  Each
// warp takes groups of SUR_GROUP consecutive owners, lays their segments end
// to end (warp scan of the counts) and walks them 16 pairs at a time: lane l
// builds half (l >> 4) of the features of row (l & 15) and stores them,
// standardised and rounded to BF16, in the warp's shared-memory tile; the
// tile is then the A operand of the tensor-core layers.  The row-to-pair
// mapping never leaves registers, so the frame path needs no scan and no
// flat pair arrays.  prob (optional) is written at pstart[i] + slot, the
// export order.
__global__ void __launch_bounds__(256) k_sur_mlp_seg(
    int n, const int32_t* __restrict__ pcount, const int32_t* __restrict__ pj,
    const float* __restrict__ pnd, const float* __restrict__ rad, const int32_t* __restrict__ hist,
    float cutoff, const float* __restrict__ norm, const __nv_bfloat16* __restrict__ wbf,
    const float* __restrict__ params, const int32_t* __restrict__ pstart, float* __restrict__ prob,
    unsigned long long* __restrict__ acc, const int32_t* __restrict__ mnl,
    const int32_t* __restrict__ mused, const int32_t* __restrict__ mfsc) {
    __shared__ SurSmem sm;
    __shared__ __align__(16) unsigned int s_x[8][16 * SUR_XS];
    sur_load_weights(sm, wbf, params, norm);
    __syncthreads();
    const float b3 = params[SUR_OFF_B3];
    const int lane = threadIdx.x & 31, gid = lane >> 2, tg = lane & 3;
    const int r = lane & 15, half = lane >> 4;
    unsigned int* xs = s_x[threadIdx.x >> 5];
    unsigned int bw1[8][2];
    sur_load_bw1(wbf, gid, tg, bw1);
    const float inv_cut_bins = (float)SUR_NB / cutoff;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int ngroups = (n + SUR_GROUP - 1) / SUR_GROUP;
    for (int grp = wid; grp < ngroups; grp += warps) {
        const int ib = grp * SUR_GROUP;
        int cnt = 0;
        if (lane < SUR_GROUP && ib + lane < n) cnt = pcount[ib + lane];
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < SUR_GROUP; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int excl = incl - cnt;
        const int total = __shfl_sync(0xffffffffu, incl, SUR_GROUP - 1);
        for (int tb = 0; tb < total; tb += 16) {
            const int t = tb + r;
            int q = 0;
#pragma unroll
            for (int step = SUR_GROUP / 2; step > 0; step >>= 1) {
                const int e = __shfl_sync(0xffffffffu, excl, q + step);
                if (e <= t) q += step;
            }
            const int eq = __shfl_sync(0xffffffffu, excl, q);
            const int i = ib + q, slot = t - eq;
            const bool valid = t < total;
            int j = 0;
            uint4 w = make_uint4(0u, 0u, 0u, 0u);
            if (valid) {
                j = pj[(size_t)i * SUR_CAP + slot];
                const float nd = pnd[(size_t)i * SUR_CAP + slot];
                int bin = (int)fmul(nd, inv_cut_bins);
                bin = bin < SUR_NB - 1 ? bin : SUR_NB - 1;
                const int32_t* hi = hist + (size_t)i * SUR_NB;
                const int32_t* hj = hist + (size_t)j * SUR_NB;
                float x[8];
                if (half == 0) {
                    const float ri = rad[i], rj = rad[j];
                    x[0] = nd;
                    x[1] = fdiv(ri, rj);
                    x[2] = nd > 0.f ? fdiv(fsub(ri, rj), fmul(fmul(2.0f, nd), fadd(ri, rj))) : 0.f;
#pragma unroll
                    for (int b = 0; b < 5; ++b)
                        x[3 + b] = (float)(__ldg(&hi[b]) + __ldg(&hj[b]) - (b == bin ? 2 : 0));
                } else {
#pragma unroll
                    for (int b = 5; b < SUR_NB; ++b)
                        x[b - 5] = (float)(__ldg(&hi[b]) + __ldg(&hj[b]) - (b == bin ? 2 : 0));
                    x[SUR_NB - 5] = sur_member(mnl, mused, i, j);
                    x[SUR_NB - 4] = (float)(__ldg(&mfsc[i]) + __ldg(&mfsc[j]));
                }
                unsigned int pk[4];
#pragma unroll
                for (int k = 0; k < 8; k += 2) {
                    const int f = half * 8 + k;
                    pk[k / 2] = pack_bf16x2((x[k] - sm.norm[f]) * sm.norm[SUR_NF + f],
                                            (x[k + 1] - sm.norm[f + 1]) * sm.norm[SUR_NF + f + 1]);
                }
                w = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            }
            *reinterpret_cast<uint4*>(xs + r * SUR_XS + half * 4) = w;
            __syncwarp();
            const unsigned int a0 = xs[gid * SUR_XS + tg];
            const unsigned int a1 = xs[(gid + 8) * SUR_XS + tg];
            const unsigned int a2 = xs[gid * SUR_XS + 4 + tg];
            const unsigned int a3 = xs[(gid + 8) * SUR_XS + 4 + tg];
            float z0, z1;
            sur_mlp_tile(sm, bw1, a0, a1, a2, a3, gid, tg, z0, z1);
            // the pair of row gid (+8) was built by lane gid (+8)
            const int rr = gid + 8 * (tg & 1);
            const int ir = __shfl_sync(0xffffffffu, i, rr);
            const int jr = __shfl_sync(0xffffffffu, j, rr);
            const int sr = __shfl_sync(0xffffffffu, slot, rr);
            const int vr = __shfl_sync(0xffffffffu, valid ? 1 : 0, rr);
            if (tg < 2 && vr) {
                const float z = (tg == 0 ? z0 : z1) + b3;
                const float pr = 1.0f / (1.0f + expf(-z));
                if (prob) prob[pstart[ir] + sr] = pr;
                const unsigned long long qv = (unsigned long long)(pr * SUR_FIX + 0.5f);
                atomicAdd(&acc[ir], qv);
                atomicAdd(&acc[jr], qv);
            }
            __syncwarp();
        }
    }
}

// ------------------------------------------------ tcgen05 inference (sm_100a)
// The same inference on the 5th-generation tensor cores: a CTA of 128
// threads takes tiles of 128 flat pair rows (row = thread = TMEM lane).  Each
// thread builds its row's 16 features into a shared-memory A tile; one thread
// issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32, M = 128, N = 64) into a
// TMEM accumulator and commits it to an mbarrier; each warp reads its 32 rows
// back with tcgen05.ld, adds the bias, applies ReLU and writes the BF16
// hidden layer as the second A tile (four K = 16 slabs); four more MMAs give
// the second layer, whose read-back feeds the 64 -> 1 output, the sigmoid and
// the per-particle fixed-point sums.  Operands sit in shared memory in the
// canonical K-major layout without swizzle: 8-row x 16-byte core matrices,
// the two K halves of a slab 128 bytes apart (leading byte offset) and
// consecutive 8-row groups 256 bytes apart (stride byte offset).
#define SUR_TC_ROWS 128
#define SUR_TC_COLS 128  // TMEM columns: layer 1 at 0, layer 2 at 64
#define SUR_TC_PAD (24 * 1024)  // dynamic shared-memory padding (residency cap)

struct SurTcSmem {
    alignas(1024) unsigned char a1[SUR_TC_ROWS * 16 * 2];
    alignas(1024) unsigned char a2[4][SUR_TC_ROWS * 16 * 2];
    alignas(1024) unsigned char w1[SUR_H * 16 * 2];
    alignas(1024) unsigned char w2[4][SUR_H * 16 * 2];
    float b1[SUR_H], b2[SUR_H], w3[SUR_H], norm[2 * SUR_NF];
    alignas(8) unsigned long long bar;
    unsigned int tmem;
};

// Byte offset of element (r, k) of a K = 16 slab in the canonical layout.
__device__ __forceinline__ int sur_tc_ofs(int r, int k) {
    return (r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// Shared-memory matrix descriptor of a slab at shared address addr:
// start >> 4, leading byte offset 128 >> 4, stride byte offset 256 >> 4,
// descriptor version 1, no swizzle.
__device__ __forceinline__ unsigned long long sur_tc_desc(unsigned int addr) {
    return (unsigned long long)((addr & 0x3FFFFu) >> 4) | (8ull << 16) | (16ull << 32) |
           (1ull << 46);
}

// Instruction descriptor: FP32 accumulate (bit 4), BF16 A (bit 7) and B
// (bit 10), both K-major, N / 8 = 8 at bit 17, M / 16 = 8 at bit 24.
#define SUR_TC_IDESC 0x08100490u

__device__ __forceinline__ void sur_tc_mma(unsigned int tmem_d, unsigned long long da,
                                           unsigned long long db, unsigned int accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(SUR_TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u),
          "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void sur_tc_commit(unsigned int bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     bar)
                 : "memory");
}

__device__ __forceinline__ bool sur_tc_try_wait(unsigned int bar, unsigned int parity) {
    unsigned int done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0u;
}

// Bounded wait (about 1 s of clock): false, with FOS_E_TIMEOUT recorded, if
// the phase never completed.
__device__ __forceinline__ bool sur_tc_wait(unsigned int bar, unsigned int parity,
                                            int* err) {
    const long long t0 = clock64();
    for (unsigned int it = 1;; ++it) {
        if (sur_tc_try_wait(bar, parity)) return true;
        if ((it & 63u) == 0u && clock64() - t0 > FOS_BAR_CYCLE_LIMIT) {
            atomicCAS(err, 0, (int)FOS_E_TIMEOUT);
            return false;
        }
    }
}

// 64 FP32 columns of this warp's 32 TMEM lanes starting at column col.
__device__ __forceinline__ void sur_tc_ld64(unsigned int taddr, float (&v)[64]) {
    unsigned int r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
        "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
        "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, "
        "[%64];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]),
          "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]),
          "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]),
          "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]),
          "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]),
          "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int c = 0; c < 64; ++c) v[c] = __uint_as_float(r[c]);
}

__global__ void __launch_bounds__(SUR_TC_ROWS) k_sur_mlp_tc(
    int n, const int32_t* __restrict__ pstart, const int32_t* __restrict__ pj,
    const float* __restrict__ pnd, const float* __restrict__ rad, const int32_t* __restrict__ hist,
    float cutoff, const float* __restrict__ norm, const __nv_bfloat16* __restrict__ wbf,
    const float* __restrict__ params, float* __restrict__ prob, unsigned long long* __restrict__ acc,
    const int32_t* __restrict__ mnl, const int32_t* __restrict__ mused,
    const int32_t* __restrict__ mfsc, int* err) {
    __shared__ SurTcSmem sm;
    const int t = threadIdx.x, warp = t >> 5;
    // weights into the canonical layout, biases and standardisation
    for (int e = t; e < SUR_H * 16; e += blockDim.x) {
        const int nrow = e >> 4, k = e & 15;
        *reinterpret_cast<__nv_bfloat16*>(sm.w1 + sur_tc_ofs(nrow, k)) = wbf[e];
    }
    for (int e = t; e < SUR_H * SUR_H; e += blockDim.x) {
        const int nrow = e >> 6, k = e & 63;
        *reinterpret_cast<__nv_bfloat16*>(sm.w2[k >> 4] + sur_tc_ofs(nrow, k & 15)) =
            wbf[SUR_H * SUR_NF + e];
    }
    for (int e = t; e < SUR_H; e += blockDim.x) {
        sm.b1[e] = params[SUR_OFF_B1 + e];
        sm.b2[e] = params[SUR_OFF_B2 + e];
        sm.w3[e] = __bfloat162float(wbf[SUR_H * SUR_NF + SUR_H * SUR_H + e]);
    }
    for (int e = t; e < 2 * SUR_NF; e += blockDim.x) sm.norm[e] = norm[e];
    const unsigned int bar = (unsigned int)__cvta_generic_to_shared(&sm.bar);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (unsigned int)__cvta_generic_to_shared(&sm.tmem)),
                     "r"(SUR_TC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned int tmem = sm.tmem;
    const unsigned int lane_base = (unsigned int)(warp * 32) << 16;
    const unsigned int a1 = (unsigned int)__cvta_generic_to_shared(sm.a1);
    const unsigned int w1 = (unsigned int)__cvta_generic_to_shared(sm.w1);
    const float inv_cut_bins = (float)SUR_NB / cutoff;
    const float b3 = params[SUR_OFF_B3];
    const int P = pstart[n];
    const int tiles = (P + SUR_TC_ROWS - 1) / SUR_TC_ROWS;
    unsigned int phase = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        // (1) this thread's row: owner i by binary search over pstart
        const int g = tile * SUR_TC_ROWS + t;
        const bool valid = g < P;
        int i = 0, j = 0;
        uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
        if (valid) {
            int a = 0, b = n;  // largest a with pstart[a] <= g
            while (b - a > 1) {
                const int m = (a + b) >> 1;
                if (__ldg(&pstart[m]) <= g) a = m;
                else b = m;
            }
            i = a;
            const int slot = g - __ldg(&pstart[i]);
            j = pj[(size_t)i * SUR_CAP + slot];
            const float nd = pnd[(size_t)i * SUR_CAP + slot];
            float x[SUR_NF];
            sur_features(rad[i], rad[j], nd, hist + (size_t)i * SUR_NB, hist + (size_t)j * SUR_NB,
                         inv_cut_bins, sur_member(mnl, mused, i, j),
                         (float)(__ldg(&mfsc[i]) + __ldg(&mfsc[j])), x);
            unsigned int pk[8];
#pragma unroll
            for (int f = 0; f < SUR_NF; f += 2)
                pk[f / 2] = pack_bf16x2((x[f] - sm.norm[f]) * sm.norm[SUR_NF + f],
                                        (x[f + 1] - sm.norm[f + 1]) * sm.norm[SUR_NF + f + 1]);
            lo = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            hi = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
        *reinterpret_cast<uint4*>(sm.a1 + sur_tc_ofs(t, 0)) = lo;
        *reinterpret_cast<uint4*>(sm.a1 + sur_tc_ofs(t, 8)) = hi;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // (2) layer 1: D[0, 64) = A1 (128 x 16) . W1^T
        if (t == 0) {
            sur_tc_mma(tmem, sur_tc_desc(a1), sur_tc_desc(w1), 0u);
            sur_tc_commit(bar);
        }
        // the block agrees on the outcome, so every thread takes the same path
        if (!__syncthreads_and(sur_tc_wait(bar, phase, err))) {
            ok = false;
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // (3) bias, ReLU, BF16 -> the second A tile (four K = 16 slabs)
        {
            float h[64];
            sur_tc_ld64(tmem + lane_base, h);
#pragma unroll
            for (int sl = 0; sl < 4; ++sl) {
                unsigned int pk[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int c = sl * 16 + 2 * q;
                    pk[q] = pack_bf16x2(fmaxf(h[c] + sm.b1[c], 0.f),
                                        fmaxf(h[c + 1] + sm.b1[c + 1], 0.f));
                }
                *reinterpret_cast<uint4*>(sm.a2[sl] + sur_tc_ofs(t, 0)) =
                    make_uint4(pk[0], pk[1], pk[2], pk[3]);
                *reinterpret_cast<uint4*>(sm.a2[sl] + sur_tc_ofs(t, 8)) =
                    make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // (4) layer 2: D[64, 128) = A2 (128 x 64) . W2^T, four K slabs
        if (t == 0) {
#pragma unroll
            for (int sl = 0; sl < 4; ++sl)
                sur_tc_mma(tmem + 64, sur_tc_desc((unsigned int)__cvta_generic_to_shared(sm.a2[sl])),
                           sur_tc_desc((unsigned int)__cvta_generic_to_shared(sm.w2[sl])),
                           sl > 0 ? 1u : 0u);
            sur_tc_commit(bar);
        }
        if (!__syncthreads_and(sur_tc_wait(bar, phase, err))) {
            ok = false;
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // (5) bias, ReLU, the 64 -> 1 output, sigmoid, fixed-point sums
        {
            float h[64];
            sur_tc_ld64(tmem + lane_base + 64, h);
            float z = 0.f;
#pragma unroll
            for (int c = 0; c < 64; ++c) z += fmaxf(h[c] + sm.b2[c], 0.f) * sm.w3[c];
            if (valid) {
                const float pr = 1.0f / (1.0f + expf(-(z + b3)));
                if (prob) prob[g] = pr;
                const unsigned long long qv = (unsigned long long)(pr * SUR_FIX + 0.5f);
                atomicAdd(&acc[i], qv);
                atomicAdd(&acc[j], qv);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    // every MMA this CTA issued has completed (waited on above); free TMEM
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(SUR_TC_COLS)
                     : "memory");
}

__global__ void k_sur_fsc(int n, const unsigned long long* __restrict__ acc,
                          float* __restrict__ raw, float* __restrict__ fs,
                          int32_t* __restrict__ fsi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = (float)((double)acc[i] * (1.0 / 1048576.0));
    raw[i] = v;
    if (fs) fs[i] = v;
    if (fsi) fsi[i] = (int)rintf(v);
}

// The FSC the controller sees: absolute f = s, or anchored
// f = max(0, base + s - anchor) once an anchor exists.
__global__ void k_sur_combine(int n, int mode, const float* __restrict__ raw,
                              const int32_t* __restrict__ base, const float* __restrict__ anchor,
                              const int* __restrict__ anchor_valid, float* __restrict__ fs,
                              int32_t* __restrict__ fsi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = raw[i];
    if (mode == FOS_SUR_ANCHORED && *anchor_valid)
        v = fmaxf(0.0f, fadd((float)base[i], fsub(v, anchor[i])));
    fs[i] = v;
    fsi[i] = (int)rintf(v);
}

// update_fsc_ema's rule (jfa.py:765-785) fed with the surrogate's float FSC.
__global__ void k_sur_ema(int n, const float* __restrict__ fs, float* ema, float alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float f = fs[i];
    float em = ema[i];
    if (em == 0.0f && f > 0.0f) em = f;
    else em = fadd(fmul(alpha, f), fmul(fsub(1.0f, alpha), em));
    ema[i] = em;
}

// Judge counters (surrogate f vs JFA fsc, previous vs current JFA fsc), then
// the anchor moves to this frame's model estimate.
__global__ void k_sur_judge(int n, const float* __restrict__ fs, const int32_t* __restrict__ fsc,
                            const int32_t* __restrict__ prev, const float* __restrict__ raw,
                            float* __restrict__ anchor, int* anchor_valid,
                            unsigned long long* cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) anchor[i] = raw[i];
    if (i == 0) *anchor_valid = 1;
    int ex = 0, w1 = 0, sx = 0, sw = 0;
    unsigned long long ae = 0, se = 0;
    if (i < n) {
        const int f = fsc[i];
        const float s = fs[i];
        const int d = (int)rintf(s) - f;
        ex = d == 0;
        w1 = d >= -1 && d <= 1;
        ae = (unsigned long long)(fabsf(s - (float)f) * SUR_FIX + 0.5f);
        const int ds = prev[i] - f;
        sx = ds == 0;
        sw = ds >= -1 && ds <= 1;
        se = (unsigned long long)(ds < 0 ? -ds : ds);
    }
    const int e = __syncthreads_count(ex), w = __syncthreads_count(w1);
    const int e2 = __syncthreads_count(sx), w2 = __syncthreads_count(sw);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ae += __shfl_xor_sync(0xffffffffu, ae, o);
        se += __shfl_xor_sync(0xffffffffu, se, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (ae) atomicAdd(&cnt[SC_ABS_ERR], ae);
        if (se) atomicAdd(&cnt[SC_STALE_ABS_ERR], se);
    }
    if (threadIdx.x == 0) {
        const int live = min((int)blockDim.x, n - (int)(blockIdx.x * blockDim.x));
        atomicAdd(&cnt[SC_JUDGED], (unsigned long long)live);
        if (e) atomicAdd(&cnt[SC_EXACT], (unsigned long long)e);
        if (w) atomicAdd(&cnt[SC_WITHIN1], (unsigned long long)w);
        if (e2) atomicAdd(&cnt[SC_STALE_EXACT], (unsigned long long)e2);
        if (w2) atomicAdd(&cnt[SC_STALE_WITHIN1], (unsigned long long)w2);
    }
}

__global__ void k_sur_judge_reset(unsigned long long* cnt) {
    if (threadIdx.x >= SC_JUDGED && threadIdx.x < SC_N) cnt[threadIdx.x] = 0ull;
}

// ------------------------------------------------------------ training
// Shared-memory layout of k_sur_train (floats); rows padded against bank
// conflicts.
#define TR_ROWS 64
#define TR_S1 17  // W1 / X row stride
#define TR_S2 65  // W2 / H row stride
#define TR_OFF_W1 0
#define TR_OFF_W2 (TR_OFF_W1 + SUR_H * TR_S1)
#define TR_OFF_B1 (TR_OFF_W2 + SUR_H * TR_S2)
#define TR_OFF_B2 (TR_OFF_B1 + SUR_H)
#define TR_OFF_W3 (TR_OFF_B2 + SUR_H)
#define TR_OFF_X (TR_OFF_W3 + SUR_H)
#define TR_OFF_H1 (TR_OFF_X + TR_ROWS * TR_S1)
#define TR_OFF_H2 (TR_OFF_H1 + TR_ROWS * TR_S2)
#define TR_OFF_DZ (TR_OFF_H2 + TR_ROWS * TR_S2)
#define TR_OFF_NORM (TR_OFF_DZ + TR_ROWS)
#define TR_OFF_LOSS (TR_OFF_NORM + 2 * SUR_NF)
#define TR_THREADS 256
#define TR_SMEM_FLOATS (TR_OFF_LOSS + TR_THREADS / 32)

// Forward + backward of the mean BCE over `batch` rows, 64-row tiles spread
// over the blocks in a fixed order; each block writes its gradient sums (and
// loss sum) to part[blockIdx.x][NPARAM + 1].
__global__ void __launch_bounds__(TR_THREADS) k_sur_train(
    const float* __restrict__ X, const float* __restrict__ y, const int32_t* __restrict__ rows,
    int batch, const float* __restrict__ params, const float* __restrict__ norm,
    float* __restrict__ part) {
    extern __shared__ float smf[];
    float* sW1 = smf + TR_OFF_W1;
    float* sW2 = smf + TR_OFF_W2;
    float* sb1 = smf + TR_OFF_B1;
    float* sb2 = smf + TR_OFF_B2;
    float* sw3 = smf + TR_OFF_W3;
    float* sX = smf + TR_OFF_X;
    float* sH1 = smf + TR_OFF_H1;
    float* sH2 = smf + TR_OFF_H2;
    float* sdz = smf + TR_OFF_DZ;
    float* snorm = smf + TR_OFF_NORM;
    float* sloss = smf + TR_OFF_LOSS;
    const int t = threadIdx.x;
    for (int e = t; e < SUR_H * SUR_NF; e += TR_THREADS)
        sW1[(e / SUR_NF) * TR_S1 + e % SUR_NF] = params[SUR_OFF_W1 + e];
    for (int e = t; e < SUR_H * SUR_H; e += TR_THREADS)
        sW2[(e / SUR_H) * TR_S2 + e % SUR_H] = params[SUR_OFF_W2 + e];
    if (t < SUR_H) {
        sb1[t] = params[SUR_OFF_B1 + t];
        sb2[t] = params[SUR_OFF_B2 + t];
        sw3[t] = params[SUR_OFF_W3 + t];
    }
    if (t < 2 * SUR_NF) snorm[t] = norm[t];
    const float b3 = params[SUR_OFF_B3];
    const float invB = 1.0f / (float)batch;
    // gradient accumulators
    float gW2[16];  // dW2[c2][q2 + 4u], c2 = t >> 2, q2 = t & 3
    float gW1[4];   // dW1[c2][q2 + 4u]
#pragma unroll
    for (int u = 0; u < 16; ++u) gW2[u] = 0.f;
#pragma unroll
    for (int u = 0; u < 4; ++u) gW1[u] = 0.f;
    // t < 64: db2[t]; 64 <= t < 128: db1[t - 64]; 128 <= t < 192: dw3[t - 128]; t == 192: db3
    float gsp = 0.f;
    float lsum = 0.f;                   // lane 0 of each warp: loss partial
    const int c = t & 63, rg = t >> 6;  // (column, 16-row group) mapping
    const int c2 = t >> 2, q2 = t & 3;  // outer-product mapping
    const int warp = t >> 5, lane = t & 31;
    __syncthreads();
    const int ntiles = (batch + TR_ROWS - 1) / TR_ROWS;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int rbase = tile * TR_ROWS;
        // (1) standardised inputs
        for (int e = t; e < TR_ROWS * SUR_NF; e += TR_THREADS) {
            const int r = e / SUR_NF, f = e % SUR_NF;
            float v = 0.f;
            if (rbase + r < batch) {
                const int row = rows[rbase + r];
                v = (X[(size_t)row * SUR_NF + f] - snorm[f]) * snorm[SUR_NF + f];
            }
            sX[r * TR_S1 + f] = v;
        }
        __syncthreads();
        // (2) H1 = relu(X W1^T + b1)
        {
            float w[SUR_NF];
#pragma unroll
            for (int f = 0; f < SUR_NF; ++f) w[f] = sW1[c * TR_S1 + f];
#pragma unroll 4
            for (int rr = 0; rr < 16; ++rr) {
                const int r = rg * 16 + rr;
                float a = sb1[c];
#pragma unroll
                for (int f = 0; f < SUR_NF; ++f) a = fmaf(sX[r * TR_S1 + f], w[f], a);
                sH1[r * TR_S2 + c] = fmaxf(a, 0.f);
            }
        }
        __syncthreads();
        // (3) H2 = relu(H1 W2^T + b2)
        {
            float a[16];
#pragma unroll
            for (int rr = 0; rr < 16; ++rr) a[rr] = sb2[c];
            for (int k = 0; k < SUR_H; ++k) {
                const float w = sW2[c * TR_S2 + k];
#pragma unroll
                for (int rr = 0; rr < 16; ++rr) a[rr] = fmaf(sH1[(rg * 16 + rr) * TR_S2 + k], w, a[rr]);
            }
#pragma unroll
            for (int rr = 0; rr < 16; ++rr) sH2[(rg * 16 + rr) * TR_S2 + c] = fmaxf(a[rr], 0.f);
        }
        __syncthreads();
        // (4) logits, loss and dL/dz (one warp per 8 rows)
        for (int rr = 0; rr < 8; ++rr) {
            const int r = warp * 8 + rr;
            float v = sH2[r * TR_S2 + lane] * sw3[lane] + sH2[r * TR_S2 + lane + 32] * sw3[lane + 32];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) {
                float dz = 0.f;
                if (rbase + r < batch) {
                    const float z = v + b3;
                    const float yy = y[rows[rbase + r]];
                    const float p = 1.0f / (1.0f + expf(-z));
                    dz = (p - yy) * invB;
                    lsum += fmaxf(z, 0.f) - z * yy + log1pf(expf(-fabsf(z)));
                }
                sdz[r] = dz;
            }
        }
        __syncthreads();
        // (5) output layer gradients, then dH2 in place of H2
        if (t >= 128 && t < 192) {
            const int cc = t - 128;
            float g = 0.f;
            for (int r = 0; r < TR_ROWS; ++r) g = fmaf(sdz[r], sH2[r * TR_S2 + cc], g);
            gsp += g;
        } else if (t == 192) {
            float g = 0.f;
            for (int r = 0; r < TR_ROWS; ++r) g += sdz[r];
            gsp += g;
        }
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < 16; ++rr) {
            const int r = rg * 16 + rr;
            const float hv = sH2[r * TR_S2 + c];
            sH2[r * TR_S2 + c] = hv > 0.f ? sdz[r] * sw3[c] : 0.f;
        }
        __syncthreads();
        // (6) dW2 += dH2^T H1, db2 += colsum dH2
        for (int r = 0; r < TR_ROWS; ++r) {
            const float d = sH2[r * TR_S2 + c2];
#pragma unroll
            for (int u = 0; u < 16; ++u) gW2[u] = fmaf(d, sH1[r * TR_S2 + q2 + 4 * u], gW2[u]);
        }
        if (t < 64) {
            float g = 0.f;
            for (int r = 0; r < TR_ROWS; ++r) g += sH2[r * TR_S2 + t];
            gsp += g;
        }
        // (7) dH1 = (dH2 W2) * (H1 > 0), into registers first
        float dh[16];
#pragma unroll
        for (int rr = 0; rr < 16; ++rr) dh[rr] = 0.f;
        for (int k = 0; k < SUR_H; ++k) {
            const float w = sW2[k * TR_S2 + c];
#pragma unroll
            for (int rr = 0; rr < 16; ++rr) dh[rr] = fmaf(sH2[(rg * 16 + rr) * TR_S2 + k], w, dh[rr]);
        }
#pragma unroll
        for (int rr = 0; rr < 16; ++rr)
            if (!(sH1[(rg * 16 + rr) * TR_S2 + c] > 0.f)) dh[rr] = 0.f;
        __syncthreads();
#pragma unroll
        for (int rr = 0; rr < 16; ++rr) sH1[(rg * 16 + rr) * TR_S2 + c] = dh[rr];
        __syncthreads();
        // (8) dW1 += dH1^T X, db1 += colsum dH1
        for (int r = 0; r < TR_ROWS; ++r) {
            const float d = sH1[r * TR_S2 + c2];
#pragma unroll
            for (int u = 0; u < 4; ++u) gW1[u] = fmaf(d, sX[r * TR_S1 + q2 + 4 * u], gW1[u]);
        }
        if (t >= 64 && t < 128) {
            float g = 0.f;
            for (int r = 0; r < TR_ROWS; ++r) g += sH1[r * TR_S2 + (t - 64)];
            gsp += g;
        }
        __syncthreads();
    }
    // per-block results
    float* out = part + (size_t)blockIdx.x * (SUR_NPARAM + 1);
#pragma unroll
    for (int u = 0; u < 16; ++u) out[SUR_OFF_W2 + c2 * SUR_H + q2 + 4 * u] = gW2[u];
#pragma unroll
    for (int u = 0; u < 4; ++u) out[SUR_OFF_W1 + c2 * SUR_NF + q2 + 4 * u] = gW1[u];
    if (t < 64) out[SUR_OFF_B2 + t] = gsp;
    else if (t < 128) out[SUR_OFF_B1 + (t - 64)] = gsp;
    else if (t < 192) out[SUR_OFF_W3 + (t - 128)] = gsp;
    else if (t == 192) out[SUR_OFF_B3] = gsp;
    if (lane == 0) sloss[warp] = lsum;
    __syncthreads();
    if (t == 0) {
        float l = 0.f;
        for (int w = 0; w < TR_THREADS / 32; ++w) l += sloss[w];
        out[SUR_NPARAM] = l * invB;
    }
}

// Sums the per-block gradients in block order; with lr > 0 applies Adam and
// refreshes the BF16 copies.
__global__ void k_sur_adam(int nblk, const float* __restrict__ part, float* params, float* am,
                           float* av, __nv_bfloat16* wbf, float lr, float bc1, float bc2,
                           float* grad_out, float* loss_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > SUR_NPARAM) return;
    float g = 0.f;
    for (int b = 0; b < nblk; ++b) g += part[(size_t)b * (SUR_NPARAM + 1) + p];
    if (p == SUR_NPARAM) {
        if (loss_out) *loss_out = g;
        return;
    }
    if (grad_out) grad_out[p] = g;
    if (lr > 0.f) {
        const float m = 0.9f * am[p] + 0.1f * g;
        const float v = 0.999f * av[p] + 0.001f * g * g;
        am[p] = m;
        av[p] = v;
        const float w = params[p] - lr * (m / bc1) / (sqrtf(v / bc2) + 1e-8f);
        params[p] = w;
        if (p < SUR_OFF_B1)
            wbf[p] = __float2bfloat16_rn(w);
        else if (p >= SUR_OFF_W2 && p < SUR_OFF_B2)
            wbf[SUR_H * SUR_NF + (p - SUR_OFF_W2)] = __float2bfloat16_rn(w);
        else if (p >= SUR_OFF_W3 && p < SUR_OFF_B3)
            wbf[SUR_H * SUR_NF + SUR_H * SUR_H + (p - SUR_OFF_W3)] = __float2bfloat16_rn(w);
    }
}

// ------------------------------------------------------------ host: model
static int sur_refresh_bf16(FosSurrogate* m, const float* hparams) {
    __nv_bfloat16 hb[SUR_H * SUR_NF + SUR_H * SUR_H + SUR_H];
    for (int e = 0; e < SUR_H * SUR_NF; ++e) hb[e] = __float2bfloat16_rn(hparams[SUR_OFF_W1 + e]);
    for (int e = 0; e < SUR_H * SUR_H; ++e)
        hb[SUR_H * SUR_NF + e] = __float2bfloat16_rn(hparams[SUR_OFF_W2 + e]);
    for (int e = 0; e < SUR_H; ++e)
        hb[SUR_H * SUR_NF + SUR_H * SUR_H + e] = __float2bfloat16_rn(hparams[SUR_OFF_W3 + e]);
    FOS_CUDA(cudaMemcpy(m->wbf, hb, sizeof(hb), cudaMemcpyHostToDevice));
    return FOS_OK;
}

extern "C" int fos_surrogate_destroy(FosSurrogate* m) {
    if (!m) return FOS_OK;
    cudaSetDevice(m->device);
    void* ptrs[] = {m->params, m->adam_m, m->adam_v, m->part, m->norm, m->wbf, m->xb};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    delete m;
    return FOS_OK;
}

static int sur_create_impl(FosSurrogate* m) {
    FOS_CUDA(cudaSetDevice(m->device));
    int sms = 0;
    FOS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device));
    m->num_sms = sms;
    m->nblk = 2 * sms;
    struct A {
        void** p;
        size_t bytes;
    } allocs[] = {
        {(void**)&m->params, SUR_NPARAM * 4},
        {(void**)&m->adam_m, SUR_NPARAM * 4},
        {(void**)&m->adam_v, SUR_NPARAM * 4},
        {(void**)&m->part, (size_t)m->nblk * (SUR_NPARAM + 1) * 4},
        {(void**)&m->norm, 2 * SUR_NF * 4},
        {(void**)&m->wbf, (SUR_H * SUR_NF + SUR_H * SUR_H + SUR_H) * 2},
    };
    for (auto& a : allocs) {
        FOS_CUDA(cudaMalloc(a.p, a.bytes));
        FOS_CUDA(cudaMemset(*a.p, 0, a.bytes));
    }
    float norm[2 * SUR_NF];
    for (int f = 0; f < SUR_NF; ++f) {
        m->host_mu[f] = 0.f;
        m->host_sd[f] = 1.f;
        norm[f] = 0.f;
        norm[SUR_NF + f] = 1.f;
    }
    FOS_CUDA(cudaMemcpy(m->norm, norm, sizeof(norm), cudaMemcpyHostToDevice));
    FOS_CUDA(cudaFuncSetAttribute(k_sur_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TR_SMEM_FLOATS * 4));
    return FOS_OK;
}

extern "C" int fos_surrogate_create(int device, float cutoff, FosSurrogate** out) {
    FOS_REQUIRE(out != nullptr, FOS_E_ARG, "out is NULL");
    *out = nullptr;
    FOS_REQUIRE(cutoff > 0.f && cutoff < 64.f, FOS_E_ARG, "cutoff must be in (0, 64)");
    FosSurrogate* m = new FosSurrogate();
    m->device = device;
    m->cutoff = cutoff;
    int rc = sur_create_impl(m);
    if (rc) {
        fos_surrogate_destroy(m);
        return rc;
    }
    *out = m;
    return FOS_OK;
}

extern "C" float fos_surrogate_cutoff(const FosSurrogate* m) { return m ? m->cutoff : 0.f; }

extern "C" int fos_surrogate_set_weights(FosSurrogate* m, const float* params, const float* mu,
                                         const float* sd) {
    FOS_REQUIRE(m && params && mu && sd, FOS_E_ARG, "NULL argument");
    for (int f = 0; f < SUR_NF; ++f)
        FOS_REQUIRE(sd[f] > 0.f && isfinite(sd[f]) && isfinite(mu[f]), FOS_E_ARG,
                    "sd must be finite and > 0, mu finite");
    for (int p = 0; p < SUR_NPARAM; ++p)
        FOS_REQUIRE(isfinite(params[p]), FOS_E_ARG, "non-finite parameter");
    FOS_CUDA(cudaSetDevice(m->device));
    float norm[2 * SUR_NF];
    for (int f = 0; f < SUR_NF; ++f) {
        m->host_mu[f] = mu[f];
        m->host_sd[f] = sd[f];
        norm[f] = mu[f];
        norm[SUR_NF + f] = 1.0f / sd[f];
    }
    FOS_CUDA(cudaMemcpy(m->params, params, SUR_NPARAM * 4, cudaMemcpyHostToDevice));
    FOS_CUDA(cudaMemcpy(m->norm, norm, sizeof(norm), cudaMemcpyHostToDevice));
    FOS_CUDA(cudaMemset(m->adam_m, 0, SUR_NPARAM * 4));
    FOS_CUDA(cudaMemset(m->adam_v, 0, SUR_NPARAM * 4));
    m->step = 0;
    return sur_refresh_bf16(m, params);
}

extern "C" int fos_surrogate_get_weights(FosSurrogate* m, float* params, float* mu, float* sd) {
    FOS_REQUIRE(m != nullptr, FOS_E_ARG, "model is NULL");
    FOS_CUDA(cudaSetDevice(m->device));
    if (params) FOS_CUDA(cudaMemcpy(params, m->params, SUR_NPARAM * 4, cudaMemcpyDeviceToHost));
    for (int f = 0; f < SUR_NF; ++f) {
        if (mu) mu[f] = m->host_mu[f];
        if (sd) sd[f] = m->host_sd[f];
    }
    return FOS_OK;
}

static int sur_backward(FosSurrogate* m, const float* X, const float* y, const int32_t* rows,
                        int batch, float lr, float* grad, float* loss, cudaStream_t s) {
    FOS_REQUIRE(m && X && y && rows, FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(batch >= 1, FOS_E_ARG, "batch must be >= 1");
    FOS_REQUIRE(lr >= 0.f && isfinite(lr), FOS_E_ARG, "lr must be finite and >= 0");
    const int ntiles = (batch + TR_ROWS - 1) / TR_ROWS;
    const int nblk = ntiles < m->nblk ? ntiles : m->nblk;
    k_sur_train<<<nblk, TR_THREADS, TR_SMEM_FLOATS * 4, s>>>(X, y, rows, batch, m->params,
                                                             m->norm, m->part);
    FOS_CUDA(cudaPeekAtLastError());
    float bc1 = 1.f, bc2 = 1.f;
    if (lr > 0.f) {
        m->step += 1;
        bc1 = (float)(1.0 - pow(0.9, (double)m->step));
        bc2 = (float)(1.0 - pow(0.999, (double)m->step));
    }
    k_sur_adam<<<fos_blocks(SUR_NPARAM + 1, 256), 256, 0, s>>>(nblk, m->part, m->params, m->adam_m,
                                                               m->adam_v, m->wbf, lr, bc1, bc2,
                                                               grad, loss);
    FOS_CUDA(cudaPeekAtLastError());
    return FOS_OK;
}

extern "C" int fos_surrogate_train_step(FosSurrogate* m, const float* X, const float* y,
                                        const int32_t* rows, int batch, float lr, float* loss,
                                        fos_stream_t s) {
    FOS_REQUIRE(lr > 0.f, FOS_E_ARG, "lr must be > 0");
    return sur_backward(m, X, y, rows, batch, lr, nullptr, loss, (cudaStream_t)s);
}

extern "C" int fos_surrogate_gradient(FosSurrogate* m, const float* X, const float* y,
                                      const int32_t* rows, int batch, float* grad, float* loss,
                                      fos_stream_t s) {
    FOS_REQUIRE(grad != nullptr, FOS_E_ARG, "grad is NULL");
    return sur_backward(m, X, y, rows, batch, 0.f, grad, loss, (cudaStream_t)s);
}

static int sur_persistent_blocks(int num_sms, long long warps_needed) {
    long long blocks = (warps_needed + 7) / 8;
    const long long cap = (long long)num_sms * 4;
    if (blocks > cap) blocks = cap;
    return (int)(blocks < 1 ? 1 : blocks);
}

extern "C" int fos_surrogate_forward(FosSurrogate* m, const float* X, int P, float* prob,
                                     fos_stream_t s) {
    FOS_REQUIRE(m && X && prob, FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(P >= 0, FOS_E_ARG, "P must be >= 0");
    if (P == 0) return FOS_OK;
    FOS_CUDA(cudaSetDevice(m->device));
    if ((size_t)P > m->xb_rows) {
        if (m->xb) cudaFree(m->xb);
        m->xb = nullptr;
        m->xb_rows = 0;
        FOS_CUDA(cudaMalloc(&m->xb, (size_t)P * SUR_NF * 2));
        m->xb_rows = (size_t)P;
    }
    k_sur_std<<<fos_blocks(P, 256), 256, 0, s>>>(P, X, m->norm, (uint4*)m->xb);
    FOS_CUDA(cudaPeekAtLastError());
    k_sur_mlp<<<sur_persistent_blocks(m->num_sms, (P + 15) / 16), 256, 0, s>>>(
        P, (const uint4*)m->xb, m->wbf, m->params, prob);
    FOS_CUDA(cudaPeekAtLastError());
    return FOS_OK;
}

// ------------------------------------------------------------ host: context
void fos_sur_free(FosCtx* c) {
    FosSurBufs* b = c->sur;
    if (!b) return;
    void* ptrs[] = {b->pj,   b->pnd,  b->pcount, b->pstart, b->hist,         b->acc,
                    b->fscf, b->fsci, b->prev,   b->raw,    b->anchor,       b->anchor_valid,
                    b->cnt};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    delete b;
    c->sur = nullptr;
}

static int sur_bufs_alloc(FosCtx* c, FosSurBufs* b) {
    const size_t n = (size_t)c->max_n, pc = n * SUR_CAP;
    struct A {
        void** p;
        size_t bytes;
    } allocs[] = {
        {(void**)&b->pj, pc * 4},           {(void**)&b->pnd, pc * 4},
        {(void**)&b->pcount, (n + 1) * 4},  {(void**)&b->pstart, (n + 1) * 4},
        {(void**)&b->hist, n * SUR_NB * 4}, {(void**)&b->acc, n * 8},
        {(void**)&b->fscf, n * 4},          {(void**)&b->fsci, n * 4},
        {(void**)&b->prev, n * 4},          {(void**)&b->raw, n * 4},
        {(void**)&b->anchor, n * 4},        {(void**)&b->anchor_valid, 16},
        {(void**)&b->cnt, SC_N * 8},
    };
    for (auto& a : allocs) {
        FOS_CUDA(cudaMalloc(a.p, a.bytes));
        FOS_CUDA(cudaMemset(*a.p, 0, a.bytes));
    }
    return FOS_OK;
}

// Allocates the context's surrogate buffers on first use (never inside a
// stream capture: the frame driver calls this before capturing).
int fos_sur_prepare(FosCtx* c) {
    if (c->sur) return FOS_OK;
    FOS_CUDA(cudaSetDevice(c->device));
    c->sur = new FosSurBufs();
    int rc = sur_bufs_alloc(c, c->sur);
    if (rc) fos_sur_free(c);
    return rc;
}

int fos_grid_gather_sorted(FosCtx* c, const int32_t* idx, const float* pos, const float* rad,
                           int n, cudaStream_t s);

static int sur_pairs_impl(FosCtx* c, const FosSurrogate* m, const float* pos, const float* rad,
                          int n, float r_max, const int32_t* cs, const int32_t* cc,
                          const int32_t* ci, cudaStream_t s) {
    int rc = fos_sur_prepare(c);
    if (rc) return rc;
    FosSurBufs* b = c->sur;
    rc = fos_grid_gather_sorted(c, ci, pos, rad, n, s);
    if (rc) return rc;
    FOS_CUDA(cudaMemsetAsync(b->cnt + SC_OVERFLOW, 0, 8, s));
    GridGeom g{c->G, c->L, c->invL, c->halfL};
    k_sur_pairs<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(c->sorted, ci, n, g, cs, cc, m->cutoff,
                                                          r_max, b->pj, b->pnd, b->pcount, b->hist,
                                                          b->cnt);
    FOS_LAUNCHED(c);
    b->n = n;
    b->cutoff = m->cutoff;
    return FOS_OK;
}

static int sur_scan(FosCtx* c, cudaStream_t s);

static int sur_predict_impl(FosCtx* c, const FosSurrogate* m, const float* rad, float* fsc_float,
                            int32_t* fsc_int, float* pair_prob, cudaStream_t s) {
    FosSurBufs* b = c->sur;
    const int n = b->n;
    FOS_CUDA(cudaMemsetAsync(b->acc, 0, (size_t)n * 8, s));
    if (c->sur_tc) {
        // tcgen05 tiles over the flat rows: pstart and the row count first
        int rc = sur_scan(c, s);
        if (rc) return rc;
        static bool attr = false;
        if (!attr) {
            FOS_CUDA(cudaFuncSetAttribute(k_sur_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          SUR_TC_PAD));
            attr = true;
        }
        // the padding keeps at most four CTAs (4 x 128 TMEM columns) on an SM
        k_sur_mlp_tc<<<c->num_sms * 4, SUR_TC_ROWS, SUR_TC_PAD, s>>>(
            n, b->pstart, b->pj, b->pnd, rad, b->hist, m->cutoff, m->norm, m->wbf, m->params,
            pair_prob, b->acc, c->nl, c->used, c->fsc, &c->ds->error);
        FOS_LAUNCHED(c);
        k_sur_fsc<<<fos_blocks(n, 256), 256, 0, s>>>(n, b->acc, b->raw, fsc_float, fsc_int);
        FOS_LAUNCHED(c);
        return FOS_OK;
    }
    const long long groups = (n + SUR_GROUP - 1) / SUR_GROUP;
    k_sur_mlp_seg<<<sur_persistent_blocks(c->num_sms, groups), 256, 0, s>>>(
        n, b->pcount, b->pj, b->pnd, rad, b->hist, m->cutoff, m->norm, m->wbf, m->params,
        b->pstart, pair_prob, b->acc, c->nl, c->used, c->fsc);
    FOS_LAUNCHED(c);
    k_sur_fsc<<<fos_blocks(n, 256), 256, 0, s>>>(n, b->acc, b->raw, fsc_float, fsc_int);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// pstart (and P = pstart[n]) of the last pair build.
static int sur_scan(FosCtx* c, cudaStream_t s) {
    FosSurBufs* b = c->sur;
    return fos_scan_exclusive(c, b->pcount, b->pstart, b->n, true, s);
}

extern "C" int fos_surrogate_pairs(FosCtx* c, const FosSurrogate* m, const float* pos,
                                   const float* rad, int n, float r_max, const int32_t* cs,
                                   const int32_t* cc, const int32_t* ci, fos_stream_t s) {
    FOS_REQUIRE(c && m && pos && rad && cs && cc && ci, FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(n >= 1 && n <= c->max_n, FOS_E_CAPACITY, "n outside [1, max_n]");
    FOS_REQUIRE(r_max > 0.f && isfinite(r_max), FOS_E_ARG, "r_max must be finite and > 0");
    FOS_REQUIRE(m->device == c->device, FOS_E_ARG, "model and context on different devices");
    return sur_pairs_impl(c, m, pos, rad, n, r_max, cs, cc, ci, (cudaStream_t)s);
}

extern "C" int fos_surrogate_pair_count(FosCtx* c, int* pairs, int* overflow, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(c->sur && c->sur->n > 0, FOS_E_STATE, "no pair build on this context");
    FosSurBufs* b = c->sur;
    int rc = sur_scan(c, (cudaStream_t)s);
    if (rc) return rc;
    int* h = (int*)c->pinned;
    FOS_CUDA(cudaMemcpyAsync(h, b->pstart + b->n, 4, cudaMemcpyDeviceToHost, (cudaStream_t)s));
    FOS_CUDA(cudaMemcpyAsync(h + 2, b->cnt + SC_OVERFLOW, 8, cudaMemcpyDeviceToHost,
                             (cudaStream_t)s));
    FOS_CUDA(cudaStreamSynchronize((cudaStream_t)s));
    if (pairs) *pairs = h[0];
    if (overflow) *overflow = (int)*(unsigned long long*)(h + 2);
    return FOS_OK;
}

extern "C" int fos_surrogate_export(FosCtx* c, const float* rad, float* X, float* y,
                                    int32_t* pair_i, int32_t* pair_j, const int32_t* mem_nl,
                                    const int32_t* mem_used, const int32_t* mem_fsc,
                                    fos_stream_t s) {
    FOS_REQUIRE(c && rad, FOS_E_ARG, "NULL argument");
    if (!mem_nl) mem_nl = c->nl;
    if (!mem_used) mem_used = c->used;
    if (!mem_fsc) mem_fsc = c->fsc;
    FOS_REQUIRE(((uintptr_t)mem_nl & 15u) == 0, FOS_E_ARG,
                "mem_nl must be 16-byte aligned (its rows are read as 16-byte vectors)");
    FOS_REQUIRE(c->sur && c->sur->n > 0, FOS_E_STATE, "no pair build on this context");
    FosSurBufs* b = c->sur;
    const int n = b->n;
    int rc = sur_scan(c, (cudaStream_t)s);
    if (rc) return rc;
    k_sur_export<<<fos_blocks(32LL * n, 256), 256, 0, (cudaStream_t)s>>>(
        n, b->pj, b->pnd, b->pstart, rad, b->hist, b->cutoff, pair_i, pair_j, X, y, c->nl,
        mem_nl, mem_used, mem_fsc);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_surrogate_predict(FosCtx* c, const FosSurrogate* m, const float* rad,
                                     float* fsc_float, int32_t* fsc_int, float* pair_prob,
                                     fos_stream_t s) {
    FOS_REQUIRE(c && m && rad, FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(c->sur && c->sur->n > 0, FOS_E_STATE, "no pair build on this context");
    FOS_REQUIRE(m->cutoff == c->sur->cutoff, FOS_E_ARG,
                "model cutoff differs from the cutoff of the last pair build");
    if (pair_prob) {
        int rc = sur_scan(c, (cudaStream_t)s);
        if (rc) return rc;
    }
    return sur_predict_impl(c, m, rad, fsc_float, fsc_int, pair_prob, (cudaStream_t)s);
}

extern "C" int fos_surrogate_set_mode(FosCtx* c, int mode) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(mode == FOS_SUR_ABSOLUTE || mode == FOS_SUR_ANCHORED, FOS_E_ARG,
                "mode must be FOS_SUR_ABSOLUTE or FOS_SUR_ANCHORED");
    c->sur_mode = mode;
    return FOS_OK;
}

extern "C" int fos_surrogate_stats(FosCtx* c, FosSurrogateStats* out, fos_stream_t s) {
    FOS_REQUIRE(c && out, FOS_E_ARG, "NULL argument");
    memset(out, 0, sizeof(*out));
    if (!c->sur) return FOS_OK;
    FosSurBufs* b = c->sur;
    if (b->n > 0) {
        int rc = sur_scan(c, (cudaStream_t)s);
        if (rc) return rc;
    }
    unsigned long long* h = (unsigned long long*)c->pinned;
    FOS_CUDA(cudaMemcpyAsync(h, b->cnt, SC_N * 8, cudaMemcpyDeviceToHost, (cudaStream_t)s));
    int* hp = (int*)(h + SC_N);
    hp[0] = 0;
    if (b->n > 0)
        FOS_CUDA(cudaMemcpyAsync(hp, b->pstart + b->n, 4, cudaMemcpyDeviceToHost, (cudaStream_t)s));
    FOS_CUDA(cudaStreamSynchronize((cudaStream_t)s));
    out->pairs = hp[0];
    out->overflow = (int)h[SC_OVERFLOW];
    out->judged = (int)h[SC_JUDGED];
    out->exact = (int)h[SC_EXACT];
    out->within1 = (int)h[SC_WITHIN1];
    out->stale_exact = (int)h[SC_STALE_EXACT];
    out->stale_within1 = (int)h[SC_STALE_WITHIN1];
    out->abs_err = (double)h[SC_ABS_ERR] / 1048576.0;
    out->stale_abs_err = (double)h[SC_STALE_ABS_ERR];
    return FOS_OK;
}

// ------------------------------------------------------------ frame hooks
// Called by the frame driver (frame.cu) after the dynamics of a frame.
int fos_sur_frame_before_jfa(FosCtx* c, const FosSurrogate* m, const FosState* st,
                             const FosFrameParams* fp, cudaStream_t s) {
    const int n = st->n;
    int rc = sur_pairs_impl(c, m, st->pos, st->rad, n, (float)fp->r_max, st->cell_start,
                            st->cell_count, st->cell_indices, s);
    if (rc) return rc;
    rc = sur_predict_impl(c, m, st->rad, nullptr, nullptr, nullptr, s);
    if (rc) return rc;
    FosSurBufs* b = c->sur;
    // the stale baseline: the fsc the reference would have kept using
    FOS_CUDA(cudaMemcpyAsync(b->prev, c->fsc, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    k_sur_combine<<<fos_blocks(n, 256), 256, 0, s>>>(n, c->sur_mode, b->raw, b->prev, b->anchor,
                                                     b->anchor_valid, b->fscf, b->fsci);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

int fos_sur_frame_judge(FosCtx* c, int n, cudaStream_t s) {
    FosSurBufs* b = c->sur;
    k_sur_judge_reset<<<1, 32, 0, s>>>(b->cnt);
    FOS_LAUNCHED(c);
    k_sur_judge<<<fos_blocks(n, 256), 256, 0, s>>>(n, b->fscf, c->fsc, b->prev, b->raw, b->anchor,
                                                   b->anchor_valid, b->cnt);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

int fos_launch_set_targets(FosCtx* c, const float* rad, float* rt, const int32_t* fsc,
                           const float* ema, int n, int f_low, int f_high, float growth,
                           float rmin, float rmax, FosDevState* gate, int warm_frames,
                           double zero_thresh, int adjust_frames, cudaStream_t s);

int fos_sur_frame_between(FosCtx* c, const FosSurrogate* m, const FosState* st,
                          const FosFrameParams* fp, cudaStream_t s) {
    const int n = st->n;
    int rc = sur_pairs_impl(c, m, st->pos, st->rad, n, (float)fp->r_max, st->cell_start,
                            st->cell_count, st->cell_indices, s);
    if (rc) return rc;
    rc = sur_predict_impl(c, m, st->rad, nullptr, nullptr, nullptr, s);
    if (rc) return rc;
    FosSurBufs* b = c->sur;
    k_sur_combine<<<fos_blocks(n, 256), 256, 0, s>>>(n, c->sur_mode, b->raw, c->fsc, b->anchor,
                                                     b->anchor_valid, b->fscf, b->fsci);
    FOS_LAUNCHED(c);
    k_sur_ema<<<fos_blocks(n, 256), 256, 0, s>>>(n, b->fscf, c->ema, c->ema_alpha);
    FOS_LAUNCHED(c);
    return fos_launch_set_targets(c, st->rad, st->rad_target, b->fsci, c->ema, n, fp->f_low,
                                  fp->f_high, (float)fp->growth_pct, (float)fp->r_min,
                                  (float)fp->r_max, c->ds, fp->warmstart_frames,
                                  fp->zero_rate_thresh, fp->adjustment_frames, s);
}

// ------------------------------------------------------------ ensemble hooks
// The surrogate over a batched ensemble's packed particles (ensemble.cu):
// candidate pairs on each foam's own hash grid (k_sur_pairs_ens), then the
// inference and the per-particle steps of the single-foam hooks above, which
// do not depend on which foam a particle belongs to.
static int sur_ens_pairs_predict(FosCtx* c, const FosSurrogate* m, const SurEnsGrid& g,
                                 cudaStream_t s) {
    int rc = fos_sur_prepare(c);
    if (rc) return rc;
    FosSurBufs* b = c->sur;
    rc = fos_grid_gather_sorted(c, g.ci, g.pos, g.rad, g.n, s);
    if (rc) return rc;
    FOS_CUDA(cudaMemsetAsync(b->cnt + SC_OVERFLOW, 0, 8, s));
    k_sur_pairs_ens<<<fos_blocks(32LL * g.n, 256), 256, 0, s>>>(
        c->sorted, g.ci, g.n, c->L, c->invL, c->halfL, g.foam_of, g.fG, g.fcell, g.frmax, g.cs,
        g.cc, m->cutoff, b->pj, b->pnd, b->pcount, b->hist, b->cnt);
    FOS_LAUNCHED(c);
    b->n = g.n;
    b->cutoff = m->cutoff;
    return sur_predict_impl(c, m, g.rad, nullptr, nullptr, nullptr, s);
}

// A non-JFA frame: the mode's FSC f and fsc_ema <- alpha f + (1 - alpha)
// fsc_ema; the caller sets the targets from fos_sur_fsc_int(c).
int fos_sur_ens_between(FosCtx* c, const FosSurrogate* m, const SurEnsGrid& g, cudaStream_t s) {
    int rc = sur_ens_pairs_predict(c, m, g, s);
    if (rc) return rc;
    FosSurBufs* b = c->sur;
    k_sur_combine<<<fos_blocks(g.n, 256), 256, 0, s>>>(g.n, c->sur_mode, b->raw, c->fsc,
                                                       b->anchor, b->anchor_valid, b->fscf,
                                                       b->fsci);
    FOS_LAUNCHED(c);
    k_sur_ema<<<fos_blocks(g.n, 256), 256, 0, s>>>(g.n, b->fscf, c->ema, c->ema_alpha);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// A JFA frame: the estimate for the same positions and the stale baseline,
// judged by fos_sur_frame_judge after the JFA.
int fos_sur_ens_before_jfa(FosCtx* c, const FosSurrogate* m, const SurEnsGrid& g,
                           cudaStream_t s) {
    int rc = sur_ens_pairs_predict(c, m, g, s);
    if (rc) return rc;
    FosSurBufs* b = c->sur;
    FOS_CUDA(cudaMemcpyAsync(b->prev, c->fsc, (size_t)g.n * 4, cudaMemcpyDeviceToDevice, s));
    k_sur_combine<<<fos_blocks(g.n, 256), 256, 0, s>>>(g.n, c->sur_mode, b->raw, b->prev,
                                                       b->anchor, b->anchor_valid, b->fscf,
                                                       b->fsci);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

const int32_t* fos_sur_fsc_int(FosCtx* c) { return c->sur ? c->sur->fsci : nullptr; }

// Inference kernel of the surrogate on ctx: 0 the mma.sync segment kernel
// (k_sur_mlp_seg), 1 the tcgen05 / TMEM tile kernel (k_sur_mlp_tc).
extern "C" int fos_surrogate_set_inference(FosCtx* c, int kind) {
    FOS_REQUIRE(c, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(kind == 0 || kind == 1, FOS_E_ARG, "kind must be 0 (mma.sync) or 1 (tcgen05)");
    c->sur_tc = kind;
    return FOS_OK;
}
