// coop.cuh -- building blocks of the persistent cooperative kernels: the
// block scan, the bounded grid barrier's tracing hook, and the hash-grid
// rebuild as grid-barrier phases (grid.py:145-309 / run.py:476-504).  The
// single-foam frame kernel (frame_coop.cu) and the ensemble frame kernel
// (ensemble.cu) share them; a Geo policy maps a particle to its cell:
//   UniGeo   one periodic grid of G^3 cells;
//   the ensemble's policy, foam f's grid at its offset in the packed table.
#pragma once

#include "phases.cuh"

#define COOP_THREADS 1024
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
    if (a.trace && blockIdx.x == 0 && threadIdx.x == 0 && k < a.trace_cap) a.trace[k] = global_ns();
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

// Rebuild of the hash grid from src into dst (wrapped), with the cell-ordered
// copy sp[k] = (pos, rad) when rad != NULL.  Ends with a grid barrier unless
// last.  Returns false if a barrier timed out.
//
// Small cell tables (G3 <= COOP_SMALL_G3): three phases -- histogram + ranks;
// every block scans the whole table into its shared memory (block 0 also
// writes cell_count/cell_start) and scatters ranks; stable placement from the
// block's own copy of the starts.  Large tables: the chunked four-phase form.
template <class Args, class Geo>
__device__ bool coop_grid(const Args& a, const Geo& geo, const float* src, float* dst,
                          const float* rad, bool last, int& tk, unsigned int& ep) {
    extern __shared__ int s_tab[];  // small form: G3 + 1 exclusive starts
    const int T = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    // P1: histogram + arrival rank (cnt is all-zero on entry)
    for (int i = tid; i < a.n; i += T) {
        float wx = grid_wrap(__ldcg(&src[3 * i + 0]), geo.L, geo.invL);
        float wy = grid_wrap(__ldcg(&src[3 * i + 1]), geo.L, geo.invL);
        float wz = grid_wrap(__ldcg(&src[3 * i + 2]), geo.L, geo.invL);
        dst[3 * i + 0] = wx;
        dst[3 * i + 1] = wy;
        dst[3 * i + 2] = wz;
        int c = geo.cell(i, wx, wy, wz);
        a.cellof[i] = c;
        a.rank[i] = atomicAdd(&a.cnt[c], 1);
    }
    if (!grid_barrier(a.ds, ep)) return false;
    trace_mark(a, tk);
    if (a.small_grid) {
        // P2: whole-table scan per block, then the rank scatter
        const int per = (a.G3 + blockDim.x - 1) / blockDim.x;
        const int b0 = threadIdx.x * per, b1 = min(a.G3, b0 + per);
        int sum = 0;
        for (int c = b0; c < b1; ++c) {
            int v = __ldcg(&a.cnt[c]);
            s_tab[c] = v;
            sum += v;
        }
        int tot;
        int run = coop_block_scan(sum, &tot);
        for (int c = b0; c < b1; ++c) {
            int v = s_tab[c];
            s_tab[c] = run;
            if (blockIdx.x == 0) {
                a.cc[c] = v;
                a.cs[c] = run;
            }
            run += v;
        }
        if (threadIdx.x == 0) s_tab[a.G3] = tot;
        __syncthreads();
        for (int i = tid; i < a.n; i += T)
            a.ci_tmp[s_tab[__ldcg(&a.cellof[i])] + __ldcg(&a.rank[i])] = i;
        if (!grid_barrier(a.ds, ep)) return false;
        trace_mark(a, tk);
        // P3: stable placement from the block's copy of the starts
        int c0 = blockIdx.x * a.chunk;
        for (int c = c0 + threadIdx.x; c < c0 + a.chunk && c < a.G3; c += blockDim.x)
            a.cnt[c] = 0;  // ready for the next rebuild; nobody reads cnt in this phase
        for (int i = tid; i < a.n; i += T) {
            int c = __ldcg(&a.cellof[i]);
            int b = s_tab[c], e = s_tab[c + 1];
            int r = 0;
            for (int k = b; k < e; ++k) r += __ldcg(&a.ci_tmp[k]) < i;
            a.ci[b + r] = i;
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
            int v = in ? __ldcg(&a.cnt[c]) : 0;
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
            a.cnt[c] = 0;  // ready for the next rebuild; nobody reads cnt in this phase
        }
        for (int i = tid; i < a.n; i += T) {
            int c = __ldcg(&a.cellof[i]);
            int slot = __ldcg(&a.part[c]) + s_pre[c / a.chunk] + __ldcg(&a.rank[i]);
            a.ci_tmp[slot] = i;
        }
    }
    if (!grid_barrier(a.ds, ep)) return false;
    trace_mark(a, tk);
    // P4: stable placement: slot = cell start + #(lower-indexed particles in the cell)
    for (int i = tid; i < a.n; i += T) {
        int c = __ldcg(&a.cellof[i]);
        int b = __ldcg(&a.cs[c]), e = b + __ldcg(&a.cc[c]);
        int r = 0;
        for (int k = b; k < e; ++k) r += __ldcg(&a.ci_tmp[k]) < i;
        a.ci[b + r] = i;
        if (rad) {
            a.sp[b + r] = make_float4(__ldcg(&dst[3 * i + 0]), __ldcg(&dst[3 * i + 1]),
                                      __ldcg(&dst[3 * i + 2]), __ldcg(&rad[i]));
        }
    }
    if (!last && !grid_barrier(a.ds, ep)) return false;
    trace_mark(a, tk);
    return true;
}

