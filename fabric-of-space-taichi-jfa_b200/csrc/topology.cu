// topology.cu -- Gabriel-graph and k-NN topological degree on the hash grid
// (topology.py), an FSC-independent neighbour count.
//
// One warp per particle.  Candidate pairs are enumerated in the reference's
// serial order (27 cells in (dx, dy, dz) order, each cell's particles in
// ascending index order, the CSR grid of the last rebuild) and appended by
// ballot + prefix popcount, so the first MAX_TOPO_NEIGHBORS candidates and the
// truncation flag are the serial loop's.  A Gabriel witness search is a pure
// existence test, so the warp tests 32 witnesses at a time and stops at the
// first chunk that holds one; degrees are integer atomics.  Every float
// expression keeps the reference's operation order (no contraction).
#include "phases.cuh"

struct TopoGeo {
    int G;
    float L, invL, halfL;
};

// grid.pdelta (grid.py:51-66): wrapP(b - a) per component.
__device__ __forceinline__ float3 topo_pdelta(float3 a, float3 b, const TopoGeo& g) {
    return make_float3(grid_wrap(fsub(b.x, a.x), g.L, g.invL),
                       grid_wrap(fsub(b.y, a.y), g.L, g.invL),
                       grid_wrap(fsub(b.z, a.z), g.L, g.invL));
}

__device__ __forceinline__ float topo_dot(float3 d) {
    return fadd(fadd(fmul(d.x, d.x), fmul(d.y, d.y)), fmul(d.z, d.z));
}

// int(((p + HALF_L) * INV_L) * GRID_RES) of an already wrapped coordinate,
// then wrap_cell (topology.py:206-209).
__device__ __forceinline__ int topo_cell_coord(float w, const TopoGeo& g) {
    return wrap_near((int)fmul(fmul(fadd(w, g.halfL), g.invL), (float)g.G), g.G);
}

__device__ __forceinline__ float3 ld3(const float* p, int i) {
    return make_float3(__ldg(&p[3 * i + 0]), __ldg(&p[3 * i + 1]), __ldg(&p[3 * i + 2]));
}

// build_topo_candidates (topology.py:68-135) for particle i (one warp).
__global__ void __launch_bounds__(256) k_topo_candidates(
    const float* __restrict__ pos, const float* __restrict__ rad,
    const int32_t* __restrict__ cs, const int32_t* __restrict__ cc,
    const int32_t* __restrict__ ci, int n, TopoGeo g, float mult, int cap,
    int32_t* __restrict__ pairs, int32_t* __restrict__ pcount, int32_t* __restrict__ trunc) {
    const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;  // warp-uniform
    const float3 pi = ld3(pos, i);
    const float ri = __ldg(&rad[i]);
    const Stencil r = stencil_ranges<LdRO>(pi.x, pi.y, pi.z, g.L, g.invL, g.halfL, g.G, cs, cc,
                                           lane);
    int count = 0;
    bool truncated = false;
    for (int base = 0; base < r.total && !truncated; base += 32) {
        const int t = base + lane;
        const int k = stencil_locate(r, t < r.total ? t : r.total - 1);
        bool take = false;
        int j = -1;
        if (t < r.total) {
            j = __ldg(&ci[k]);
            if (j > i) {
                const float d2 = topo_dot(topo_pdelta(pi, ld3(pos, j), g));
                const float th = fmul(mult, fadd(ri, __ldg(&rad[j])));
                take = d2 <= fmul(th, th);
            }
        }
        const unsigned int m = __ballot_sync(0xffffffffu, take);
        const int slot = count + __popc(m & ((1u << lane) - 1u));
        if (take && slot < cap) pairs[(size_t)i * cap + slot] = j;
        count += __popc(m);
        if (count > cap) truncated = true;  // warp-uniform
    }
    if (lane == 0) {
        pcount[i] = count < cap ? count : cap;
        trunc[i] = truncated ? 1 : 0;
    }
}

// Is there a witness k (k != i, j) with |pdelta| ^ 2 < thr around the
// midpoint m (cells [-s, s]^3 around mid cell (mx, my, mz))?  rev selects the
// argument order of pdelta (pdelta(pos[k], m) or pdelta(m, pos[k])).  All 32
// lanes; returns the same answer on every lane.
__device__ bool topo_witness(float3 m, float thr, int i, int j, int mx, int my, int mz, int s,
                             bool rev, const float* __restrict__ pos,
                             const int32_t* __restrict__ cs, const int32_t* __restrict__ cc,
                             const int32_t* __restrict__ ci, const TopoGeo& g, int lane) {
    const int w = 2 * s + 1;
    const int ncell = w * w * w;
    for (int c0 = 0; c0 < ncell; c0 += 32) {
        const int cidx = c0 + lane;
        int st = 0, ct = 0;
        if (cidx < ncell) {
            const int dx = cidx / (w * w) - s, dy = (cidx / w) % w - s, dz = cidx % w - s;
            const int nx = wrap_mod(mx + dx, g.G), ny = wrap_mod(my + dy, g.G),
                      nz = wrap_mod(mz + dz, g.G);
            const int cid = (nx * g.G + ny) * g.G + nz;
            st = __ldg(&cs[cid]);
            ct = __ldg(&cc[cid]);
        }
        int incl = ct;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        Stencil r{st, incl - ct, incl, __shfl_sync(0xffffffffu, incl, 31)};
        for (int base = 0; base < r.total; base += 32) {
            const int t = base + lane;
            const int kk = stencil_locate(r, t < r.total ? t : r.total - 1);
            bool hit = false;
            if (t < r.total) {
                const int k = __ldg(&ci[kk]);
                if (k != i && k != j) {
                    const float3 pk = ld3(pos, k);
                    const float d2 = topo_dot(rev ? topo_pdelta(m, pk, g) : topo_pdelta(pk, m, g));
                    hit = d2 < thr;
                }
            }
            if (__any_sync(0xffffffffu, hit)) return true;
        }
    }
    return false;
}

// The witness test of one pair (topology.py:198-253 / 407-443).
__device__ bool topo_gabriel_pair(int i, int j, float3 pi, float3 pj, float d2, float cell_size,
                                  bool rev, const float* __restrict__ pos,
                                  const int32_t* __restrict__ cs, const int32_t* __restrict__ cc,
                                  const int32_t* __restrict__ ci, const TopoGeo& g, int lane) {
    const float3 d = topo_pdelta(pi, pj, g);
    const float3 m = make_float3(grid_wrap(fadd(pi.x, fmul(0.5f, d.x)), g.L, g.invL),
                                 grid_wrap(fadd(pi.y, fmul(0.5f, d.y)), g.L, g.invL),
                                 grid_wrap(fadd(pi.z, fmul(0.5f, d.z)), g.L, g.invL));
    const float r_sq = fmul(0.25f, d2);
    const float r_d = fmul(__fsqrt_rn(d2), 0.5f);
    int s = (int)ceilf(fdiv(r_d, cell_size));
    s = max(1, min(s, 3));
    s = min(s, g.G / 2);
    const float eps = fmaxf(1e-12f, fmul(1e-6f, r_sq));
    const float thr = fsub(r_sq, eps);
    return !topo_witness(m, thr, i, j, topo_cell_coord(m.x, g), topo_cell_coord(m.y, g),
                         topo_cell_coord(m.z, g), s, rev, pos, cs, cc, ci, g, lane);
}

// hash of the pair subsampling (topology.py:181-184, 325-333) in wrapping
// int32 arithmetic; kept when divisible by q.
__device__ __forceinline__ bool topo_keep(int i, int j, int frame, int q) {
    const unsigned int h = ((unsigned int)i * 73856093u) ^ ((unsigned int)j * 19349663u) ^
                           ((unsigned int)frame * 83492791u);
    return q <= 1 || ((int)h % q) == 0;
}

// gabriel_test_topological_degree (topology.py:140-262), particle i's
// candidate list (one warp); deg must be zeroed before.
__global__ void __launch_bounds__(256) k_topo_gabriel(
    const float* __restrict__ pos, const int32_t* __restrict__ cs,
    const int32_t* __restrict__ cc, const int32_t* __restrict__ ci, int n, TopoGeo g,
    float cell_size, int frame, int stride, int early_exit, float deg_high, int cap,
    const int32_t* __restrict__ pairs, const int32_t* __restrict__ pcount,
    const float* __restrict__ deg_ema, int32_t* deg) {
    const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const int pc = __ldg(&pcount[i]);
    const float3 pi = ld3(pos, i);
    // lane p < pc screens candidate p; the survivors are tested one by one
    bool need = false;
    int j = -1;
    float d2 = 0.f;
    if (lane < pc) {
        j = __ldg(&pairs[(size_t)i * cap + lane]);
        need = topo_keep(i, j, frame, stride);
        if (need && early_exit && __ldg(&deg_ema[i]) >= deg_high && __ldg(&deg_ema[j]) >= deg_high)
            need = false;
        if (need) {
            d2 = topo_dot(topo_pdelta(pi, ld3(pos, j), g));
            need = !(d2 < 1e-16f);
        }
    }
    unsigned int m = __ballot_sync(0xffffffffu, need);
    int found = 0;
    while (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1;
        const int jb = __shfl_sync(0xffffffffu, j, b);
        const float db = __shfl_sync(0xffffffffu, d2, b);
        const bool gab = topo_gabriel_pair(i, jb, pi, ld3(pos, jb), db, cell_size, false, pos, cs,
                                           cc, ci, g, lane);
        if (gab && jb > i) {
            ++found;
            if (lane == 0) atomicAdd(&deg[jb], 1);
        }
    }
    if (lane == 0 && found) atomicAdd(&deg[i], found);
}

// gabriel_update_batched (topology.py:335-446): particles with
// i % num_batches == batch build their subsampled candidates (j > i,
// should_sample_pair) and test them; deg accumulates across batches.
__global__ void __launch_bounds__(256) k_topo_batched(
    const float* __restrict__ pos, const float* __restrict__ rad,
    const int32_t* __restrict__ cs, const int32_t* __restrict__ cc,
    const int32_t* __restrict__ ci, int n, TopoGeo g, float mult, float cell_size, int batch,
    int num_batches, int q, int frame, int cap, int32_t* __restrict__ pairs,
    int32_t* __restrict__ pcount, int32_t* __restrict__ trunc, int32_t* deg) {
    const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int i = w * num_batches + batch;
    if (i >= n) return;
    const float3 pi = ld3(pos, i);
    const float ri = __ldg(&rad[i]);
    const Stencil r = stencil_ranges<LdRO>(pi.x, pi.y, pi.z, g.L, g.invL, g.halfL, g.G, cs, cc,
                                           lane);
    int count = 0;
    for (int base = 0; base < r.total; base += 32) {
        const int t = base + lane;
        const int k = stencil_locate(r, t < r.total ? t : r.total - 1);
        bool take = false;
        int j = -1;
        if (t < r.total) {
            j = __ldg(&ci[k]);
            if (j > i && topo_keep(i, j, frame, q)) {
                const float d2 = topo_dot(topo_pdelta(pi, ld3(pos, j), g));
                const float th = fmul(mult, fadd(ri, __ldg(&rad[j])));
                take = d2 <= fmul(th, th);
            }
        }
        const unsigned int m = __ballot_sync(0xffffffffu, take);
        const int slot = count + __popc(m & ((1u << lane) - 1u));
        if (take && slot < cap) pairs[(size_t)i * cap + slot] = j;
        count += __popc(m);
    }
    const int pc = count < cap ? count : cap;
    if (lane == 0) {
        pcount[i] = count;  // the reference's counter keeps counting past the cap
        trunc[i] = count > cap ? 1 : 0;
    }
    __syncwarp();
    int found = 0;
    for (int p = 0; p < pc; ++p) {
        const int j = __ldg(&pairs[(size_t)i * cap + p]);
        const float3 pj = ld3(pos, j);
        const float d2 = topo_dot(topo_pdelta(pi, pj, g));
        if (d2 < 1e-16f) continue;
        if (topo_gabriel_pair(i, j, pi, pj, d2, cell_size, true, pos, cs, cc, ci, g, lane)) {
            ++found;
            if (lane == 0) atomicAdd(&deg[j], 1);
        }
    }
    if (lane == 0 && found) atomicAdd(&deg[i], found);
}

// knn_topo_degree (topology.py:458-505): neighbours within (mult * r_i)^2,
// capped at k.
__global__ void __launch_bounds__(256) k_topo_knn(
    const float* __restrict__ pos, const float* __restrict__ rad,
    const int32_t* __restrict__ cs, const int32_t* __restrict__ cc,
    const int32_t* __restrict__ ci, int n, TopoGeo g, float mult, int kmax,
    int32_t* __restrict__ deg) {
    const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const float3 pi = ld3(pos, i);
    const float lim = fmul(mult, __ldg(&rad[i]));
    const float lim2 = fmul(lim, lim);
    const Stencil r = stencil_ranges<LdRO>(pi.x, pi.y, pi.z, g.L, g.invL, g.halfL, g.G, cs, cc,
                                           lane);
    int count = 0;
    for (int base = 0; base < r.total && count < kmax; base += 32) {
        const int t = base + lane;
        const int k = stencil_locate(r, t < r.total ? t : r.total - 1);
        bool hit = false;
        if (t < r.total) {
            const int j = __ldg(&ci[k]);
            if (j != i) hit = topo_dot(topo_pdelta(pi, ld3(pos, j), g)) <= lim2;
        }
        count += __popc(__ballot_sync(0xffffffffu, hit));
    }
    if (lane == 0) deg[i] = count < kmax ? count : kmax;
}

// update_topo_ema (topology.py:265-283) and commit_topo_to_ema (topology.py:448-455).
__global__ void k_topo_ema(const int32_t* __restrict__ deg, float* __restrict__ ema, float alpha,
                           int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ema[i] = fadd(fmul(alpha, (float)deg[i]), fmul(fsub(1.0f, alpha), ema[i]));
}

// update_radii_topological (topology.py:286-322).
__global__ void k_topo_radii(float* __restrict__ rad, const float* __restrict__ deg_eff,
                             float lo, float hi, float grow, float shrink, float rmin, float rmax,
                             int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float d = deg_eff[i];
    float r = rad[i];
    if (d < lo) r = fmul(r, fadd(1.0f, grow));
    else if (d > hi) r = fmul(r, fsub(1.0f, shrink));
    rad[i] = fmaxf(rmin, fminf(rmax, r));
}

// ---------------------------------------------------------------- host side
static TopoGeo topo_geo(const FosCtx* c) { return TopoGeo{c->G, c->L, c->invL, c->halfL}; }

static int topo_check(FosCtx* c, int n) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(n >= 0 && n <= c->max_n, FOS_E_CAPACITY, "n outside [0, max_n]");
    return FOS_OK;
}

extern "C" int fos_topo_candidates(FosCtx* c, const float* pos, const float* rad,
                                   const int32_t* cell_start, const int32_t* cell_count,
                                   const int32_t* cell_indices, int n, double max_radius_multiple,
                                   int cap, int32_t* topo_pairs, int32_t* pair_count,
                                   int32_t* truncated, fos_stream_t s) {
    int rc = topo_check(c, n);
    if (rc) return rc;
    FOS_REQUIRE(cap >= 1 && cap <= 32, FOS_E_ARG, "cap must be in [1, 32]");
    FOS_REQUIRE(n == 0 || (pos && rad && cell_start && cell_count && cell_indices && topo_pairs &&
                           pair_count && truncated),
                FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    k_topo_candidates<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(
        pos, rad, cell_start, cell_count, cell_indices, n, topo_geo(c), (float)max_radius_multiple,
        cap, topo_pairs, pair_count, truncated);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_topo_gabriel(FosCtx* c, const float* pos, const int32_t* cell_start,
                                const int32_t* cell_count, const int32_t* cell_indices, int n,
                                int frame, double cell_size, int stride, int early_exit,
                                double deg_high, int cap, const int32_t* topo_pairs,
                                const int32_t* pair_count, const float* deg_ema, int32_t* deg,
                                fos_stream_t s) {
    int rc = topo_check(c, n);
    if (rc) return rc;
    FOS_REQUIRE(cap >= 1 && cap <= 32 && cell_size > 0.0, FOS_E_ARG,
                "cap must be in [1, 32] and cell_size > 0");
    FOS_REQUIRE(n == 0 || (pos && cell_start && cell_count && cell_indices && topo_pairs &&
                           pair_count && deg_ema && deg),
                FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    FOS_CUDA(cudaMemsetAsync(deg, 0, (size_t)n * 4, s));
    k_topo_gabriel<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(
        pos, cell_start, cell_count, cell_indices, n, topo_geo(c), (float)cell_size, frame, stride,
        early_exit, (float)deg_high, cap, topo_pairs, pair_count, deg_ema, deg);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_topo_batched(FosCtx* c, const float* pos, const float* rad,
                                const int32_t* cell_start, const int32_t* cell_count,
                                const int32_t* cell_indices, int n, int batch, int num_batches,
                                int subsample_q, int frame, double max_radius_multiple,
                                double cell_size, int cap, int32_t* topo_pairs,
                                int32_t* pair_count, int32_t* truncated, int32_t* deg,
                                fos_stream_t s) {
    int rc = topo_check(c, n);
    if (rc) return rc;
    FOS_REQUIRE(num_batches >= 1 && batch >= 0 && batch < num_batches && subsample_q >= 1,
                FOS_E_ARG, "need 0 <= batch < num_batches and subsample_q >= 1");
    FOS_REQUIRE(cap >= 1 && cap <= 32 && cell_size > 0.0, FOS_E_ARG,
                "cap must be in [1, 32] and cell_size > 0");
    FOS_REQUIRE(n == 0 || (pos && rad && cell_start && cell_count && cell_indices && topo_pairs &&
                           pair_count && truncated && deg),
                FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    const long long warps = ((long long)n + num_batches - 1) / num_batches;
    k_topo_batched<<<fos_blocks(32LL * warps, 256), 256, 0, s>>>(
        pos, rad, cell_start, cell_count, cell_indices, n, topo_geo(c), (float)max_radius_multiple,
        (float)cell_size, batch, num_batches, subsample_q, frame, cap, topo_pairs, pair_count,
        truncated, deg);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_topo_knn(FosCtx* c, const float* pos, const float* rad,
                            const int32_t* cell_start, const int32_t* cell_count,
                            const int32_t* cell_indices, int n, int k, double max_radius_multiple,
                            int32_t* deg, fos_stream_t s) {
    int rc = topo_check(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (pos && rad && cell_start && cell_count && cell_indices && deg),
                FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    k_topo_knn<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(pos, rad, cell_start, cell_count,
                                                         cell_indices, n, topo_geo(c),
                                                         (float)max_radius_multiple, k, deg);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_topo_ema(FosCtx* c, const int32_t* deg, float* deg_ema, float alpha, int n,
                            fos_stream_t s) {
    int rc = topo_check(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (deg && deg_ema), FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    k_topo_ema<<<fos_blocks(n, 256), 256, 0, s>>>(deg, deg_ema, alpha, n);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_topo_update_radii(FosCtx* c, float* rad, const float* deg_effective,
                                     float deg_low, float deg_high, float gain_grow,
                                     float gain_shrink, float r_min, float r_max, int n,
                                     fos_stream_t s) {
    int rc = topo_check(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (rad && deg_effective), FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    k_topo_radii<<<fos_blocks(n, 256), 256, 0, s>>>(rad, deg_effective, deg_low, deg_high,
                                                    gain_grow, gain_shrink, r_min, r_max, n);
    FOS_LAUNCHED(c);
    return FOS_OK;
}
