// phases.cuh -- per-particle / per-warp device functions of the frame's
// stages.  The standalone kernels (grid.cu, dynamics.cu) and the persistent
// cooperative frame kernel (frame_coop.cu) both call these, so each stage's
// arithmetic exists once.
//
// Reference: grid.py (cells, wrap), dynamics.py (PBD, max overlap, pressure,
// Brownian, FSC controller).  FP32 expressions keep the reference's operator
// order with explicit round-to-nearest intrinsics (no FMA contraction).
#pragma once

#include <math.h>

#include "fos_internal.cuh"

// Load policies.  Standalone kernels read data no thread of the same launch
// writes, through the read-only path (LdRO); the persistent cooperative frame
// kernel rewrites cells, positions and radii between its phases, and other
// SMs' L1 lines would go stale, so it reads through L2 (LdL2).
struct LdRO {
    template <class T>
    __device__ __forceinline__ static T ld(const T* p) { return __ldg(p); }
};
struct LdL2 {
    template <class T>
    __device__ __forceinline__ static T ld(const T* p) { return __ldcg(p); }
};
// Plain, L1-allocating loads, for the cooperative kernel's data that no thread
// writes during the current phase.  Each phase starts after a grid barrier:
// thread 0's acquire load, then the block barrier, orders every later load of
// the block after all writes released before the barrier (PTX memory model),
// so no line cached in an earlier phase is read.
struct LdL1 {
    template <class T>
    __device__ __forceinline__ static T ld(const T* p) { return *p; }
};

// ------------------------------------------------------------------ grid
// Cell of an already wrapped position (grid.py:204-222):
// floor(((w + HALF_L) + 1e-7) * INV_L * GRID_RES), wrapped, c0*G*G + c1*G + c2.
__device__ __forceinline__ int cell_of_wrapped(float wx, float wy, float wz, float invL,
                                               float halfL, int G) {
    float q0 = fmul(fadd(fadd(wx, halfL), 1e-7f), invL);
    float q1 = fmul(fadd(fadd(wy, halfL), 1e-7f), invL);
    float q2 = fmul(fadd(fadd(wz, halfL), 1e-7f), invL);
    int c0 = wrap_near((int)floorf(fmul(q0, (float)G)), G);
    int c1 = wrap_near((int)floorf(fmul(q1, (float)G)), G);
    int c2 = wrap_near((int)floorf(fmul(q2, (float)G)), G);
    return (c0 * G + c1) * G + c2;
}

// Home cell as project_overlaps / compute_local_max_overlaps compute it
// (dynamics.py:101-103): int(((wrapP(p) + HALF_L) * INV_L) * GRID_RES), no
// epsilon and no wrap before the +-1 offsets.
__device__ __forceinline__ int home_coord(float p, float L, float invL, float halfL, int G) {
    float w = grid_wrap(p, L, invL);
    float q = fmul(fadd(w, halfL), invL);
    return (int)fmul(q, (float)G);
}

// Block-wide max of one value per warp (lane 0's), then a single atomicMax
// per block: same-address atomics from every warp serialise in L2.  Every
// warp of the block must call it once.
__device__ __forceinline__ void block_max_atomic(unsigned int warp_val, unsigned int* target) {
    __shared__ unsigned int s_max;
    if (threadIdx.x == 0) s_max = 0u;
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && warp_val) atomicMax(&s_max, warp_val);
    __syncthreads();
    if (threadIdx.x == 0 && s_max) atomicMax(target, s_max);
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

// cap > 0: fixed-capacity cell rows, cell cid starting at slot
// (cell_base + cid) * cap (cs unused); otherwise CSR starts cs[cid].
template <class LD>
__device__ __forceinline__ Stencil stencil_ranges(float px, float py, float pz, float L, float invL,
                                                  float halfL, int G, const int32_t* cs,
                                                  const int32_t* cc, int lane, int cap = 0,
                                                  int cell_base = 0) {
    int hx = home_coord(px, L, invL, halfL, G);
    int hy = home_coord(py, L, invL, halfL, G);
    int hz = home_coord(pz, L, invL, halfL, G);
    int st = 0, ct = 0;
    if (lane < 27) {
        int nx = wrap_near(hx + lane / 9 - 1, G);
        int ny = wrap_near(hy + (lane / 3) % 3 - 1, G);
        int nz = wrap_near(hz + lane % 3 - 1, G);
        int cid = (nx * G + ny) * G + nz;
        st = cap ? (cell_base + cid) * cap : LD::ld(&cs[cid]);
        ct = LD::ld(&cc[cid]);
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

// Stencil cell (lane index) holding candidate t (t < total).
__device__ __forceinline__ int stencil_cell(const Stencil& r, int t) {
    int c = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
        int v = __shfl_sync(0xffffffffu, r.incl, c + step - 1);
        if (v <= t) c += step;
    }
    return c & 31;
}

// Sorted-array position of candidate t (t < total).
__device__ __forceinline__ int stencil_locate(const Stencil& r, int t) {
    const int src = stencil_cell(r, t);
    int st = __shfl_sync(0xffffffffu, r.st, src);
    int ex = __shfl_sync(0xffffffffu, r.excl, src);
    return st + (t - ex);
}

struct GridGeom {
    int G;
    float L, invL, halfL;
};

// stencil_ranges on fixed-capacity rows (cap slots a cell) with the cells that
// cannot hold a particle within `reach` of p dropped (their count taken as 0).
// Per axis, the nearest point of a neighbour cell is at least as far from p
// as the home cell's face on that side (rel: p's offset from the home cell's
// lower face, cs: the cell width), less `margin`, which covers float error and
// the 1e-7 offset of the cell assignment; a cell whose squared bound exceeds
// reach2 is skipped.  The other candidates keep their stencil order, so any
// pair within reach is enumerated exactly as by stencil_ranges.  Needs G >= 5,
// so that the adjacent cells are the nearest periodic images.  cap == 0: the
// CSR form, cell cid starting at cstart[cid]; cell_base as in stencil_ranges.
template <class LD>
__device__ __forceinline__ Stencil stencil_ranges_near(float px, float py, float pz,
                                                       const GridGeom& g, float cs,
                                                       const int32_t* cc, int lane, int cap,
                                                       float reach2, float margin,
                                                       const int32_t* cstart = nullptr,
                                                       int cell_base = 0) {
    const float p3[3] = {px, py, pz};
    int h[3];
    float rel[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {  // home_coord, keeping the wrapped position
        const float w = grid_wrap(p3[a], g.L, g.invL);
        h[a] = (int)fmul(fmul(fadd(w, g.halfL), g.invL), (float)g.G);
        rel[a] = w - ((float)h[a] * cs - g.halfL);
    }
    int st = 0, ct = 0;
    if (lane < 27) {
        const int o[3] = {lane / 9 - 1, (lane / 3) % 3 - 1, lane % 3 - 1};
        const int nx = wrap_near(h[0] + o[0], g.G);
        const int ny = wrap_near(h[1] + o[1], g.G);
        const int nz = wrap_near(h[2] + o[2], g.G);
        const int cid = (nx * g.G + ny) * g.G + nz;
        float b2 = 0.f;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float b = o[a] == 0 ? 0.f : fmaxf(0.f, (o[a] < 0 ? rel[a] : cs - rel[a]) - margin);
            b2 += b * b;
        }
        if (b2 <= reach2) {
            st = cap ? (cell_base + cid) * cap : LD::ld(&cstart[cid]);
            ct = LD::ld(&cc[cid]);
        }
    }
    int incl = ct;
#pragma unroll
    for (int k = 1; k < 32; k <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, k);
        if (lane >= k) incl += y;
    }
    Stencil r;
    r.st = st;
    r.incl = incl;
    r.excl = incl - ct;
    r.total = __shfl_sync(0xffffffffu, incl, 31);
    return r;
}

// Correction of project_overlaps (dynamics.py:120-160) from candidate q on a
// particle at p with radius ri (md = mdf * ri); false when they do not overlap.
__device__ __forceinline__ bool pbd_term(float4 q, float px, float py, float pz, float ri,
                                         float md, float gap1, const GridGeom& g, float& vx,
                                         float& vy, float& vz) {
    float ddx = grid_wrap(fsub(q.x, px), g.L, g.invL);
    float ddy = grid_wrap(fsub(q.y, py), g.L, g.invL);
    float ddz = grid_wrap(fsub(q.z, pz), g.L, g.invL);
    float d2 = fadd(fadd(fadd(fmul(ddx, ddx), fmul(ddy, ddy)), fmul(ddz, ddz)), 1e-12f);
    float dist = __fsqrt_rn(d2);
    float tsep = fmul(fadd(ri, q.w), gap1);
    if (!(dist < tsep)) return false;
    float ov = fsub(tsep, dist);
    float ux = fdiv(ddx, dist), uy = fdiv(ddy, dist), uz = fdiv(ddz, dist);
    float mag = fminf(fmul(ov, 0.5f), md);
    vx = fmaxf(-md, fminf(md, fmul(-ux, mag)));
    vy = fmaxf(-md, fminf(md, fmul(-uy, mag)));
    vz = fmaxf(-md, fminf(md, fmul(-uz, mag)));
    return true;
}

// Adds the hits' corrections in lane order (candidate order).  All 32 lanes.
__device__ __forceinline__ void warp_ordered_add3(bool hit, float vx, float vy, float vz,
                                                  float& cx, float& cy, float& cz) {
    unsigned int m = __ballot_sync(0xffffffffu, hit);
    while (m) {
        int b = __ffs(m) - 1;
        m &= m - 1;
        cx = fadd(cx, __shfl_sync(0xffffffffu, vx, b));
        cy = fadd(cy, __shfl_sync(0xffffffffu, vy, b));
        cz = fadd(cz, __shfl_sync(0xffffffffu, vz, b));
    }
}

// Adds the hits' corrections in ascending key order (keys distinct).  When
// every hit's key exceeds the previous hit's (lane order) they already are in
// order and are added as warp_ordered_add3 does; otherwise each hit takes its
// rank among the hits.  All 32 lanes.
__device__ __forceinline__ void warp_keyed_add3(bool hit, int key, float vx, float vy, float vz,
                                                float& cx, float& cy, float& cz) {
    const unsigned int m = __ballot_sync(0xffffffffu, hit);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const unsigned int before = m & ((1u << lane) - 1u);
    const int prev = 31 - __clz(before);  // -1: no earlier hit
    const int kp = __shfl_sync(0xffffffffu, key, prev & 31);
    if (!__ballot_sync(0xffffffffu, hit && prev >= 0 && kp > key)) {
        for (unsigned int mm = m; mm; mm &= mm - 1) {
            const int b = __ffs(mm) - 1;
            cx = fadd(cx, __shfl_sync(0xffffffffu, vx, b));
            cy = fadd(cy, __shfl_sync(0xffffffffu, vy, b));
            cz = fadd(cz, __shfl_sync(0xffffffffu, vz, b));
        }
        return;
    }
    int rank = 0;
    for (unsigned int mm = m; mm; mm &= mm - 1) rank += __shfl_sync(0xffffffffu, key, __ffs(mm) - 1) < key;
    const int h = __popc(m);
    for (int q = 0; q < h; ++q) {
        const int b = __ffs(__ballot_sync(0xffffffffu, hit && rank == q)) - 1;
        cx = fadd(cx, __shfl_sync(0xffffffffu, vx, b));
        cy = fadd(cy, __shfl_sync(0xffffffffu, vy, b));
        cz = fadd(cz, __shfl_sync(0xffffffffu, vz, b));
    }
}

// End of project_overlaps for one particle (dynamics.py:160-171): cap the
// summed correction at mdf * ri * dmul and return the wrapped new position.
__device__ __forceinline__ float3 pbd_move(float px, float py, float pz, float ri, float cx,
                                           float cy, float cz, float mdf, float dmul,
                                           const GridGeom& g) {
    float mt = fmul(fmul(mdf, ri), dmul);
    float cm = __fsqrt_rn(fadd(fadd(fmul(cx, cx), fmul(cy, cy)), fmul(cz, cz)));
    if (cm > mt) {
        float sc = fdiv(mt, cm);
        cx = fmul(cx, sc);
        cy = fmul(cy, sc);
        cz = fmul(cz, sc);
    }
    return make_float3(grid_wrap(fadd(px, cx), g.L, g.invL), grid_wrap(fadd(py, cy), g.L, g.invL),
                       grid_wrap(fadd(pz, cz), g.L, g.invL));
}

// project_overlaps (dynamics.py:77-171) for the particle at sorted position
// kk, as one Jacobi sweep: reads the pre-sweep positions (the cell-ordered
// copy sp holds pos and rad) and writes pout[i].  The whole warp cooperates:
// lanes evaluate 32 candidates at a time and the corrections of overlapping
// pairs are added in candidate order, so the FP32 sum is the reference loop's
// sum bit for bit.  Must be called by all 32 lanes.
// Returns particle i to lane 0 (-1 to the other lanes); with np != NULL,
// lane 0 also gets the new (wrapped) position and the radius in *np.
// cap / cell_base as in stencil_ranges.  rmax > 0 (the largest radius of any
// candidate; G >= 5): only the cells that can hold a particle within
// (ri + rmax) * gap1 are visited, as in pbd_warp_rows; the candidates left keep
// their order, so the hits and their sum are unchanged.
template <class LD>
__device__ __forceinline__ int pbd_warp(int kk, int lane, const float4* sp, const int32_t* ci,
                                        float* pout, const GridGeom g, const int32_t* cs,
                                        const int32_t* cc, float gap1, float mdf, float dmul,
                                        float4* np = nullptr, int cap = 0, int cell_base = 0,
                                        float rmax = 0.f, float cell_w = 0.f) {
    float4 me = LD::ld(&sp[kk]);
    float px = me.x, py = me.y, pz = me.z, ri = me.w;
    Stencil r;
    if (rmax > 0.f) {
        const float reach = (ri + rmax) * gap1 * 1.0001f;
        r = stencil_ranges_near<LD>(px, py, pz, g, cell_w, cc, lane, cap, reach * reach,
                                    1e-5f * g.L + 1e-6f, cs, cell_base);
    } else {
        r = stencil_ranges<LD>(px, py, pz, g.L, g.invL, g.halfL, g.G, cs, cc, lane, cap,
                               cell_base);
    }
    float md = fmul(mdf, ri);
    float cx = 0.f, cy = 0.f, cz = 0.f;
    for (int base = 0; base < r.total; base += 32) {
        int t = base + lane;
        int k = stencil_locate(r, t < r.total ? t : r.total - 1);
        bool hit = false;
        float vx = 0.f, vy = 0.f, vz = 0.f;
        if (t < r.total && k != kk)
            hit = pbd_term(LD::ld(&sp[k]), px, py, pz, ri, md, gap1, g, vx, vy, vz);
        warp_ordered_add3(hit, vx, vy, vz, cx, cy, cz);
    }
    if (lane == 0) {
        int i = LD::ld(&ci[kk]);
        const float3 n3 = pbd_move(px, py, pz, ri, cx, cy, cz, mdf, dmul, g);
        pout[3 * i + 0] = n3.x;
        pout[3 * i + 1] = n3.y;
        pout[3 * i + 2] = n3.z;
        if (np) *np = make_float4(n3.x, n3.y, n3.z, ri);
        return i;
    }
    return -1;
}

// pbd_warp on fixed-capacity rows (cap <= 32 slots a cell, cell c at c * cap)
// whose particles sit in arrival order, not index order.  Each chunk of
// candidates covers whole stencil cells (a row holds at most 32), and
// a chunk's hits are added in the key order (stencil cell, particle index):
// the reference's loop order, so the sum is pbd_warp's bit for bit.  The
// candidates' particle indices come with their (pos, rad); requires
// n <= 2^26 (the key packs the cell above bit 26).
//
// rmax > 0 (the largest radius of any particle; G >= 5): the stencil keeps only
// the cells that can hold a particle within (ri + rmax) * gap1 of p
// (stencil_ranges_near), which is every cell that can hold an overlap.
// cell_base as in stencil_ranges (cc then indexed from the grid's first cell).
template <class LD>
__device__ __forceinline__ int pbd_warp_rows(int kk, int lane, const float4* sp, const int32_t* ci,
                                             float* pout, const GridGeom g, const int32_t* cc,
                                             int cap, float gap1, float mdf, float dmul,
                                             float4* np, float rmax = 0.f, float cs = 0.f,
                                             int cell_base = 0) {
    float4 me = LD::ld(&sp[kk]);
    float px = me.x, py = me.y, pz = me.z, ri = me.w;
    Stencil r;
    if (rmax > 0.f) {
        const float reach = (ri + rmax) * gap1 * 1.0001f;
        r = stencil_ranges_near<LD>(px, py, pz, g, cs, cc, lane, cap, reach * reach,
                                    1e-5f * g.L + 1e-6f, nullptr, cell_base);
    } else {
        r = stencil_ranges<LD>(px, py, pz, g.L, g.invL, g.halfL, g.G, nullptr, cc, lane, cap,
                               cell_base);
    }
    float md = fmul(mdf, ri);
    float cx = 0.f, cy = 0.f, cz = 0.f;
    for (int base = 0; base < r.total;) {  // warp-uniform
        // the chunk ends with the last stencil cell that ends within base + 32
        const unsigned int fit = __ballot_sync(0xffffffffu, lane < 27 && r.incl <= base + 32);
        const int end = __shfl_sync(0xffffffffu, r.incl, 31 - __clz(fit));
        const int t = base + lane;
        const int c = stencil_cell(r, t < r.total ? t : r.total - 1);  // same cell for t < end
        const int k = __shfl_sync(0xffffffffu, r.st, c) + (t - __shfl_sync(0xffffffffu, r.excl, c));
        bool hit = false;
        int key = 0;
        float vx = 0.f, vy = 0.f, vz = 0.f;
        if (t < end && k != kk) {
            const float4 q = LD::ld(&sp[k]);
            key = (c << 26) | LD::ld(&ci[k]);
            hit = pbd_term(q, px, py, pz, ri, md, gap1, g, vx, vy, vz);
        }
        warp_keyed_add3(hit, key, vx, vy, vz, cx, cy, cz);
        base = end;
    }
    if (lane == 0) {
        int i = LD::ld(&ci[kk]);
        const float3 n3 = pbd_move(px, py, pz, ri, cx, cy, cz, mdf, dmul, g);
        pout[3 * i + 0] = n3.x;
        pout[3 * i + 1] = n3.y;
        pout[3 * i + 2] = n3.z;
        if (np) *np = make_float4(n3.x, n3.y, n3.z, ri);
        return i;
    }
    return -1;
}

// Deepest overlap of candidate q below a particle at `me` (dynamics.py:330-345).
__device__ __forceinline__ float maxov_term(float4 q, float4 me, float eps, const GridGeom& g) {
    float ddx = grid_wrap(fsub(q.x, me.x), g.L, g.invL);
    float ddy = grid_wrap(fsub(q.y, me.y), g.L, g.invL);
    float ddz = grid_wrap(fsub(q.z, me.z), g.L, g.invL);
    float dist =
        __fsqrt_rn(fadd(fadd(fadd(fmul(ddx, ddx), fmul(ddy, ddy)), fmul(ddz, ddz)), eps));
    float td = fadd(me.w, q.w);
    return dist < td ? fsub(td, dist) : 0.f;
}

// compute_local_max_overlaps (dynamics.py:304-352) for the particle at
// sorted position kk (pairs i < j only); writes lmd[i] and returns the depth's
// float bits (non-negative floats order as their bits).  All 32 lanes.
// rmax > 0 (G >= 5; rmax the largest radius): only the cells that can hold a
// particle within ri + rmax, the only ones with a positive depth, are visited
// (stencil_ranges_near).
template <class LD>
__device__ __forceinline__ unsigned int maxov_warp(int kk, int lane, const float4* sp,
                                                   const int32_t* ci, const GridGeom g,
                                                   const int32_t* cs, const int32_t* cc, float eps,
                                                   float* lmd, int cap = 0, int cell_base = 0,
                                                   float rmax = 0.f, float cell_w = 0.f) {
    float4 me = LD::ld(&sp[kk]);
    int i = LD::ld(&ci[kk]);
    Stencil r;
    if (rmax > 0.f) {
        const float reach = (me.w + rmax) * 1.0001f;
        r = stencil_ranges_near<LD>(me.x, me.y, me.z, g, cell_w, cc, lane, cap, reach * reach,
                                    1e-5f * g.L + 1e-6f, cs, cell_base);
    } else {
        r = stencil_ranges<LD>(me.x, me.y, me.z, g.L, g.invL, g.halfL, g.G, cs, cc, lane, cap,
                               cell_base);
    }
    float lm = 0.f;
    for (int base = 0; base < r.total; base += 32) {
        int t = base + lane;
        int k = stencil_locate(r, t < r.total ? t : r.total - 1);
        if (t < r.total) {  // both loads before the test: one round trip
            const int j = LD::ld(&ci[k]);
            const float4 q = LD::ld(&sp[k]);
            if (i < j) lm = fmaxf(lm, maxov_term(q, me, eps, g));
        }
    }
    unsigned int b = __reduce_max_sync(0xffffffffu, __float_as_uint(lm));
    if (lane == 0) lmd[i] = __uint_as_float(b);
    return b;
}

// Powers of the pressure sweeps (dynamics.py:1504-1543: rad ** P_exp and
// V ** (1.0 / P_exp) with f32 P_exp, which Taichi's CPU backend evaluates with
// libm powf).  For PRESSURE_EXP = 3 (config.py:113) both are computed to the
// correctly rounded float, which glibc's powf returns for >99.9 % of these
// arguments (CUDA's powf differs from it more often):
//   x^3: the product in double (x^2 is exact; one rounding), then one
//   rounding to float;
//   y^invP, invP = f32(1/3) = 1/3 + 9.934107481e-9: cbrtf (within 1 ulp),
//   one Newton step in double (error ~2^-46), times
//   y^9.934e-9 = 1 + 9.934e-9 ln y (the next term is ~2^-47), rounded once.
// B200 runs FP64 at half the FP32 rate, so each costs a fraction of powf's
// instructions: the twenty barrier-free sweeps of a headline frame fell from
// 50.1 to 45.6 us.  Other exponents use powf.
__device__ __forceinline__ float pow_P(float x, float P) {
    if (P == 3.0f) {
        const double d = (double)x;
        return __double2float_rn(__dmul_rn(__dmul_rn(d, d), d));
    }
    return powf(x, P);
}

__device__ __forceinline__ float root_P(float y, float invP) {
    if (invP == 0.333333343f) {
        const float c = cbrtf(y);
        const double cd = (double)c;
        const double e = __dadd_rn(__dmul_rn(__dmul_rn(cd, cd), cd), -(double)y);
        const double inv = (double)__frcp_rn(fmul(3.0f, fmul(c, c)));
        const double cn = __dadd_rn(cd, -__dmul_rn(e, inv));
        const double k = __dmul_rn(9.934107481e-9, (double)__logf(y));
        return __double2float_rn(__dadd_rn(cn, __dmul_rn(cn, k)));
    }
    return powf(y, invP);
}

// hash_func (dynamics.py:1436-1451) in wrapping int32 arithmetic.
__device__ __forceinline__ int hash_func(int i, int frame) {
    unsigned int t = (unsigned int)i + 12345u * (unsigned int)frame;
    return (int)((1103515245u * t + 12345u) & 0x7fffffffu);
}

struct PressureArgs {
    int n, frame, max_nei;
    float k, P, cap, rmin, rmax;
    const int32_t* face_ids;
    const int32_t* fsc;
    int hoff;  // particle i hashes as i - hoff (its index within its own foam)
};

// equilibrate_pressure (dynamics.py:1454-1557) for particle i, one Jacobi
// sweep, by a group of GS lanes: lane t handles the t-th budgeted neighbour
// of the hashed rotation and the radius deltas are summed in neighbour order
// (the reference's serial accumulation).  Lane 0 of the group writes
// rout[i] and delta_r[i] and gets d back; all GS lanes of the group call it
// (i may be >= n: the group then does nothing).
template <int GS, class LD>
__device__ __forceinline__ float pressure_group(int i, int lane, const PressureArgs a,
                                                const float* rin, float* rout, float* delta_r) {
    int gl = lane & (GS - 1);
    unsigned int gmask = GS == 32 ? 0xffffffffu : (0xffffu << (lane & 16));
    bool live = i < a.n;
    float ri = live ? LD::ld(&rin[i]) : 0.f;
    int fc = live ? LD::ld(&a.fsc[i]) : 0;
    float d = 0.f;
    if (fc > 0) {
        int an = fc < a.max_nei ? fc : a.max_nei;
        int st = hash_func(i - a.hoff, a.frame) % fc;
        float Vi = pow_P(ri, a.P);
        float invP = fdiv(1.0f, a.P);
        for (int base = 0; base < an; base += GS) {
            int kk = base + gl;
            bool hit = false;
            float term = 0.f;
            if (kk < an) {
                int ni = (st + kk) % fc;
                int j = LD::ld(&a.face_ids[(size_t)i * FOS_S + ni]);
                if (!(j < 0 || j >= a.n || j == i)) {
                    float Vj = pow_P(LD::ld(&rin[j]), a.P);
                    float dvr = fmul(a.k, fsub(Vi, Vj));
                    float vmin = fminf(Vi, Vj);
                    float dv = fmaxf(fmul(-a.cap, vmin), fminf(fmul(a.cap, vmin), dvr));
                    term = fsub(root_P(fsub(Vi, dv), invP), ri);
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
        rout[i] = fmaxf(a.rmin, fminf(a.rmax, fadd(ri, d)));
    }
    return d;
}

// pressure_group for max_nei <= 16 with a group of 8 lanes: lane t handles
// the budgeted neighbours t and t + 8 at once (independent loads and powf),
// and the terms are summed in neighbour order 0..an-1 as in pressure_group,
// so the result is bit-identical.  The neighbour choice (fsc, face_ids, the
// hashed rotation) does not change within a frame, so it is split out
// (PressureNbr) and a caller may keep it in registers across the sweeps.
struct PressureNbr {
    int fc;       // fsc[i] (0: no neighbours, or i >= n)
    int j[2];     // neighbours t and t + 8 of this lane
    bool ok[2];   // whether each takes part (in budget, valid, not i)
};

template <class LD>
__device__ __forceinline__ PressureNbr pressure_nbr8x2(int i, int lane, const PressureArgs a) {
    PressureNbr nb;
    const int gl = lane & 7;
    nb.fc = i < a.n ? LD::ld(&a.fsc[i]) : 0;
    nb.j[0] = nb.j[1] = 0;
    nb.ok[0] = nb.ok[1] = false;
    if (nb.fc > 0) {
        const int an = nb.fc < a.max_nei ? nb.fc : a.max_nei;
        const int st = hash_func(i - a.hoff, a.frame) % nb.fc;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int kk = gl + 8 * h;
            if (kk < an) {
                const int ni = (st + kk) % nb.fc;
                const int j = LD::ld(&a.face_ids[(size_t)i * FOS_S + ni]);
                nb.j[h] = j;
                nb.ok[h] = !(j < 0 || j >= a.n || j == i);
            }
        }
    }
    return nb;
}

// The same for a group of NL lanes (NL divides 16): lane t of the group takes
// neighbours t, t + NL, t + 2 NL, ... of the hashed rotation.
template <int NL>
struct PressureNbrN {
    int fc;
    int j[16 / NL];
    bool ok[16 / NL];
};

template <int NL, class LD>
__device__ __forceinline__ PressureNbrN<NL> pressure_nbr_n(int i, int lane, const PressureArgs a) {
    PressureNbrN<NL> nb;
    const int gl = lane & (NL - 1);
    nb.fc = i < a.n ? LD::ld(&a.fsc[i]) : 0;
#pragma unroll
    for (int h = 0; h < 16 / NL; ++h) {
        nb.j[h] = 0;
        nb.ok[h] = false;
    }
    if (nb.fc > 0) {
        const int an = nb.fc < a.max_nei ? nb.fc : a.max_nei;
        const int st = hash_func(i - a.hoff, a.frame) % nb.fc;
#pragma unroll
        for (int h = 0; h < 16 / NL; ++h) {
            const int kk = gl + NL * h;
            if (kk < an) {
                const int ni = (st + kk) % nb.fc;
                const int j = LD::ld(&a.face_ids[(size_t)i * FOS_S + ni]);
                nb.j[h] = j;
                nb.ok[h] = !(j < 0 || j >= a.n || j == i);
            }
        }
    }
    return nb;
}

// pressure_sum8x2 for NL-lane groups (vj[h]: the power of neighbour h of this
// lane); the terms are added in neighbour order, so the sum is the same float.
template <int NL>
__device__ __forceinline__ float pressure_sum_n(const PressureArgs& a, const PressureNbrN<NL>& nb,
                                                int lane, float ri, float Vi, const float* vj) {
    constexpr int H = 16 / NL;
    const int base_lane = lane & (32 - NL);
    const unsigned int gmask = ((1u << NL) - 1u) << base_lane;
    const float invP = fdiv(1.0f, a.P);
    float term[H];
#pragma unroll
    for (int h = 0; h < H; ++h) {
        term[h] = 0.f;
        if (nb.ok[h]) {
            const float Vj = vj[h];
            const float dvr = fmul(a.k, fsub(Vi, Vj));
            const float vmin = fminf(Vi, Vj);
            const float dv = fmaxf(fmul(-a.cap, vmin), fminf(fmul(a.cap, vmin), dvr));
            term[h] = fsub(root_P(fsub(Vi, dv), invP), ri);
        }
    }
    float d = 0.f;
#pragma unroll
    for (int h = 0; h < H; ++h) {
        const unsigned int m = (__ballot_sync(gmask, nb.ok[h]) & gmask) >> base_lane;
        float v[NL];
#pragma unroll
        for (int t = 0; t < NL; ++t) v[t] = __shfl_sync(gmask, term[h], t, NL);
#pragma unroll
        for (int t = 0; t < NL; ++t)
            if ((m >> t) & 1u) d = fadd(d, v[t]);
    }
    return d;
}

template <class LD>
__device__ __forceinline__ float pressure_sweep8x2(int i, int lane, const PressureArgs a,
                                                   const PressureNbr& nb, const float* rin,
                                                   float* rout, float* delta_r) {
    const int gl = lane & 7;
    const int base_lane = lane & 24;
    const unsigned int gmask = 0xffu << base_lane;
    const bool live = i < a.n;
    const float ri = live ? LD::ld(&rin[i]) : 0.f;
    float d = 0.f;
    if (nb.fc > 0) {
        const float rj0 = nb.ok[0] ? LD::ld(&rin[nb.j[0]]) : 0.f;
        const float rj1 = nb.ok[1] ? LD::ld(&rin[nb.j[1]]) : 0.f;
        const float Vi = pow_P(ri, a.P);
        const float invP = fdiv(1.0f, a.P);
        float term[2] = {0.f, 0.f};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (nb.ok[h]) {
                const float Vj = pow_P(h == 0 ? rj0 : rj1, a.P);
                const float dvr = fmul(a.k, fsub(Vi, Vj));
                const float vmin = fminf(Vi, Vj);
                const float dv = fmaxf(fmul(-a.cap, vmin), fminf(fmul(a.cap, vmin), dvr));
                term[h] = fsub(root_P(fsub(Vi, dv), invP), ri);
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            unsigned int m = (__ballot_sync(gmask, nb.ok[h]) & gmask) >> base_lane;
            while (m) {
                const int b = __ffs(m) - 1;
                m &= m - 1;
                d = fadd(d, __shfl_sync(gmask, term[h], b, 8));
            }
        }
    }
    if (live && gl == 0) {
        delta_r[i] = d;
        rout[i] = fmaxf(a.rmin, fminf(a.rmax, fadd(ri, d)));
    }
    return d;
}

// pressure_sweep8x2 with the particle powers V = r^P carried between sweeps:
// vin[j] == pow_P(rin[j], P) for every j, so a neighbour costs one root (its
// new-radius term) instead of two, and lane 0 also writes vout[i] =
// pow_P(rout[i], P) for the next sweep (vout may be NULL).  The result is
// pressure_sweep8x2's bit for bit: the same powers of the same values.
// The radius delta of one 8-lane group's particle (radius ri, power Vi = ri^P)
// from its neighbours' powers vj0 / vj1 (lane t: neighbours t and t + 8 of
// the hashed rotation), summed in neighbour order; every lane of the group
// gets it.  Only called when nb.fc > 0 (uniform over the group).
__device__ __forceinline__ float pressure_sum8x2(const PressureArgs& a, const PressureNbr& nb,
                                                 int lane, float ri, float Vi, float vj0,
                                                 float vj1) {
    const int base_lane = lane & 24;
    const unsigned int gmask = 0xffu << base_lane;
    const float invP = fdiv(1.0f, a.P);
    float term[2] = {0.f, 0.f};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        if (nb.ok[h]) {
            const float Vj = h == 0 ? vj0 : vj1;
            const float dvr = fmul(a.k, fsub(Vi, Vj));
            const float vmin = fminf(Vi, Vj);
            const float dv = fmaxf(fmul(-a.cap, vmin), fminf(fmul(a.cap, vmin), dvr));
            term[h] = fsub(root_P(fsub(Vi, dv), invP), ri);
        }
    }
    // neighbour order: lanes 0..7 of the group for h = 0, then for h = 1; the
    // eight shuffles of each h are issued before the adds that consume them
    float d = 0.f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const unsigned int m = (__ballot_sync(gmask, nb.ok[h]) & gmask) >> base_lane;
        float v[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) v[t] = __shfl_sync(gmask, term[h], t, 8);
#pragma unroll
        for (int t = 0; t < 8; ++t)
            if ((m >> t) & 1u) d = fadd(d, v[t]);
    }
    return d;
}

template <class LD>
__device__ __forceinline__ float pressure_sweep8x2v(int i, int lane, const PressureArgs a,
                                                    const PressureNbr& nb, const float* rin,
                                                    const float* vin, float* rout, float* vout,
                                                    float* delta_r) {
    const int gl = lane & 7;
    const bool live = i < a.n;
    const float ri = live ? LD::ld(&rin[i]) : 0.f;
    float d = 0.f;
    if (nb.fc > 0) {
        const float Vi = LD::ld(&vin[i]);
        const float vj0 = nb.ok[0] ? LD::ld(&vin[nb.j[0]]) : 0.f;
        const float vj1 = nb.ok[1] ? LD::ld(&vin[nb.j[1]]) : 0.f;
        d = pressure_sum8x2(a, nb, lane, ri, Vi, vj0, vj1);
    }
    if (live && gl == 0) {
        delta_r[i] = d;
        const float rn = fmaxf(a.rmin, fminf(a.rmax, fadd(ri, d)));
        rout[i] = rn;
        if (vout) vout[i] = pow_P(rn, a.P);
    }
    return d;
}

// The budgeted neighbours of particle i for one frame's pressure sweeps, all
// sixteen slots at once: nbr[16 i + t] = neighbour t of the hashed rotation
// (pressure_nbr8x2's choice) or -1 where none takes part (past the budget,
// invalid, or i itself).  The choice does not change within a frame, so the
// sweeps then read one coalesced word per neighbour instead of fsc, the
// rotation and face_ids.  st < fc and t < an <= fc, so (st + t) % fc is
// st + t less fc once it reaches fc.  Needs max_nei <= 16.
template <class LD>
__device__ __forceinline__ void pressure_nbr_fill(int i, const PressureArgs& a, int32_t* nbr) {
    const int fc = LD::ld(&a.fsc[i]);
    const int an = fc > 0 ? (fc < a.max_nei ? fc : a.max_nei) : 0;
    const int st = fc > 0 ? hash_func(i - a.hoff, a.frame) % fc : 0;
    int v[16];
#pragma unroll
    for (int t = 0; t < 16; ++t) {
        v[t] = -1;
        if (t < an) {
            const int ni = st + t >= fc ? st + t - fc : st + t;
            const int j = LD::ld(&a.face_ids[(size_t)i * FOS_S + ni]);
            if (!(j < 0 || j >= a.n || j == i)) v[t] = j;
        }
    }
    int4* o = reinterpret_cast<int4*>(nbr + (size_t)i * 16);
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = make_int4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

// One 8-lane group's inputs of a pressure sweep from the frame's neighbour
// table (pressure_nbr_fill): lane t takes neighbours t and t + 8.  Loading
// two groups' inputs before either sum keeps two dependent chains in flight.
struct PressureIn {
    PressureNbr nb;
    float ri, Vi, vj0, vj1;
};

template <class LD>
__device__ __forceinline__ PressureIn pressure_in8x2n(int i, int lane, int n, const int32_t* nbr,
                                                      const float* rin, const float* vin) {
    PressureIn p;
    const int gl = lane & 7;
    const bool live = i < n;
    const int j0 = live ? LD::ld(&nbr[(size_t)i * 16 + gl]) : -1;
    const int j1 = live ? LD::ld(&nbr[(size_t)i * 16 + gl + 8]) : -1;
    p.ri = live ? LD::ld(&rin[i]) : 0.f;
    p.Vi = live ? LD::ld(&vin[i]) : 0.f;
    p.nb.fc = 1;
    p.nb.j[0] = j0;
    p.nb.j[1] = j1;
    p.nb.ok[0] = j0 >= 0;
    p.nb.ok[1] = j1 >= 0;
    p.vj0 = j0 >= 0 ? LD::ld(&vin[j0]) : 0.f;
    p.vj1 = j1 >= 0 ? LD::ld(&vin[j1]) : 0.f;
    return p;
}

// Loads of the table-driven pressure sweeps (pressure_in8x2n): L1-allocating
// (LdL1) or L2 only (LdL2).  The sweeps read what the sweep before wrote,
// behind a grid barrier whose acquire makes it visible to plain loads.
#ifndef PRESS_LD
#define PRESS_LD LdL1
#endif

// pressure_sweep8x2v's result from PressureIn: a group with no neighbour
// taking part sums nothing and gets +0, as when fsc[i] == 0.  Lane 0 of the
// group writes delta_r[i], rout[i] (clamped to [rmin, rmax]) and, with vout,
// the new power.  All 32 lanes.
__device__ __forceinline__ float pressure_out8x2n(int i, int lane, int n, const PressureArgs& a,
                                                  const PressureIn& p, float rmin, float rmax,
                                                  float* rout, float* vout, float* delta_r) {
    const float d = pressure_sum8x2(a, p.nb, lane, p.ri, p.Vi, p.vj0, p.vj1);
    if (i < n && (lane & 7) == 0) {
        delta_r[i] = d;
        const float rn = fmaxf(rmin, fminf(rmax, fadd(p.ri, d)));
        rout[i] = rn;
        if (vout) vout[i] = pow_P(rn, a.P);
    }
    return d;
}

template <class LD>
__device__ __forceinline__ float pressure_group8x2(int i, int lane, const PressureArgs a,
                                                   const float* rin, float* rout, float* delta_r) {
    const PressureNbr nb = pressure_nbr8x2<LD>(i, lane, a);
    return pressure_sweep8x2<LD>(i, lane, a, nb, rin, rout, delta_r);
}

// apply_brownian_motion (dynamics.py:1596-1634) for particle i.  ti.random()
// is replaced by Philox-4x32-10 with counter (ctr, frame, 'BROW', 0) and key =
// seed, ctr being i's index within its own foam; each axis draws
// u = (x >> 8) * 2^-24.
template <class LD>
__device__ __forceinline__ void brownian_one(int i, unsigned int ctr, float* pos, float strength,
                                             float domain, float halfL, uint32_t k0, uint32_t k1,
                                             unsigned int frame) {
    uint4 r = philox4x32_10(make_uint4(ctr, frame, 0x42524f57u, 0u), k0, k1);
    unsigned int rr[3] = {r.x, r.y, r.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float u = fmul((float)(rr[d] >> 8), 0x1p-24f);
        float dd = fmul(fmul(fsub(u, 0.5f), 2.0f), strength);
        float p = fadd(LD::ld(&pos[3 * i + d]), dd);
        if (p < -halfL) p = fadd(p, domain);
        else if (p >= halfL) p = fsub(p, domain);
        pos[3 * i + d] = p;
    }
}

// OU jitter (dynamics.py:607-660).  Constants the reference folds in Python
// (double) arrive folded and rounded once to float32:
//   tau   = max(1e-6, JITTER_TAU)
//   sq2   = sqrt(2 / max(1e-6, JITTER_TAU))
//   capk  = MAX_DRIFT_FRACTION * GAP_FRACTION
struct OuParams {
    float rms, sq2, tau, capk, dt, L, invL;
    uint32_t k0, k1;
};

static inline OuParams ou_params(double rms, double tau, double max_drift, double gap, float dt,
                                 float L, float invL, uint64_t seed) {
    const double t = tau > 1e-6 ? tau : 1e-6;
    OuParams o;
    o.rms = (float)rms;
    o.sq2 = (float)sqrt(2.0 / t);
    o.tau = (float)t;
    o.capk = (float)(max_drift * gap);
    o.dt = dt;
    o.L = L;
    o.invL = invL;
    o.k0 = (uint32_t)seed;
    o.k1 = (uint32_t)(seed >> 32);
    return o;
}

// Radius r as a 2^-40 fixed-point integer: exact for r in [2^-17, 2^23), so a
// sum of these is the exact sum of the radii in any order.
__device__ __forceinline__ long long rad_fixed(float r) {
    return __float2ll_rn(fmul(r, 0x1p40f));
}

// mean_radius from the fixed-point sum (the radii's exact mean rounded once
// to float32).
__device__ __forceinline__ float mean_from_fixed(unsigned long long sum, int n) {
    return (float)((double)(long long)sum * 0x1p-40 / (double)(n > 1 ? n : 1));
}

// sigma * sqrt(dt) of apply_brownian, from the mean radius.
__device__ __forceinline__ float ou_kick(const OuParams& o, float mean_r) {
    return fmul(fmul(fmul(o.rms, mean_r), o.sq2), __fsqrt_rn(o.dt));
}

// apply_brownian for particle i (counter index ctr) with kick = sigma *
// sqrt(dt): v += (-v / tau) * dt + kick * r, r = U[-0.5, 0.5)^3 from
// Philox-4x32-10 (ctr, frame, 'OUJT', 0); a step |v| dt above
// capk * (r_i + r_i) is scaled back to the cap.  Returns the new velocity.
__device__ __forceinline__ float3 ou_velocity(unsigned int ctr, float3 v, float r_i, float kick,
                                              const OuParams& o, unsigned int frame) {
    uint4 rr = philox4x32_10(make_uint4(ctr, frame, 0x4f554a54u, 0u), o.k0, o.k1);
    float ux = fsub(fmul((float)(rr.x >> 8), 0x1p-24f), 0.5f);
    float uy = fsub(fmul((float)(rr.y >> 8), 0x1p-24f), 0.5f);
    float uz = fsub(fmul((float)(rr.z >> 8), 0x1p-24f), 0.5f);
    v.x = fadd(v.x, fadd(fmul(fdiv(-v.x, o.tau), o.dt), fmul(kick, ux)));
    v.y = fadd(v.y, fadd(fmul(fdiv(-v.y, o.tau), o.dt), fmul(kick, uy)));
    v.z = fadd(v.z, fadd(fmul(fdiv(-v.z, o.tau), o.dt), fmul(kick, uz)));
    const float cap = fmul(o.capk, fadd(r_i, r_i));
    const float len = fmul(__fsqrt_rn(fadd(fadd(fmul(v.x, v.x), fmul(v.y, v.y)), fmul(v.z, v.z))),
                           o.dt);
    if (len > cap) {
        const float sc = fdiv(fdiv(cap, fmaxf(1e-6f, len)), o.dt);
        v.x = fmul(v.x, sc);
        v.y = fmul(v.y, sc);
        v.z = fmul(v.z, sc);
    }
    return v;
}

// integrate_jitter for one position: wrapP(p + v * dt) with grid.wrapP.
__device__ __forceinline__ float3 ou_move(float3 p, float3 v, const OuParams& o) {
    return make_float3(grid_wrap(fadd(p.x, fmul(v.x, o.dt)), o.L, o.invL),
                       grid_wrap(fadd(p.y, fmul(v.y, o.dt)), o.L, o.invL),
                       grid_wrap(fadd(p.z, fmul(v.z, o.dt)), o.L, o.invL));
}

// apply_brownian + integrate_jitter for particle i at position p: updates
// vjit[i] and returns the moved position.
__device__ __forceinline__ float3 ou_one(int i, unsigned int ctr, float3 p, float* vjit, float r_i,
                                         float kick, const OuParams& o, unsigned int frame) {
    float3 v = make_float3(__ldcg(&vjit[3 * i + 0]), __ldcg(&vjit[3 * i + 1]),
                           __ldcg(&vjit[3 * i + 2]));
    v = ou_velocity(ctr, v, r_i, kick, o, frame);
    vjit[3 * i + 0] = v.x;
    vjit[3 * i + 1] = v.y;
    vjit[3 * i + 2] = v.z;
    return ou_move(p, v, o);
}

// smoothstep (dynamics.py:1226-1240)
__device__ __forceinline__ float smoothstep(float e0, float e1, float x) {
    float t = fminf(1.0f, fmaxf(0.0f, fdiv(fsub(x, e0), fsub(e1, e0))));
    return fmul(fmul(t, t), fsub(3.0f, fmul(2.0f, t)));
}

// set_fsc_targets (dynamics.py:1242-1320) for particle i.
__device__ __forceinline__ float target_one(float r0, float e, int f_i, int f_low, int f_high,
                                            float growth, float rmin, float rmax, float db) {
    const float hg = 1.0f, idle = 0.003f;
    float f = e > 0.0f ? e : (float)f_i;
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
    return out;
}

// nudge_radii_adaptive_ema (dynamics.py:1366-1427) for particle i; b_global
// is the global backpressure (used in mode 1).
__device__ __forceinline__ float nudge_one(float r0, float rt_i, float lmd_i, float alpha,
                                           float max_step, float rmin, float rmax, float b_global,
                                           int mode, float contact_tol) {
    float r_t = fminf(rmax, fmaxf(rmin, rt_i));
    float d = fmul(alpha, fsub(r_t, r0));
    float b = 1.0f;
    if (mode == 1) b = b_global;
    else if (mode == 2) {
        b = fdiv(fsub(contact_tol, lmd_i), contact_tol);
        b = fminf(1.0f, fmaxf(0.25f, b));
    }
    d = fmul(d, b);
    float cap = fmul(max_step, r0);
    if (d > cap) d = cap;
    if (d < -cap) d = -cap;
    return fminf(rmax, fmaxf(rmin, fadd(r0, d)));
}

// backpressure_from_overlap (run.py:454-470), evaluated in double like the
// reference's host code, from the device max-overlap bits.
__device__ __forceinline__ float back_global_from_bits(unsigned int bits, double contact_tol) {
    if (!(contact_tol > 0)) return 1.0f;
    double om = (double)__uint_as_float(bits);
    double raw = (contact_tol - om) / contact_tol;
    return (float)fmax(0.25, fmin(1.0, raw));
}
