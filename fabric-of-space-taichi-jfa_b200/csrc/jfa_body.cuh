// jfa_body.cuh -- per-voxel / per-slot device bodies of the JFA and FSC
// stages.  The single-foam kernels (jfa.cu) and the batched-ensemble kernels
// (ensemble.cu) call the same bodies, so each stage's arithmetic exists once;
// a body takes its element index instead of reading blockIdx.
//
// Reference: jfa.py (VirtualOrganics/Fabric-of-Space-Taichi-JFA).
#pragma once

#include "fos_internal.cuh"

#define EMPTY_KEY 0xFFFFFFFFFFFFFFFFull

// ---------------------------------------------------------------- jfa_init
// world_to_voxel (jfa.py:254-270): floor(((p + 0.5L)/L) * R), wrapped.
__device__ __forceinline__ int world_to_voxel(float p, float halfL, float L, int R) {
    float nrm = fdiv(fadd(p, halfL), L);
    int v = (int)floorf(fmul(nrm, (float)R));
    return wrap_mod(v, R);
}

// ------------------------------------------------------------ JFA pass
// True when the reference's early exit (jfa.py:1108-1112) fired after some
// pass q < p: q >= MIN_JFA_PASSES-1 and changes[q]/V < TH_PASS_DELTA.
__device__ __forceinline__ bool jfa_exited_before(const FosDevState* ds, int p, double V,
                                                  int min_passes, double th) {
    for (int q = min_passes - 1; q < p; ++q)
        if (q >= 0 && (double)ds->changes[q] / V < th) return true;
    return false;
}

// One pass: own label first (1e10 when unassigned), then the 27 offsets in
// lexicographic (dx, dy, dz) order, dz fastest, each times `step` and wrapped;
// a candidate replaces the best only on a strictly smaller power distance.
// A candidate whose label equals the voxel's own label or the label of the
// previous offset in scan order is skipped: that label's distance has already
// been compared, so it cannot win again and the result is unchanged.
//
// One thread per voxel, z fastest, so each of the 27 label loads of a warp is
// one coalesced 128-byte row.  All 27 labels are loaded up front; the seed
// gathers are then issued nine at a time (one dx plane) independently of the
// running minimum, so a voxel waits for three rounds of gather latency rather
// than one per evaluated candidate.  A plane no lane of the warp needs is
// skipped with one vote.
template <bool UNIT_L>
__device__ __forceinline__ float jfa_dist(float vx, float vy, float vz, float4 s, float L) {
    if (!UNIT_L) return power_dist<false>(vx, vy, vz, s, L);
    return power_dist_unit(vx, vy, vz, s);
}

template <bool UNIT_L, bool POW2, bool TIE_LOWER>
__device__ __forceinline__ void jfa_pass_body(const int32_t* __restrict__ in,
                                              int32_t* __restrict__ out,
                                              const float4* __restrict__ seeds, int R, int lgR,
                                              float vs, float halfL, float L, int step,
                                              unsigned long long* changes, int pass,
                                              long long lin) {
    const long long V = (long long)R * R * R;
    bool live = lin < V;
    long long l = live ? lin : 0;
    int x, y, z;
    if (POW2) {
        z = (int)(l & (R - 1));
        y = (int)((l >> lgR) & (R - 1));
        x = (int)(l >> (2 * lgR));
    } else {  // 32-bit: R <= 512
        const int l32 = (int)l;
        z = l32 % R;
        const int t = l32 / R;
        y = t % R;
        x = t / R;
    }
    int xs[3], ys[3], zs[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int o = (k - 1) * step;
        if (POW2) {
            xs[k] = ((x + o) & (R - 1)) << (2 * lgR);
            ys[k] = ((y + o) & (R - 1)) << lgR;
            zs[k] = (z + o) & (R - 1);
        } else {
            xs[k] = wrap_small(x + o, R) * R * R;
            ys[k] = wrap_small(y + o, R) * R;
            zs[k] = wrap_small(z + o, R);
        }
    }
    int ids[27];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) ids[a * 9 + b * 3 + c] = in[xs[a] + ys[b] + zs[c]];
    int own = live ? ids[13] : -1;  // offset (0,0,0) is the voxel itself
    float vx = voxel_centre(x, vs, halfL), vy = voxel_centre(y, vs, halfL),
          vz = voxel_centre(z, vs, halfL);
    int best = own;
    float bd = 1e10f;
    if (own >= 0) bd = jfa_dist<UNIT_L>(vx, vy, vz, __ldg(&seeds[own]), L);
    const float2 vxy = make_float2(vx, vy);
#pragma unroll
    for (int g = 0; g < 3; ++g) {
        bool ok[9];
        bool any = false;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            int idx = g * 9 + k;
            int id = ids[idx];
            int prv = idx == 0 ? own : ids[idx - 1];
            ok[k] = live && id >= 0 && id != own && id != prv;
            any |= ok[k];
        }
        if (!__any_sync(0xffffffffu, any)) continue;
        // a skipped candidate loads seed 0 (a cached line) and its distance
        // is ignored, so the loads need no predicate or fill
        float4 sv[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) sv[k] = __ldg(&seeds[ok[k] ? ids[g * 9 + k] : 0]);
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            int id = ids[g * 9 + k];
            float d = UNIT_L ? power_dist_unit2(vxy, vz, sv[k])
                             : jfa_dist<false>(vx, vy, vz, sv[k], L);
            if (ok[k] && (d < bd || (TIE_LOWER && d == bd && id < best))) {
                bd = d;
                best = id;
            }
        }
    }
    int changed = 0;
    if (live) {
        out[lin] = best;
        changed = best != own;
    }
    // one atomic per block: same-address atomics from every warp serialise in L2
    int cnt = __syncthreads_count(changed);
    if (threadIdx.x == 0 && cnt) atomicAdd(&changes[pass], (unsigned long long)cnt);
}

// ------------------------------------------------- JFA pass over records
// The owner grid is mirrored by a record grid: record v = the seed
// (x, y, z, (beta r)^2) of label v, or all-ones bits (NaN) for an unassigned
// voxel.  A pass then reads each candidate's seed as part of a coalesced
// 512-byte row of records instead of a label followed by a 16-byte gather per
// lane (the gathers were ~12 L1 data-pipe wavefronts each and held the pass on
// L1 throughput).  A NaN record's distance is NaN, and every comparison with
// NaN is false, so an unassigned candidate never wins and an unassigned
// voxel's own distance falls back to 1e10 through fminf, as in the reference.
__device__ __forceinline__ float4 rec_none() {
    const float q = __int_as_float(-1);
    return make_float4(q, q, q, q);
}

// One pass over records with the reference's rule: own label first (1e10 when
// unassigned), then the 27 offsets in lexicographic (dx, dy, dz) order, a
// candidate replacing the best only on a strictly smaller power distance.  The
// winner is tracked by its voxel index, and its label and record are read once
// at the end.  The distance of a candidate with the voxel's own label equals
// the own distance, so it can never replace it and no label is needed per
// candidate; offset (0, 0, 0) is the voxel itself and is not re-evaluated.
template <bool UNIT_L>
__device__ __forceinline__ void jfa_rec_core(const int32_t* __restrict__ in,
                                             const float4* __restrict__ rin,
                                             int32_t* __restrict__ out,
                                             float4* __restrict__ rout, float vs, float halfL,
                                             float L, unsigned long long* changes, int pass,
                                             int l, bool live, int x, int y, int z,
                                             const int (&xs)[3], const int (&ys)[3],
                                             const int (&zs)[3]) {
    const int own = in[l];
    const float4 orec = __ldg(&rin[l]);
    const float vx = voxel_centre(x, vs, halfL), vy = voxel_centre(y, vs, halfL),
                vz = voxel_centre(z, vs, halfL);
    const float2 vxy = make_float2(vx, vy);
    float bd = fminf(UNIT_L ? power_dist_unit2m(vxy, vz, orec)
                            : jfa_dist<false>(vx, vy, vz, orec, L), 1e10f);
    int bl = l;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int idx[9];
        float4 r[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            idx[k] = xs[a] + ys[k / 3] + zs[k % 3];
            if (!(a == 1 && k == 4)) r[k] = __ldg(&rin[idx[k]]);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            if (a == 1 && k == 4) continue;  // the voxel itself
            const float d = UNIT_L ? power_dist_unit2m(vxy, vz, r[k])
                                   : jfa_dist<false>(vx, vy, vz, r[k], L);
            if (d < bd) {
                bd = d;
                bl = idx[k];
            }
        }
    }
    int best = own;
    float4 brec = orec;
    if (bl != l) {
        best = in[bl];
        brec = __ldg(&rin[bl]);
    }
    int changed = 0;
    if (live) {
        out[l] = best;
        rout[l] = brec;
        changed = best != own;
    }
    int cnt = __syncthreads_count(changed);
    if (threadIdx.x == 0 && cnt) atomicAdd(&changes[pass], (unsigned long long)cnt);
}

template <bool UNIT_L, bool POW2>
__device__ __forceinline__ void jfa_pass_rec_body(const int32_t* __restrict__ in,
                                                  const float4* __restrict__ rin,
                                                  int32_t* __restrict__ out,
                                                  float4* __restrict__ rout, int R, int lgR,
                                                  float vs, float halfL, float L, int step,
                                                  unsigned long long* changes, int pass,
                                                  long long lin) {
    const int V = R * R * R;  // R <= 512, so V < 2^31
    const bool live = lin < V;
    const int l = live ? (int)lin : 0;
    int x, y, z;
    if (POW2) {
        z = l & (R - 1);
        y = (l >> lgR) & (R - 1);
        x = l >> (2 * lgR);
    } else {
        z = l % R;
        const int t = l / R;
        y = t % R;
        x = t / R;
    }
    int xs[3], ys[3], zs[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int o = (k - 1) * step;
        if (POW2) {
            xs[k] = ((x + o) & (R - 1)) << (2 * lgR);
            ys[k] = ((y + o) & (R - 1)) << lgR;
            zs[k] = (z + o) & (R - 1);
        } else {
            xs[k] = wrap_small(x + o, R) * R * R;
            ys[k] = wrap_small(y + o, R) * R;
            zs[k] = wrap_small(z + o, R);
        }
    }
    jfa_rec_core<UNIT_L>(in, rin, out, rout, vs, halfL, L, changes, pass, l, live, x, y, z, xs,
                         ys, zs);
}

// The same pass for a grid whose R is known only at run time (the batched
// ensembles mix power-of-two and other resolutions in one launch): the
// coordinates come from shifts or divisions by a block-uniform branch, the
// wraps from compare-and-add (|x + o| < 2R since step <= R/2), and the
// candidate loop is shared, so the kernel holds one copy of it.
template <bool UNIT_L>
__device__ __forceinline__ void jfa_pass_rec_body_any(const int32_t* __restrict__ in,
                                                      const float4* __restrict__ rin,
                                                      int32_t* __restrict__ out,
                                                      float4* __restrict__ rout, int R, int lgR,
                                                      bool pow2, float vs, float halfL, float L,
                                                      int step, unsigned long long* changes,
                                                      int pass, long long lin) {
    const int V = R * R * R;
    const bool live = lin < V;
    const int l = live ? (int)lin : 0;
    int x, y, z;
    if (pow2) {
        z = l & (R - 1);
        y = (l >> lgR) & (R - 1);
        x = l >> (2 * lgR);
    } else {
        z = l % R;
        const int t = l / R;
        y = t % R;
        x = t / R;
    }
    const int RR = R * R;
    int xs[3], ys[3], zs[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int o = (k - 1) * step;
        xs[k] = wrap_small(x + o, R) * RR;
        ys[k] = wrap_small(y + o, R) * R;
        zs[k] = wrap_small(z + o, R);
    }
    jfa_rec_core<UNIT_L>(in, rin, out, rout, vs, halfL, L, changes, pass, l, live, x, y, z, xs,
                         ys, zs);
}

// The candidate scan of M voxels at x-planes 1..M of xp[] (offsets of the
// M + 2 planes, y rows ys[], z offsets zs[]) that share y and z: the 9 rows of
// each plane are read once, in increasing plane and (dy, dz) order, and each
// row updates the voxels it serves (dx = plane - m - 1 in {-1, 0, 1}, less
// the voxel itself) with power_dist_unit2m's floats (pdist_yz2m once per
// row, pdist_x2m / pdist_x1m per voxel).  bd / bl hold each voxel's best
// distance and voxel index, started from its own record.
//
// HALF (the step is R / 2): on every axis the offsets -step and +step reach
// the same voxel, and -1 comes first in the scan order, so a candidate with
// any +1 offset repeats an earlier one: the same record, the same distance,
// which a strict < never takes.  Only the offsets {-1, 0}^3 are scanned then
// (7 candidates besides the voxel itself instead of 26); the result is the
// full scan's.
template <int M, bool HALF = false>
__device__ __forceinline__ bool recx_serves(int p, int m, int k) {
    const int dx = p - m;  // the candidate's x offset + 1
    if (HALF) return dx >= 0 && dx <= 1 && k / 3 <= 1 && k % 3 <= 1 && !(dx == 1 && k == 4);
    return dx >= 0 && dx <= 2 && !(dx == 1 && k == 4);
}

template <int M, bool HALF = false>
__device__ __forceinline__ void recx_scan(const float4* __restrict__ rin, const int (&xp)[M + 2],
                                          const int (&ys)[3], const int (&zs)[3],
                                          const float (&vx)[M], float vy, float vz,
                                          float (&bd)[M], int (&bl)[M]) {
#pragma unroll
    for (int p = 0; p < M + 2; ++p) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            // voxels m with dx = p - m - 1 in {-1, 0, 1}, less the voxel itself
            bool used = false;
#pragma unroll
            for (int m = 0; m < M; ++m)
                if (recx_serves<M, HALF>(p, m, k)) used = true;
            if (!used) continue;
            const int idx = xp[p] + ys[k / 3] + zs[k % 3];
            const float4 r = __ldg(&rin[idx]);
            // the voxels this row serves (at most three), y and z terms once,
            // the x terms of two voxels in a packed pair
            int vm[3] = {0, 0, 0}, nv = 0;
#pragma unroll
            for (int m = 0; m < M; ++m)
                if (recx_serves<M, HALF>(p, m, k)) vm[nv++] = m;
            const float2 qyz = pdist_yz2m(make_float2(vy, vz), r);
            float dv[3];
            if (nv >= 2) {
                const float2 d2 = pdist_x2m(make_float2(vx[vm[0]], vx[vm[1]]), qyz, r);
                dv[0] = d2.x;
                dv[1] = d2.y;
                if (nv == 3) dv[2] = pdist_x1m(vx[vm[2]], qyz, r);
            } else {
                dv[0] = pdist_x1m(vx[vm[0]], qyz, r);
            }
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (q >= nv) break;
                if (dv[q] < bd[vm[q]]) {
                    bd[vm[q]] = dv[q];
                    bl[vm[q]] = idx;
                }
            }
        }
    }
}

// Voxel coordinates of linear index l (z fastest) in 32-bit arithmetic
// (R <= 512, so R^3 < 2^31): shifts for a power-of-two R, else divisions.
__device__ __forceinline__ void vox_xyz(int l, int R, int& x, int& y, int& z) {
    if ((R & (R - 1)) == 0) {
        const int lg = __ffs(R) - 1;
        z = l & (R - 1);
        y = (l >> lg) & (R - 1);
        x = l >> (2 * lg);
    } else {
        z = l % R;
        const int t = l / R;
        y = t % R;
        x = t / R;
    }
}

// One voxel of the majority filter: lab is the final owner grid of R^3.
__device__ __forceinline__ void majority_body(const int32_t* __restrict__ lab, int R,
                                              int32_t* __restrict__ outp, long long lin) {
    const int V = R * R * R;
    if (lin >= V) return;
    const int l = (int)lin;
    int x, y, z;
    vox_xyz(l, R, x, y, z);
    int me = lab[l];
    if (me < 0) {
        outp[l] = -1;
        return;
    }
    int nb[6];
    nb[0] = lab[(wrap_small(x - 1, R) * R + y) * R + z];
    nb[1] = lab[(wrap_small(x + 1, R) * R + y) * R + z];
    nb[2] = lab[(x * R + wrap_small(y - 1, R)) * R + z];
    nb[3] = lab[(x * R + wrap_small(y + 1, R)) * R + z];
    nb[4] = lab[(x * R + y) * R + wrap_small(z - 1, R)];
    nb[5] = lab[(x * R + y) * R + wrap_small(z + 1, R)];
    // The most frequent label among me and the six neighbours (unassigned
    // neighbours do not count), ties to the first seen in the order me, nb[0],
    // ..., nb[5]: the reference's insertion-order count, as 21 pairwise
    // comparisons.  A later copy of a label has the same count as its first
    // copy, so the strict '>' keeps the first.
    int v[7] = {me, nb[0], nb[1], nb[2], nb[3], nb[4], nb[5]};
    int c[7] = {1, 1, 1, 1, 1, 1, 1};
#pragma unroll
    for (int a = 0; a < 7; ++a)
#pragma unroll
        for (int b = a + 1; b < 7; ++b) {
            const int e = v[a] == v[b] ? 1 : 0;
            c[a] += e;
            c[b] += e;
        }
    int mc = 0, best = me;
#pragma unroll
    for (int k = 0; k < 7; ++k)
        if (v[k] >= 0 && c[k] > mc) {
            mc = c[k];
            best = v[k];
        }
    outp[l] = best;
}

// ------------------------------------------------------------ face pairs
// murmur3 fmix64 (Austin Appleby, public domain)
__device__ __forceinline__ unsigned long long fmix64(unsigned long long k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

// Where a claimed pair-table slot goes: gathered in shared memory and appended
// to the table's claimed list with one atomic per block (faces_claims_flush).
// One counter shared by every claim serialises in L2: at 200,000 particles
// (1.4 M pairs) the face kernel took 1.73 ms with an atomic per claim and
// 0.99 ms with one per block.
struct ClaimBuf {
    unsigned int* slot;  // >= 3 * blockDim.x entries
    int* n;
    unsigned int* claimed;
};

// Insert (or find) pair key pk in the open-addressed table and add its
// count c and first-touch key fk.  h is the pair's home slot and k the key
// already loaded from it (the caller issues the first probes of a warp's
// three axes together).
__device__ __forceinline__ void pair_insert_at(unsigned long long pk, unsigned int fk,
                                               unsigned int c, unsigned long long h,
                                               unsigned long long k, unsigned long long* keys,
                                               unsigned int* hmin, unsigned int* hcnt,
                                               const ClaimBuf& cb, FosDevState* ds,
                                               unsigned long long mask) {
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
        bool hit = (k == pk);
        if (!hit && k == EMPTY_KEY) {
            unsigned long long prev = atomicCAS(&keys[h], EMPTY_KEY, pk);
            if (prev == EMPTY_KEY) {
                cb.slot[atomicAdd(cb.n, 1)] = (unsigned int)h;
                hit = true;
            } else {
                hit = (prev == pk);
            }
        }
        if (hit) {
            atomicMin(&hmin[h], fk);
            atomicAdd(&hcnt[h], c);
            return;
        }
        h = (h + 1) & mask;
        k = keys[h];
    }
    atomicCAS(&ds->error, 0, (int)FOS_E_CAPACITY);
}

// accumulate_face_area (jfa.py:702-762).  Each geometric voxel face is visited
// once (the +1 face of every voxel, wrapped).  A face between labels a != b,
// both in [0, n), belongs to the pair lo = min(a,b), hi = max(a,b); the serial
// reference visits it from the lower-label voxel, so its first-touch key is
// (that voxel's linear index)*6 + axis*2 + (dir == +1).  Lanes of a warp that
// hit the same pair are merged (__match_any_sync) before one atomic update of
// the pair's count and minimum first-touch key.
//
// Element lin is a thread slot, not a voxel: when R is a multiple of 8 each
// warp (32 consecutive slots) takes a 2 (x) x 2 (y) x 8 (z) voxel tile, whose
// four z-rows are whole 32-byte sectors.  A tile meets fewer distinct pairs
// per axis than a 32-voxel z-run (cells are a few voxels across), so fewer
// merged groups reach the table.  The count and the minimum key of a pair do
// not depend on which thread visits which face, so the result is the same.
__device__ __forceinline__ void faces_body(const int32_t* __restrict__ filt, int R, int n,
                                           unsigned long long* keys, unsigned int* hmin,
                                           unsigned int* hcnt, const ClaimBuf& cb,
                                           FosDevState* ds, unsigned long long mask,
                                           long long lin) {
    const int V = R * R * R;
    bool live = lin < V;
    const int s = live ? (int)lin : 0;
    int lane = threadIdx.x & 31;
    int z, y, x;
    if ((R & 7) == 0) {  // V is then a multiple of 32: whole tiles only
        const int w = s >> 5, tz = R >> 3, ty = R >> 1;
        const int t = w / tz;
        z = ((w - t * tz) << 3) + (s & 7);
        y = ((t % ty) << 1) + ((s >> 3) & 1);
        x = ((t / ty) << 1) + ((s >> 4) & 1);
    } else {
        vox_xyz(s, R, x, y, z);
    }
    const int l = (x * R + y) * R + z;
    // the voxel's label and its three +1 neighbours' labels are loaded
    // together (every index is in range, live or not)
    int nlin[3], b[3];
    nlin[0] = (wrap_small(x + 1, R) * R + y) * R + z;
    nlin[1] = (x * R + wrap_small(y + 1, R)) * R + z;
    nlin[2] = (x * R + y) * R + wrap_small(z + 1, R);
    const int a = live ? filt[l] : -1;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) b[ax] = filt[nlin[ax]];
    bool va = a >= 0 && a < n;
    unsigned long long pk[3];
    unsigned int mn[3], cntv[3];
    bool lead[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const bool valid = va && b[ax] >= 0 && b[ax] < n && b[ax] != a;
        pk[ax] = 0;
        unsigned int fk = 0;
        if (valid) {
            int lo = a < b[ax] ? a : b[ax], hi = a < b[ax] ? b[ax] : a;
            pk[ax] = ((unsigned long long)(unsigned int)lo << 32) | (unsigned int)hi;
            fk = (a < b[ax]) ? (unsigned int)l * 6u + (unsigned int)(ax * 2 + 1)
                             : (unsigned int)nlin[ax] * 6u + (unsigned int)(ax * 2);
        }
        lead[ax] = false;
        mn[ax] = 0;
        cntv[ax] = 0;
        unsigned int m = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            unsigned int grp = __match_any_sync(m, pk[ax]);
            mn[ax] = __reduce_min_sync(grp, fk);
            cntv[ax] = __popc(grp);
            lead[ax] = lane == __ffs(grp) - 1;
        }
    }
    // first probes of the (up to) three inserts together, then each insert
    unsigned long long h[3], k[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        h[ax] = fmix64(pk[ax]) & mask;
        k[ax] = lead[ax] ? keys[h[ax]] : 0ull;
    }
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
        if (lead[ax])
            pair_insert_at(pk[ax], mn[ax], cntv[ax], h[ax], k[ax], keys, hmin, hcnt, cb, ds,
                           mask);
}

// faces_body with a second merge per block (R a multiple of 8): block blk takes
// a (2 FACES_TILE_WX) x (2 FACES_TILE_WY) x 8 voxel tile made of
// FACES_TILE_WX x FACES_TILE_WY warp tiles of 2 x 2 x 8 (default 4 x 8 x 8,
// eight warps).  Each warp merges its lanes' pairs as faces_body does; the
// warps' merged groups then meet in a shared-memory table (count sum, minimum
// first-touch key), and each distinct pair of the tile makes one update of
// the global table, so a pair whose faces span several warps of the tile
// probes the global table once instead of once per warp.  A group that finds
// the shared table full goes to the global table directly.  Counts are sums
// and keys minima, so the table ends as faces_body leaves it.  cb.n must be
// zeroed before the call (the first barrier here publishes it).
#ifndef FACES_TILE_WX
#define FACES_TILE_WX 2  // warp tiles along x (2 voxels each)
#endif
#ifndef FACES_TILE_WY
#define FACES_TILE_WY 4  // warp tiles along y (2 voxels each)
#endif
// R a multiple of 8 then tiles the grid: 2 WX and 2 WY divide 8
static_assert(8 % (2 * FACES_TILE_WX) == 0 && 8 % (2 * FACES_TILE_WY) == 0,
              "face tile sides must divide 8");
#define FACES_TILE_THREADS (32 * FACES_TILE_WX * FACES_TILE_WY)
#define FACES_TILE_SLOTS FACES_TILE_THREADS  // shared-table slots (a power of two)
__device__ __forceinline__ void faces_tile_body(const int32_t* __restrict__ filt, int R, int n,
                                                unsigned long long* keys, unsigned int* hmin,
                                                unsigned int* hcnt, const ClaimBuf& cb,
                                                FosDevState* ds, unsigned long long mask,
                                                int blk) {
    __shared__ unsigned long long s_key[FACES_TILE_SLOTS];
    __shared__ unsigned int s_min[FACES_TILE_SLOTS], s_cnt[FACES_TILE_SLOTS];
    for (int t = threadIdx.x; t < FACES_TILE_SLOTS; t += blockDim.x) {
        s_key[t] = EMPTY_KEY;
        s_min[t] = 0xFFFFFFFFu;
        s_cnt[t] = 0u;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nbz = R >> 3, nby = R / (2 * FACES_TILE_WY);
    const int bz = blk % nbz, t1 = blk / nbz, by = t1 % nby, bx = t1 / nby;
    const int z = (bz << 3) + (lane & 7);
    const int y = by * (2 * FACES_TILE_WY) + (w / FACES_TILE_WX) * 2 + ((lane >> 3) & 1);
    const int x = bx * (2 * FACES_TILE_WX) + (w % FACES_TILE_WX) * 2 + ((lane >> 4) & 1);
    const int l = (x * R + y) * R + z;
    int nlin[3], b[3];
    nlin[0] = (wrap_small(x + 1, R) * R + y) * R + z;
    nlin[1] = (x * R + wrap_small(y + 1, R)) * R + z;
    nlin[2] = (x * R + y) * R + wrap_small(z + 1, R);
    const int a = filt[l];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) b[ax] = filt[nlin[ax]];
    const bool va = a >= 0 && a < n;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const bool valid = va && b[ax] >= 0 && b[ax] < n && b[ax] != a;
        unsigned long long pk = 0;
        unsigned int fk = 0;
        if (valid) {
            const int lo = a < b[ax] ? a : b[ax], hi = a < b[ax] ? b[ax] : a;
            pk = ((unsigned long long)(unsigned int)lo << 32) | (unsigned int)hi;
            fk = (a < b[ax]) ? (unsigned int)l * 6u + (unsigned int)(ax * 2 + 1)
                             : (unsigned int)nlin[ax] * 6u + (unsigned int)(ax * 2);
        }
        const unsigned int m = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const unsigned int grp = __match_any_sync(m, pk);
            const unsigned int mn = __reduce_min_sync(grp, fk);
            if (lane == __ffs(grp) - 1) {
                const unsigned int c = __popc(grp);
                unsigned int hs = (unsigned int)fmix64(pk) & (FACES_TILE_SLOTS - 1);
                bool done = false;
                for (int p = 0; p < FACES_TILE_SLOTS; ++p) {
                    const unsigned long long prev = atomicCAS(&s_key[hs], EMPTY_KEY, pk);
                    if (prev == EMPTY_KEY || prev == pk) {
                        atomicMin(&s_min[hs], mn);
                        atomicAdd(&s_cnt[hs], c);
                        done = true;
                        break;
                    }
                    hs = (hs + 1) & (FACES_TILE_SLOTS - 1);
                }
                if (!done) {
                    const unsigned long long h = fmix64(pk) & mask;
                    pair_insert_at(pk, mn, c, h, keys[h], keys, hmin, hcnt, cb, ds, mask);
                }
            }
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < FACES_TILE_SLOTS; t += blockDim.x) {
        const unsigned long long pk = s_key[t];
        if (pk != EMPTY_KEY) {
            const unsigned long long h = fmix64(pk) & mask;
            pair_insert_at(pk, s_min[t], s_cnt[t], h, keys[h], keys, hmin, hcnt, cb, ds, mask);
        }
    }
}

// A faces kernel block's gathered claims: call with every thread of the block
// after faces_body; cb.n was zeroed (and synchronised) before it.
__device__ __forceinline__ void faces_claims_flush(const ClaimBuf& cb, unsigned int* claimed,
                                                   FosDevState* ds) {
    __shared__ int s_base;
    __syncthreads();
    const int m = *cb.n;
    if (threadIdx.x == 0) s_base = m ? atomicAdd(&ds->pair_count, m) : 0;
    __syncthreads();
    for (int t = threadIdx.x; t < m; t += blockDim.x) claimed[s_base + t] = cb.slot[t];
}

// Per face slot t = a*32 + s: the normalised score of finalize_faces_kernel
// with expected_area (jfa.py:378-397, 810-830); -1 marks a slot the reference
// skips (partner outside [0, n), no voxels, or expected <= 0).  Also seeds the
// acceptance fixed point with "score >= T_ADD" and counts each partner's
// incoming lower pairs.
__device__ __forceinline__ void score_slot(long long t, int n, const int32_t* __restrict__ face_ids,
                                           const int32_t* __restrict__ face_counts,
                                           const float* __restrict__ rad, float vs, float face_scale,
                                           float t_add, float* __restrict__ score, uint8_t* acc,
                                           int32_t* revcnt) {
    int a = (int)(t >> 5);
    int j = face_ids[t];
    int cnt = face_counts[t];
    float sc = -1.0f;
    if (j >= 0 && j < n && cnt > 0) {
        float rm = fmul(0.5f, fadd(rad[a], rad[j]));
        float q = fdiv(fmul(2.0f, rm), vs);
        float expected = fmul(face_scale, fmul(q, q));
        if (expected > 0.0f) sc = fdiv((float)cnt, expected);
    }
    score[t] = sc;
    acc[t] = (sc >= 0.0f && sc >= t_add) ? 1 : 0;
    if (sc >= 0.0f) atomicAdd(&revcnt[j], 1);
}
