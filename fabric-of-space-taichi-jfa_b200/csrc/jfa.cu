// jfa.cu -- jump-flood power diagram and face-sharing-count extraction.
//
// Reference: jfa.py (VirtualOrganics/Fabric-of-Space-Taichi-JFA).  The result
// of every stage equals the reference's kernels run with serial semantics
// (each top-level loop in index order on one thread):
//   jfa_init            jfa.py:484-520  -> 64-bit atomicMin on (power distance, seed)
//   jfa_step_ping0/1    jfa.py:523-623  -> k_jfa_pass (int32 owner labels, ping-pong)
//   majority filter     jfa.py:639-699  -> k_majority
//   accumulate_face_area jfa.py:702-762 -> warp-aggregated pair table + first-touch order
//   finalize_faces      jfa.py:788-857  -> exact fixed point of the serial hysteresis
//   update_fsc_ema      jfa.py:765-785  -> fused into the finalize kernel
#include <math.h>
#include <string.h>

#include "fos_internal.cuh"

#define EMPTY_KEY 0xFFFFFFFFFFFFFFFFull

// ---------------------------------------------------------------- jfa_init
// world_to_voxel (jfa.py:254-270): floor(((p + 0.5L)/L) * R), wrapped.
__device__ __forceinline__ int world_to_voxel(float p, float halfL, float L, int R) {
    float nrm = fdiv(fadd(p, halfL), L);
    int v = (int)floorf(fmul(nrm, (float)R));
    return wrap_mod(v, R);
}

__global__ void k_seed_prepare(const float* __restrict__ pos, const float* __restrict__ rad, int n,
                               int R, float halfL, float L, float beta, float4* __restrict__ seeds,
                               int32_t* __restrict__ seedlin, unsigned long long* __restrict__ slot) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float px = pos[3 * i + 0], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    float br = fmul(beta, rad[i]);
    seeds[i] = make_float4(px, py, pz, fmul(br, br));
    int x = world_to_voxel(px, halfL, L, R);
    int y = world_to_voxel(py, halfL, L, R);
    int z = world_to_voxel(pz, halfL, L, R);
    int lin = (x * R + y) * R + z;
    seedlin[i] = lin;
    slot[lin] = ~0ull;
}

template <bool UNIT_L>
__global__ void k_seed_min(const float4* __restrict__ seeds, const int32_t* __restrict__ seedlin,
                           int n, int R, float vs, float halfL, float L,
                           unsigned long long* __restrict__ slot) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lin = seedlin[i];
    int z = lin % R, y = (lin / R) % R, x = lin / (R * R);
    float d = power_dist<UNIT_L>(voxel_centre(x, vs, halfL), voxel_centre(y, vs, halfL),
                                 voxel_centre(z, vs, halfL), seeds[i], L);
    unsigned long long key = ((unsigned long long)float_order_key(d) << 32) | (unsigned int)i;
    atomicMin(&slot[lin], key);
}

__global__ void k_seed_write(const int32_t* __restrict__ seedlin, int n,
                             const unsigned long long* __restrict__ slot,
                             int32_t* __restrict__ labels) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lin = seedlin[i];
    labels[lin] = (int32_t)(unsigned int)(slot[lin] & 0xFFFFFFFFull);
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
                                              FosDevState* ds, int pass) {
    const long long V = (long long)R * R * R;
    long long lin = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool live = lin < V;
    long long l = live ? lin : 0;
    int x, y, z;
    if (POW2) {
        z = (int)(l & (R - 1));
        y = (int)((l >> lgR) & (R - 1));
        x = (int)(l >> (2 * lgR));
    } else {
        z = (int)(l % R);
        y = (int)((l / R) % R);
        x = (int)(l / ((long long)R * R));
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
        float4 sv[9];
#pragma unroll
        for (int k = 0; k < 9; ++k)
            sv[k] = ok[k] ? __ldg(&seeds[ids[g * 9 + k]]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            int id = ids[g * 9 + k];
            float d = jfa_dist<UNIT_L>(vx, vy, vz, sv[k], L);
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
    if (threadIdx.x == 0 && cnt) atomicAdd(&ds->changes[pass], (unsigned long long)cnt);
}

template <bool UNIT_L, bool POW2, bool TIE_LOWER>
__global__ void __launch_bounds__(256) k_jfa_pass(const int32_t* __restrict__ in,
                                                  int32_t* __restrict__ out,
                                                  const float4* __restrict__ seeds, int R, int lgR,
                                                  float vs, float halfL, float L, int step,
                                                  FosDevState* ds, int pass, int early_exit,
                                                  int min_passes, double th) {
    const long long V = (long long)R * R * R;
    if (early_exit && jfa_exited_before(ds, pass, (double)V, min_passes, th)) return;
    jfa_pass_body<UNIT_L, POW2, TIE_LOWER>(in, out, seeds, R, lgR, vs, halfL, L, step, ds, pass);
}

__global__ void k_jfa_finish(FosDevState* ds, int passes, long long V, int early_exit,
                             int min_passes, double th) {
    int done = passes;
    int ex = 0;
    if (early_exit) {
        for (int q = 0; q < passes; ++q) {
            if (q >= min_passes - 1 && (double)ds->changes[q] / (double)V < th) {
                done = q + 1;
                ex = 1;
                break;
            }
        }
    }
    ds->passes_done = done;
    ds->early_exited = ex;
    ds->final_buf = done & 1;  // pass p writes buffer (p+1)&1
}

// Per-run reset of the face-pair counters (one launch instead of memsets).
__global__ void k_faces_reset(FosDevState* ds, int32_t* rowcnt, int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    for (int i = t; i < n; i += gridDim.x * blockDim.x) rowcnt[i] = 0;
    if (t == 0) {
        ds->pair_count = 0;
        ds->row_overflow = 0;
        ds->max_rowcnt = 0;
    }
}

__global__ void k_fin_reset(FosDevState* ds, int* fin_changed, int32_t* revcnt, int32_t* revfill,
                            int n) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int stride = gridDim.x * blockDim.x;
    for (int i = t; i < n; i += stride) {
        revcnt[i] = 0;
        revfill[i] = 0;
    }
    for (int i = t; i < FOS_FIN_MAXIT; i += stride) fin_changed[i] = 0;
    if (t == 0) {
        revcnt[n] = 0;
        ds->zero_fsc = 0;
        ds->fin_iters = 0;
        ds->bar_count = 0;
        ds->bar_gen = 0;
    }
}

// ------------------------------------------------------------ majority filter
// majority_filter_labels (jfa.py:639-699): tally the centre (count 1) then the
// six face neighbours, axis 0..2 x dir (-1, +1); the first label in insertion
// order with the strictly greatest count wins; -1 stays -1.
__global__ void __launch_bounds__(256) k_majority(const int32_t* __restrict__ labA,
                                                  const int32_t* __restrict__ labB,
                                                  const FosDevState* __restrict__ ds, int R,
                                                  int32_t* __restrict__ outp) {
    const int32_t* lab = ds->final_buf ? labB : labA;
    long long V = (long long)R * R * R;
    long long lin = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (lin >= V) return;
    int z = (int)(lin % R), y = (int)((lin / R) % R), x = (int)(lin / ((long long)R * R));
    int me = lab[lin];
    if (me < 0) {
        outp[lin] = -1;
        return;
    }
    int nb[6];
    nb[0] = lab[((long long)wrap_small(x - 1, R) * R + y) * R + z];
    nb[1] = lab[((long long)wrap_small(x + 1, R) * R + y) * R + z];
    nb[2] = lab[((long long)x * R + wrap_small(y - 1, R)) * R + z];
    nb[3] = lab[((long long)x * R + wrap_small(y + 1, R)) * R + z];
    nb[4] = lab[((long long)x * R + y) * R + wrap_small(z - 1, R)];
    nb[5] = lab[((long long)x * R + y) * R + wrap_small(z + 1, R)];
    int ids[7], cnt[7], nu = 1;
    ids[0] = me;
    cnt[0] = 1;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        int id = nb[k];
        if (id >= 0) {
            bool found = false;
#pragma unroll
            for (int u = 0; u < 7; ++u)
                if (!found && u < nu && ids[u] == id) {
                    cnt[u]++;
                    found = true;
                }
            if (!found) {
#pragma unroll
                for (int u = 0; u < 7; ++u)
                    if (u == nu) {
                        ids[u] = id;
                        cnt[u] = 1;
                    }
                nu++;
            }
        }
    }
    int mc = 0, best = me;
#pragma unroll
    for (int u = 0; u < 7; ++u)
        if (u < nu && cnt[u] > mc) {
            mc = cnt[u];
            best = ids[u];
        }
    outp[lin] = best;
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

__device__ __forceinline__ void pair_insert(unsigned long long pk, unsigned int fk, unsigned int c,
                                            unsigned long long* keys, unsigned int* hmin,
                                            unsigned int* hcnt, unsigned int* claimed,
                                            FosDevState* ds, unsigned long long mask) {
    unsigned long long h = fmix64(pk) & mask;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
        unsigned long long k = keys[h];
        bool hit = (k == pk);
        if (!hit && k == EMPTY_KEY) {
            unsigned long long prev = atomicCAS(&keys[h], EMPTY_KEY, pk);
            if (prev == EMPTY_KEY) {
                int idx = atomicAdd(&ds->pair_count, 1);
                claimed[idx] = (unsigned int)h;
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
__global__ void __launch_bounds__(256) k_faces(const int32_t* __restrict__ filt, int R, int n,
                                               unsigned long long* keys, unsigned int* hmin,
                                               unsigned int* hcnt, unsigned int* claimed,
                                               FosDevState* ds, unsigned long long mask) {
    long long V = (long long)R * R * R;
    long long lin = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool live = lin < V;
    int lane = threadIdx.x & 31;
    int a = live ? filt[lin] : -1;
    bool va = a >= 0 && a < n;
    int z = 0, y = 0, x = 0;
    if (live) {
        z = (int)(lin % R);
        y = (int)((lin / R) % R);
        x = (int)(lin / ((long long)R * R));
    }
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        long long nlin = 0;
        if (live) {
            if (ax == 0) nlin = ((long long)wrap_small(x + 1, R) * R + y) * R + z;
            else if (ax == 1) nlin = ((long long)x * R + wrap_small(y + 1, R)) * R + z;
            else nlin = ((long long)x * R + y) * R + wrap_small(z + 1, R);
        }
        int b = va ? filt[nlin] : -1;
        bool valid = va && b >= 0 && b < n && b != a;
        unsigned long long pk = 0;
        unsigned int fk = 0;
        if (valid) {
            int lo = a < b ? a : b, hi = a < b ? b : a;
            pk = ((unsigned long long)(unsigned int)lo << 32) | (unsigned int)hi;
            fk = (a < b) ? (unsigned int)(lin * 6 + ax * 2 + 1) : (unsigned int)(nlin * 6 + ax * 2);
        }
        unsigned int m = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            unsigned int grp = __match_any_sync(m, pk);
            unsigned int mn = __reduce_min_sync(grp, fk);
            if (lane == __ffs(grp) - 1) pair_insert(pk, mn, __popc(grp), keys, hmin, hcnt, claimed, ds, mask);
        }
    }
}

// Moves every claimed pair into its lower particle's candidate row and resets
// the table slot for the next run.
__global__ void k_compact(unsigned long long* keys, unsigned int* hmin, unsigned int* hcnt,
                          const unsigned int* __restrict__ claimed, FosDevState* ds,
                          int32_t* rowcnt, uint4* rowbuf) {
    int total = ds->pair_count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        unsigned int h = claimed[t];
        unsigned long long pk = keys[h];
        unsigned int fk = hmin[h], c = hcnt[h];
        keys[h] = EMPTY_KEY;
        hmin[h] = 0xFFFFFFFFu;
        hcnt[h] = 0u;
        int a = (int)(pk >> 32);
        unsigned int b = (unsigned int)(pk & 0xFFFFFFFFull);
        int p = atomicAdd(&rowcnt[a], 1);
        if (p < FOS_ROWCAP) rowbuf[(size_t)a * FOS_ROWCAP + p] = make_uint4(fk, b, c, 0u);
        else if (p == FOS_ROWCAP) {
            atomicAdd(&ds->row_overflow, 1);
            atomicCAS(&ds->error, 0, (int)FOS_E_CAPACITY);
        }
    }
}

// Slot order of face_ids[a] = ascending first-touch key; the first 32 partners
// get slots, later ones are dropped as the reference's slot search drops them.
__global__ void k_rows(int n, const int32_t* __restrict__ rowcnt, const uint4* __restrict__ rowbuf,
                       int32_t* __restrict__ face_ids, int32_t* __restrict__ face_counts,
                       FosDevState* ds) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    int m = rowcnt[a];
    if (m > 0) atomicMax(&ds->max_rowcnt, m);
    if (m > FOS_ROWCAP) m = FOS_ROWCAP;
    uint4 e[FOS_ROWCAP];
    for (int k = 0; k < m; ++k) {
        uint4 v = rowbuf[(size_t)a * FOS_ROWCAP + k];
        int j = k - 1;
        while (j >= 0 && e[j].x > v.x) {
            e[j + 1] = e[j];
            --j;
        }
        e[j + 1] = v;
    }
    for (int s = 0; s < FOS_S; ++s) {
        size_t o = (size_t)a * FOS_S + s;
        face_ids[o] = s < m ? (int)e[s].y : -1;
        face_counts[o] = s < m ? (int)e[s].z : 0;
    }
}

// Per face slot: the normalised score of finalize_faces_kernel with
// expected_area (jfa.py:378-397, 810-830); -1 marks a slot the reference skips
// (partner outside [0, n), no voxels, or expected <= 0).  Also seeds the
// acceptance fixed point with "score >= T_ADD" and counts each partner's
// incoming lower pairs.
__global__ void k_scores(int n, const int32_t* __restrict__ face_ids,
                         const int32_t* __restrict__ face_counts, const float* __restrict__ rad,
                         float vs, float face_scale, float t_add, float* __restrict__ score,
                         uint8_t* acc, int32_t* revcnt) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * FOS_S) return;
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

__global__ void k_rev_fill(int n, const int32_t* __restrict__ face_ids,
                           const float* __restrict__ score, const int32_t* __restrict__ revstart,
                           int32_t* revfill, int32_t* __restrict__ rev) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * FOS_S) return;
    if (score[t] < 0.0f) return;
    int j = face_ids[t];
    int p = atomicAdd(&revfill[j], 1);
    rev[revstart[j] + p] = (int)t;  // encodes (a, s) as a*32 + s
}

__global__ void k_rev_sort(int n, const int32_t* __restrict__ revstart, int32_t* __restrict__ rev) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int b = revstart[j], e = revstart[j + 1];
    for (int k = b + 1; k < e; ++k) {
        int v = rev[k];
        int q = k - 1;
        while (q >= b && rev[q] > v) {
            rev[q + 1] = rev[q];
            --q;
        }
        rev[q + 1] = v;
    }
}

// ------------------------------------------------------------ finalize
// Serial semantics of finalize_faces_kernel: particles in index order, each
// scanning its 32 face slots; an accepted pair appends to BOTH neighbour lists
// (add_neighbor, jfa.py:400-443, writing the score at the neighbour-list
// slot), a rejected one zeroes neighbor_prev_scores at the FACE slot, and the
// hysteresis test reads neighbor_prev_scores at the face slot.  So particle
// i's decisions depend on the pairs (a, i), a < i, accepted before it.
//
// Each sweep recomputes every decision from the previous sweep's decisions of
// lower rows (Jacobi).  Row i depends only on rows a < i, so rows are final
// after (1 + dependency depth) sweeps and a sweep with no change is the unique
// fixed point, which equals the serial result.
__device__ __forceinline__ int fin_row(int i, const int32_t* __restrict__ revstart,
                                       const int32_t* __restrict__ rev,
                                       const uint8_t* acc_in, uint8_t* acc_out,
                                       const float* __restrict__ score, const float* __restrict__ prev,
                                       float t_add, float t_drop) {
    float app[FOS_S];
    int used = 0;
    int b = revstart[i], e = revstart[i + 1];
    for (int k = b; k < e; ++k) {
        int t = rev[k];
        if (__ldcg(&acc_in[t]) && used < FOS_S) app[used++] = score[t];
    }
    int changed = 0;
    for (int s = 0; s < FOS_S; ++s) {
        size_t o = (size_t)i * FOS_S + s;
        float sc = score[o];
        uint8_t ok = 0;
        if (sc >= 0.0f) {
            float pr = (s < used) ? app[s] : prev[o];
            ok = (sc >= t_add) || (pr >= t_drop && sc >= t_drop);
            if (ok && used < FOS_S) app[used++] = sc;
        }
        if (ok != __ldcg(&acc_in[o])) changed = 1;
        __stcg(&acc_out[o], ok);
    }
    return changed;
}

__global__ void __launch_bounds__(256) k_finalize(int n, const int32_t* __restrict__ revstart,
                                                  const int32_t* __restrict__ rev,
                                                  uint8_t* acc0, uint8_t* acc1,
                                                  const float* __restrict__ score,
                                                  const int32_t* __restrict__ face_ids,
                                                  float* prev, int32_t* nl, int32_t* used_out,
                                                  int32_t* fsc, float* ema, float t_add,
                                                  float t_drop, float alpha, int apply_ema,
                                                  FosDevState* ds, int* fin_changed,
                                                  int max_iters) {
    int stride = gridDim.x * blockDim.x;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint8_t* cur = acc0;
    uint8_t* nxt = acc1;
    int it = 0;
    unsigned int epoch = 0;
    for (;;) {
        int ch = 0;
        for (int i = tid; i < n; i += stride)
            ch |= fin_row(i, revstart, rev, cur, nxt, score, prev, t_add, t_drop);
        if (__syncthreads_or(ch) && threadIdx.x == 0) atomicOr(&fin_changed[it], 1);
        if (!grid_barrier(ds, epoch)) return;
        int any = *((volatile int*)&fin_changed[it]);
        uint8_t* t = cur;
        cur = nxt;
        nxt = t;
        ++it;
        if (!any) break;
        if (it >= max_iters) {
            if (tid == 0) atomicCAS(&ds->error, 0, (int)FOS_E_TIMEOUT);
            return;
        }
    }
    if (tid == 0) ds->fin_iters = it;
    // Materialise the serial result from the converged decisions `cur`.
    for (int i = tid; i < n; i += stride) {
        float pr[FOS_S];
        int used = 0;
        size_t row = (size_t)i * FOS_S;
#pragma unroll
        for (int s = 0; s < FOS_S; ++s) pr[s] = prev[row + s];
        int b = revstart[i], e = revstart[i + 1];
        for (int k = b; k < e; ++k) {
            int t = rev[k];
            if (__ldcg(&cur[t]) && used < FOS_S) {
                nl[row + used] = t >> 5;
                pr[used] = score[t];
                used++;
            }
        }
        for (int s = 0; s < FOS_S; ++s) {
            float sc = score[row + s];
            if (sc < 0.0f) continue;
            if (__ldcg(&cur[row + s])) {
                if (used < FOS_S) {
                    nl[row + used] = face_ids[row + s];
                    pr[used] = sc;
                    used++;
                }
            } else {
                pr[s] = 0.0f;
            }
        }
        for (int s = used; s < FOS_S; ++s) nl[row + s] = -1;
#pragma unroll
        for (int s = 0; s < FOS_S; ++s) prev[row + s] = pr[s];
        used_out[i] = used;
        fsc[i] = used;
        if (apply_ema) {  // update_fsc_ema (jfa.py:765-785)
            float em = ema[i];
            if (em == 0.0f && used > 0) em = (float)used;
            else em = fadd(fmul(alpha, (float)used), fmul(fsub(1.0f, alpha), em));
            ema[i] = em;
        }
        if (used == 0) atomicAdd(&ds->zero_fsc, 1);
    }
}

// Standalone EMA (for callers that run the stages one by one).
__global__ void k_ema(int n, const int32_t* __restrict__ fsc, float* ema, float alpha) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float em = ema[i];
    int f = fsc[i];
    if (em == 0.0f && f > 0) em = (float)f;
    else em = fadd(fmul(alpha, (float)f), fmul(fsub(1.0f, alpha), em));
    ema[i] = em;
}

// ------------------------------------------------------------ host side
static bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

static int ilog2(int v) {
    int r = 0;
    while ((1 << r) < v) ++r;
    return r;
}

static int check_n(FosCtx* c, int n) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(n >= 0 && n <= c->max_n, FOS_E_CAPACITY, "n outside [0, max_n]");
    return FOS_OK;
}

extern "C" int fos_jfa_init(FosCtx* c, const float* pos, const float* rad, int n, fos_stream_t s) {
    int rc = check_n(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (pos && rad), FOS_E_ARG, "pos/rad is NULL");
    const int R = c->res;
    size_t V = (size_t)R * R * R;
    FOS_CUDA(cudaMemsetAsync(c->labA, 0xFF, V * 4, s));
    if (n == 0) return FOS_OK;
    int nb = fos_blocks(n, 256);
    k_seed_prepare<<<nb, 256, 0, s>>>(pos, rad, n, R, c->halfL, c->L, c->beta, c->seeds, c->cellof,
                                      c->seedslot);
    FOS_LAUNCHED(c);
    if (c->L == 1.0f)
        k_seed_min<true><<<nb, 256, 0, s>>>(c->seeds, c->cellof, n, R, c->vs, c->halfL, c->L, c->seedslot);
    else
        k_seed_min<false><<<nb, 256, 0, s>>>(c->seeds, c->cellof, n, R, c->vs, c->halfL, c->L, c->seedslot);
    FOS_LAUNCHED(c);
    k_seed_write<<<nb, 256, 0, s>>>(c->cellof, n, c->seedslot, c->labA);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

template <bool UL, bool P2, bool TIE>
static void launch_pass(FosCtx* c, const int32_t* in, int32_t* out, int step, int pass,
                        cudaStream_t s) {
    const int R = c->res;
    long long V = (long long)R * R * R;
    k_jfa_pass<UL, P2, TIE><<<fos_blocks(V, 256), 256, 0, s>>>(
        in, out, c->seeds, R, ilog2(R), c->vs, c->halfL, c->L, step, c->ds, pass, c->p.early_exit,
        c->p.min_jfa_passes, c->p.th_pass_delta);
}

extern "C" int fos_jfa_passes(FosCtx* c, int n, fos_stream_t s) {
    int rc = check_n(c, n);
    if (rc) return rc;
    const int R = c->res;
    long long V = (long long)R * R * R;
    FOS_CUDA(cudaMemsetAsync(c->ds->changes, 0, sizeof(c->ds->changes), s));
    bool ul = (c->L == 1.0f), p2 = is_pow2(R), tie = c->p.tie_lower_index != 0;
    int step = R / 2;
    for (int p = 0; p < c->passes; ++p) {
        if (step < 1) step = 1;
        const int32_t* in = (p & 1) ? c->labB : c->labA;
        int32_t* out = (p & 1) ? c->labA : c->labB;
        if (ul && p2 && !tie) launch_pass<true, true, false>(c, in, out, step, p, s);
        else if (ul && p2 && tie) launch_pass<true, true, true>(c, in, out, step, p, s);
        else if (ul && !p2 && !tie) launch_pass<true, false, false>(c, in, out, step, p, s);
        else if (ul && !p2 && tie) launch_pass<true, false, true>(c, in, out, step, p, s);
        else if (!ul && p2 && !tie) launch_pass<false, true, false>(c, in, out, step, p, s);
        else if (!ul && p2 && tie) launch_pass<false, true, true>(c, in, out, step, p, s);
        else if (!ul && !p2 && !tie) launch_pass<false, false, false>(c, in, out, step, p, s);
        else launch_pass<false, false, true>(c, in, out, step, p, s);
        FOS_LAUNCHED(c);
        step /= 2;
    }
    k_jfa_finish<<<1, 1, 0, s>>>(c->ds, c->passes, V, c->p.early_exit, c->p.min_jfa_passes,
                                 c->p.th_pass_delta);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_jfa_load_labels(FosCtx* c, const int32_t* labels, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr && labels != nullptr, FOS_E_ARG, "NULL argument");
    size_t V = (size_t)c->res * c->res * c->res;
    FOS_CUDA(cudaMemcpyAsync(c->labA, labels, V * 4, cudaMemcpyDeviceToDevice, s));
    FOS_CUDA(cudaMemsetAsync(&c->ds->final_buf, 0, sizeof(int), s));
    return FOS_OK;
}

extern "C" int fos_jfa_majority_filter(FosCtx* c, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    long long V = (long long)c->res * c->res * c->res;
    k_majority<<<fos_blocks(V, 256), 256, 0, s>>>(c->labA, c->labB, c->ds, c->res, c->filt);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_jfa_accumulate_faces(FosCtx* c, int n, fos_stream_t s) {
    int rc = check_n(c, n);
    if (rc) return rc;
    if (n == 0) return FOS_OK;
    long long V = (long long)c->res * c->res * c->res;
    k_faces_reset<<<fos_blocks(n, 256), 256, 0, s>>>(c->ds, c->rowcnt, n);
    FOS_LAUNCHED(c);
    k_faces<<<fos_blocks(V, 256), 256, 0, s>>>(c->filt, c->res, n, c->hkeys, c->hmin, c->hcnt,
                                               c->claimed, c->ds, (unsigned long long)(c->H - 1));
    FOS_LAUNCHED(c);
    k_compact<<<c->num_sms * 4, 256, 0, s>>>(c->hkeys, c->hmin, c->hcnt, c->claimed, c->ds,
                                             c->rowcnt, c->rowbuf);
    FOS_LAUNCHED(c);
    k_rows<<<fos_blocks(n, 256), 256, 0, s>>>(n, c->rowcnt, c->rowbuf, c->face_ids, c->face_counts,
                                              c->ds);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

static int finalize_impl(FosCtx* c, const float* rad, int n, bool apply_ema, cudaStream_t s) {
    int nb = fos_blocks(n, 256);
    k_fin_reset<<<nb, 256, 0, s>>>(c->ds, c->fin_changed, c->revcnt, c->revfill, n);
    FOS_LAUNCHED(c);
    k_scores<<<fos_blocks((long long)n * FOS_S, 256), 256, 0, s>>>(
        n, c->face_ids, c->face_counts, rad, c->vs, c->face_scale, c->t_add, c->face_score, c->acc0,
        c->revcnt);
    FOS_LAUNCHED(c);
    int rc = fos_scan_exclusive(c, c->revcnt, c->revstart, n, true, s);
    if (rc) return rc;
    k_rev_fill<<<fos_blocks((long long)n * FOS_S, 256), 256, 0, s>>>(n, c->face_ids, c->face_score,
                                                                     c->revstart, c->revfill, c->rev);
    FOS_LAUNCHED(c);
    k_rev_sort<<<nb, 256, 0, s>>>(n, c->revstart, c->rev);
    FOS_LAUNCHED(c);
    int per_sm = 0;
    FOS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_finalize, 256, 0));
    int grid = nb;
    int cap = per_sm * c->num_sms;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    int max_it = n + 2 < FOS_FIN_MAXIT ? n + 2 : FOS_FIN_MAXIT;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FOS_CUDA(cudaLaunchKernelEx(&cfg, k_finalize, n, (const int32_t*)c->revstart,
                                (const int32_t*)c->rev, c->acc0, c->acc1,
                                (const float*)c->face_score, (const int32_t*)c->face_ids, c->prev,
                                c->nl, c->used, c->fsc, c->ema, c->t_add, c->t_drop, c->ema_alpha,
                                apply_ema ? 1 : 0, c->ds, c->fin_changed, max_it));
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// finalize_faces_kernel alone (reads face_ids/face_counts, rad, prev scores).
extern "C" int fos_jfa_finalize(FosCtx* c, const float* rad, int n, fos_stream_t s) {
    int rc = check_n(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || rad, FOS_E_ARG, "rad is NULL");
    if (n == 0) return FOS_OK;
    return finalize_impl(c, rad, n, false, s);
}

extern "C" int fos_jfa_update_ema(FosCtx* c, int n, fos_stream_t s) {
    int rc = check_n(c, n);
    if (rc) return rc;
    if (n == 0) return FOS_OK;
    k_ema<<<fos_blocks(n, 256), 256, 0, s>>>(n, c->fsc, c->ema, c->ema_alpha);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// finalize_faces_kernel + update_fsc_ema, the EMA fused into the
// materialisation of each particle's new fsc (what run_jfa does).
int fos_jfa_finalize_ema(FosCtx* c, const float* rad, int n, cudaStream_t s) {
    if (n == 0) return FOS_OK;
    return finalize_impl(c, rad, n, true, s);
}

extern "C" int fos_jfa_run(FosCtx* c, const float* pos, const float* rad, int n, fos_stream_t s) {
    int rc = fos_jfa_init(c, pos, rad, n, s);
    if (rc) return rc;
    rc = fos_jfa_passes(c, n, s);
    if (rc) return rc;
    rc = fos_jfa_majority_filter(c, s);
    if (rc) return rc;
    rc = fos_jfa_accumulate_faces(c, n, s);
    if (rc) return rc;
    if (n == 0) return FOS_OK;
    // finalize_faces_kernel + update_fsc_ema, the EMA fused into the
    // materialisation of each particle's new fsc.
    return finalize_impl(c, rad, n, true, s);
}
