/*
 * fos_oracle.c -- CPU restatement of the foam simulator's per-frame hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA library is
 * compared against; it is never linked into, loaded by, or called from the
 * product path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.
 *
 * PARITY UNPINNED against the reference itself: the reference is Python with
 * Taichi kernels (taichi>=1.7.0, unpinned, not vendored), Taichi cannot be
 * installed in this environment, and the reference ships no golden vectors or
 * known-answer tests.  The restatement is instead pinned by analytic
 * known-answer tests (tests/test_oracle_kat.py) and by the reference's own
 * runtime invariants (CSR sum, symmetric neighbour lists, no self loops).
 *
 * Semantics: "serial semantics" -- the result the reference's Taichi kernels
 * give when every top-level loop runs in index order on one thread.  All FP32
 * expressions follow the reference's operator order with no FMA contraction
 * (build with -ffp-contract=off, no fast-math).  Python-scope constants that
 * Taichi folds are folded in double and rounded to float once, by the caller.
 *
 * Deviations, each stated where it occurs:
 *   - project_overlaps is restated as a Jacobi sweep (read a snapshot, write a
 *     new buffer); the reference's in-place atomic update is scheduling
 *     dependent.
 *   - ti.random() is replaced by Philox-4x32-10 (Salmon et al., SC'11) keyed by
 *     (seed, frame, particle) so the Brownian jitter is an identical input.
 *   - ti.round() is taken as round-half-away-from-zero (roundf).
 *
 * Layout: voxel (x, y, z) lives at linear index (x*R + y)*R + z, z fastest,
 * which is also Taichi's ti.ndrange(R, R, R) iteration order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_S 32 /* MAX_NEIGHBORS, jfa.py:74 */

static inline int wrapi(int v, int R) { return ((v % R) + R) % R; }

/* ---------------------------------------------------------------- JFA helpers
 * jfa.wrapP (jfa.py:290-308): d - L*round(d/L), per component. */
static inline float jfa_wrap(float d, float L) { return d - L * roundf(d / L); }

/* power_distance_sq (jfa.py:450-477): |wrapP(v-p)|^2 - (beta*r)^2 */
static inline float power_dist(float vx, float vy, float vz, const float* p, float r,
                               float L, float beta) {
    float dx = jfa_wrap(vx - p[0], L);
    float dy = jfa_wrap(vy - p[1], L);
    float dz = jfa_wrap(vz - p[2], L);
    float d2 = dx * dx + dy * dy + dz * dz;
    float br = beta * r;
    return d2 - br * br;
}

/* voxel_to_world (jfa.py:273-287): (idx + 0.5)*VOXEL_SIZE - 0.5*L */
static inline float v2w(int idx, float vs, float halfL) { return ((float)idx + 0.5f) * vs - halfL; }

/* world_to_voxel (jfa.py:254-270): floor(((p + 0.5L)/L) * R), wrapped */
static inline int w2v(float p, float halfL, float L, int R) {
    float nrm = (p + halfL) / L;
    int v = (int)floorf(nrm * (float)R);
    return wrapi(v, R);
}

/* jfa_init (jfa.py:484-520).  Serial semantics: seed i in index order; a later
 * seed replaces the occupant only on a strictly smaller power distance at the
 * voxel centre.  labels[] must hold R^3 entries; all are reset to -1. */
void orc_jfa_init(const float* pos, const float* rad, int n, int R, float L, float halfL,
                  float vs, float beta, int32_t* labels) {
    size_t V = (size_t)R * R * R;
    for (size_t k = 0; k < V; ++k) labels[k] = -1;
    for (int i = 0; i < n; ++i) {
        int x = w2v(pos[3 * i + 0], halfL, L, R);
        int y = w2v(pos[3 * i + 1], halfL, L, R);
        int z = w2v(pos[3 * i + 2], halfL, L, R);
        size_t lin = ((size_t)x * R + y) * R + z;
        int cur = labels[lin];
        if (cur == -1) {
            labels[lin] = i;
        } else {
            float wx = v2w(x, vs, halfL), wy = v2w(y, vs, halfL), wz = v2w(z, vs, halfL);
            float dc = power_dist(wx, wy, wz, pos + 3 * cur, rad[cur], L, beta);
            float dn = power_dist(wx, wy, wz, pos + 3 * i, rad[i], L, beta);
            if (dn < dc) labels[lin] = i;
        }
    }
}

/* jfa_step_ping0/1 (jfa.py:523-623): one jump-flood pass.  Own label first
 * (distance 1e10 when unassigned), then the 27 offsets (dx,dy,dz) in
 * lexicographic order, dz fastest, each scaled by step and wrapped; replace on
 * strictly smaller power distance.  tie_lower: optional rule that breaks exact
 * distance ties toward the lower seed index instead of scan order.
 * Returns the number of voxels whose label changed. */
long long orc_jfa_pass(const int32_t* in, int32_t* out, const float* pos, const float* rad,
                       int R, float L, float halfL, float vs, float beta, int step,
                       int tie_lower) {
    long long changes = 0;
#pragma omp parallel for schedule(static) reduction(+ : changes)
    for (int x = 0; x < R; ++x) {
        for (int y = 0; y < R; ++y) {
            for (int z = 0; z < R; ++z) {
                size_t lin = ((size_t)x * R + y) * R + z;
                float wx = v2w(x, vs, halfL), wy = v2w(y, vs, halfL), wz = v2w(z, vs, halfL);
                int best = in[lin];
                float bd = 1e10f;
                if (best >= 0) bd = power_dist(wx, wy, wz, pos + 3 * best, rad[best], L, beta);
                for (int dx = -1; dx <= 1; ++dx)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dz = -1; dz <= 1; ++dz) {
                            int nx = wrapi(x + dx * step, R);
                            int ny = wrapi(y + dy * step, R);
                            int nz = wrapi(z + dz * step, R);
                            int id = in[((size_t)nx * R + ny) * R + nz];
                            if (id >= 0) {
                                float d = power_dist(wx, wy, wz, pos + 3 * id, rad[id], L, beta);
                                if (d < bd || (tie_lower && d == bd && id < best)) {
                                    bd = d;
                                    best = id;
                                }
                            }
                        }
                out[lin] = best;
                if (best != in[lin]) changes++;
            }
        }
    }
    return changes;
}

/* run_jfa pass schedule (jfa.py:1082-1116): step R/2, R/4, ..., clamped to 1
 * for the remaining passes; optional early exit after pass index >=
 * min_passes-1 when changes/V < th.  The result is copied into labels_out.
 * changes_out[p] receives the change count of pass p.  Returns passes run. */
int orc_jfa_run(const float* pos, const float* rad, int n, int R, float L, float halfL,
                float vs, float beta, int num_passes, int early_exit, int min_passes,
                double th_delta, int tie_lower, int32_t* labels_out, int32_t* scratch,
                long long* changes_out) {
    orc_jfa_init(pos, rad, n, R, L, halfL, vs, beta, labels_out);
    int32_t* a = labels_out;
    int32_t* b = scratch;
    int step = R / 2;
    int done = 0;
    size_t V = (size_t)R * R * R;
    for (int p = 0; p < num_passes; ++p) {
        if (step < 1) step = 1;
        long long ch = orc_jfa_pass(a, b, pos, rad, R, L, halfL, vs, beta, step, tie_lower);
        if (changes_out) changes_out[p] = ch;
        int32_t* t = a; a = b; b = t;
        step /= 2;
        done++;
        double frac = (double)ch / (double)(V > 0 ? V : 1);
        if (early_exit && p >= min_passes - 1 && frac < th_delta) break;
    }
    if (a != labels_out) memcpy(labels_out, a, V * sizeof(int32_t));
    return done;
}

/* majority_filter_labels (jfa.py:639-699): tally centre (count 1) then the six
 * face neighbours in order axis 0..2 x dir (-1,+1); the first label in
 * insertion order with the strictly greatest count wins; -1 stays -1. */
void orc_majority_filter(const int32_t* lab, int R, int32_t* out) {
#pragma omp parallel for schedule(static)
    for (int x = 0; x < R; ++x)
        for (int y = 0; y < R; ++y)
            for (int z = 0; z < R; ++z) {
                size_t lin = ((size_t)x * R + y) * R + z;
                int me = lab[lin];
                if (me < 0) { out[lin] = -1; continue; }
                int ids[7], cnt[7], nu = 1;
                ids[0] = me; cnt[0] = 1;
                for (int ax = 0; ax < 3; ++ax)
                    for (int dir = -1; dir <= 1; dir += 2) {
                        int c[3] = {x, y, z};
                        c[ax] = wrapi(c[ax] + dir, R);
                        int id = lab[((size_t)c[0] * R + c[1]) * R + c[2]];
                        if (id >= 0) {
                            int found = 0;
                            for (int k = 0; k < nu; ++k)
                                if (ids[k] == id) { cnt[k]++; found = 1; break; }
                            if (!found && nu < 7) { ids[nu] = id; cnt[nu] = 1; nu++; }
                        }
                    }
                int mc = 0, best = me;
                for (int k = 0; k < nu; ++k)
                    if (cnt[k] > mc) { mc = cnt[k]; best = ids[k]; }
                out[lin] = best;
            }
}

/* accumulate_face_area (jfa.py:702-762), serial semantics: voxels in raster
 * order, then axis 0..2 x dir (-1,+1); a face between labels a<b (both in
 * [0,n)) is counted from the lower-label side into face_ids/face_counts[a],
 * claiming the first free slot on first touch; a 33rd distinct partner is
 * dropped. */
void orc_accumulate_faces(const int32_t* filt, int R, int n, int32_t* face_ids,
                          int32_t* face_counts) {
    for (size_t k = 0; k < (size_t)n * ORC_S; ++k) { face_ids[k] = -1; face_counts[k] = 0; }
    for (int x = 0; x < R; ++x)
        for (int y = 0; y < R; ++y)
            for (int z = 0; z < R; ++z) {
                int a = filt[((size_t)x * R + y) * R + z];
                if (a < 0 || a >= n) continue;
                for (int ax = 0; ax < 3; ++ax)
                    for (int dir = -1; dir <= 1; dir += 2) {
                        int c[3] = {x, y, z};
                        c[ax] = wrapi(c[ax] + dir, R);
                        int b = filt[((size_t)c[0] * R + c[1]) * R + c[2]];
                        if (b >= 0 && b < n && a < b) {
                            int32_t* ids = face_ids + (size_t)a * ORC_S;
                            int32_t* cnt = face_counts + (size_t)a * ORC_S;
                            for (int s = 0; s < ORC_S; ++s) {
                                if (ids[s] == b) { cnt[s]++; break; }
                                if (ids[s] == -1) { ids[s] = b; cnt[s]++; break; }
                            }
                        }
                    }
            }
}

/* add_neighbor (jfa.py:400-443) */
static int add_neighbor(int i, int j, float score, int32_t* nl, int32_t* used, int32_t* fsc,
                        float* prev) {
    int u = used[i];
    for (int s = 0; s < u; ++s)
        if (nl[(size_t)i * ORC_S + s] == j) { prev[(size_t)i * ORC_S + s] = score; return s; }
    if (u < ORC_S) {
        nl[(size_t)i * ORC_S + u] = j;
        prev[(size_t)i * ORC_S + u] = score;
        fsc[i] += 1;
        used[i] += 1;
        return u;
    }
    return -1;
}

/* finalize_faces_kernel (jfa.py:788-857) with expected_area (jfa.py:378-397),
 * serial semantics.  prev (neighbor_prev_scores) persists across calls and is
 * read at face-slot index but written at neighbour-list index, exactly as the
 * reference does.  neighbor_count equals used and is not returned separately. */
void orc_finalize(int n, const float* rad, const int32_t* face_ids, const int32_t* face_counts,
                  float vs, float face_scale, float t_add, float t_drop, float* prev,
                  int32_t* nl, int32_t* used, int32_t* fsc) {
    for (int i = 0; i < n; ++i) {
        fsc[i] = 0; used[i] = 0;
        for (int s = 0; s < ORC_S; ++s) nl[(size_t)i * ORC_S + s] = -1;
    }
    for (int i = 0; i < n; ++i) {
        float ri = rad[i];
        for (int s = 0; s < ORC_S; ++s) {
            int j = face_ids[(size_t)i * ORC_S + s];
            if (j < 0 || j >= n) continue;
            int vox = face_counts[(size_t)i * ORC_S + s];
            if (vox <= 0) continue;
            float rj = rad[j];
            float rm = 0.5f * (ri + rj);
            float q = (2.0f * rm) / vs;
            float expected = face_scale * (q * q);
            if (expected <= 0.0f) continue;
            float score = (float)vox / expected;
            float ps = prev[(size_t)i * ORC_S + s];
            int keep = (ps >= t_drop && score >= t_drop);
            int acc = (score >= t_add) || keep;
            if (acc) {
                add_neighbor(i, j, score, nl, used, fsc, prev);
                add_neighbor(j, i, score, nl, used, fsc, prev);
            } else {
                prev[(size_t)i * ORC_S + s] = 0.0f;
            }
        }
    }
}

/* update_fsc_ema (jfa.py:765-785) */
void orc_fsc_ema(int n, const int32_t* fsc, float* ema, float alpha) {
    for (int i = 0; i < n; ++i) {
        if (ema[i] == 0.0f && fsc[i] > 0) ema[i] = (float)fsc[i];
        else ema[i] = alpha * (float)fsc[i] + (1.0f - alpha) * ema[i];
    }
}

/* ----------------------------------------------------------------- hash grid
 * grid.wrapP (grid.py:30-48): p - L*floor(p*INV_L + 0.5) */
static inline float grid_wrap(float p, float L, float invL) { return p - L * floorf(p * invL + 0.5f); }

/* cell of an already wrapped position as count/scatter compute it
 * (grid.py:204-222, 287-301): floor(((w + HALF_L) + 1e-7) * INV_L * GRID_RES) */
static inline int grid_cell_w(const float* w, float invL, float halfL, int G) {
    int c[3];
    for (int d = 0; d < 3; ++d) {
        float q = ((w[d] + halfL) + 1e-7f) * invL;
        c[d] = wrapi((int)floorf(q * (float)G), G);
    }
    return c[0] * G * G + c[1] * G + c[2];
}

/* rebuild_grid (run.py:476-504) = clear_grid, count_particles_per_cell,
 * prefix_sum, copy_cell_pointers, scatter_particles (grid.py:145-309), serial
 * semantics: scatter visits particles in index order, so each cell's slice of
 * cell_indices is ascending.  pos is wrapped in place as scatter does. */
void orc_grid_build(float* pos, int n, int G, float L, float invL, float halfL,
                    int32_t* cell_count, int32_t* cell_start, int32_t* cell_indices) {
    int GC = G * G * G;
    for (int c = 0; c < GC; ++c) cell_count[c] = 0;
    for (int i = 0; i < n; ++i) {
        float w[3];
        for (int d = 0; d < 3; ++d) w[d] = grid_wrap(pos[3 * i + d], L, invL);
        cell_count[grid_cell_w(w, invL, halfL, G)]++;
    }
    cell_start[0] = 0;
    for (int c = 1; c < GC; ++c) cell_start[c] = cell_start[c - 1] + cell_count[c - 1];
    int32_t* wr = (int32_t*)malloc(sizeof(int32_t) * (size_t)GC);
    memcpy(wr, cell_start, sizeof(int32_t) * (size_t)GC);
    for (int i = 0; i < n; ++i) {
        float w[3];
        for (int d = 0; d < 3; ++d) w[d] = grid_wrap(pos[3 * i + d], L, invL);
        for (int d = 0; d < 3; ++d) pos[3 * i + d] = w[d];
        cell_indices[wr[grid_cell_w(w, invL, halfL, G)]++] = i;
    }
    free(wr);
}

/* home cell as project_overlaps / compute_local_max_overlaps compute it
 * (dynamics.py:101-103): int(q*GRID_RES), no epsilon, no wrap before +-1 */
static inline void home_cell(const float* p, float L, float invL, float halfL, int G, int c[3]) {
    for (int d = 0; d < 3; ++d) {
        float w = grid_wrap(p[d], L, invL);
        float q = (w + halfL) * invL;
        c[d] = (int)(q * (float)G);
    }
}

/* project_overlaps (dynamics.py:77-171) restated as one Jacobi sweep: every
 * particle reads pos_in and writes pos_out.  gap1 = f32(1+GAP_FRACTION),
 * mdf = f32(MAX_DISPLACEMENT_FRAC), dmul = f32(DISPLACEMENT_MULTIPLIER). */
void orc_pbd(const float* pos_in, float* pos_out, const float* rad, int n, int G, float L,
             float invL, float halfL, const int32_t* cell_start, const int32_t* cell_count,
             const int32_t* cell_indices, float gap1, float mdf, float dmul) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const float* pi = pos_in + 3 * i;
        float cx = 0.0f, cy = 0.0f, cz = 0.0f;
        int hc[3];
        home_cell(pi, L, invL, halfL, G, hc);
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    int nx = wrapi(hc[0] + dx, G), ny = wrapi(hc[1] + dy, G), nz = wrapi(hc[2] + dz, G);
                    int cid = nx * G * G + ny * G + nz;
                    int st = cell_start[cid], ct = cell_count[cid];
                    for (int k = st; k < st + ct; ++k) {
                        int j = cell_indices[k];
                        if (j == i) continue;
                        const float* pj = pos_in + 3 * j;
                        float ddx = grid_wrap(pj[0] - pi[0], L, invL);
                        float ddy = grid_wrap(pj[1] - pi[1], L, invL);
                        float ddz = grid_wrap(pj[2] - pi[2], L, invL);
                        float dist = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz + 1e-12f);
                        float tsep = (rad[i] + rad[j]) * gap1;
                        if (dist < tsep) {
                            float ov = tsep - dist;
                            float ux = ddx / dist, uy = ddy / dist, uz = ddz / dist;
                            float mag = ov * 0.5f;
                            float md = mdf * rad[i];
                            mag = fminf(mag, md);
                            float vx = -ux * mag, vy = -uy * mag, vz = -uz * mag;
                            vx = fmaxf(-md, fminf(md, vx));
                            vy = fmaxf(-md, fminf(md, vy));
                            vz = fmaxf(-md, fminf(md, vz));
                            cx += vx; cy += vy; cz += vz;
                        }
                    }
                }
        float mt = mdf * rad[i] * dmul;
        float cm = sqrtf(cx * cx + cy * cy + cz * cz);
        if (cm > mt) {
            float s = mt / cm;
            cx = cx * s; cy = cy * s; cz = cz * s;
        }
        pos_out[3 * i + 0] = grid_wrap(pi[0] + cx, L, invL);
        pos_out[3 * i + 1] = grid_wrap(pi[1] + cy, L, invL);
        pos_out[3 * i + 2] = grid_wrap(pi[2] + cz, L, invL);
    }
}

/* compute_local_max_overlaps + reduce_max_depth (dynamics.py:304-372) */
float orc_max_overlap(const float* pos, const float* rad, int n, int G, float L, float invL,
                      float halfL, const int32_t* cell_start, const int32_t* cell_count,
                      const int32_t* cell_indices, float eps, float* local_max) {
    float gmax = 0.0f;
#pragma omp parallel for schedule(static) reduction(max : gmax)
    for (int i = 0; i < n; ++i) {
        const float* pi = pos + 3 * i;
        float ri = rad[i];
        int hc[3];
        home_cell(pi, L, invL, halfL, G, hc);
        float lm = 0.0f;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    int nx = wrapi(hc[0] + dx, G), ny = wrapi(hc[1] + dy, G), nz = wrapi(hc[2] + dz, G);
                    int cid = nx * G * G + ny * G + nz;
                    int st = cell_start[cid], ct = cell_count[cid];
                    for (int k = st; k < st + ct; ++k) {
                        int j = cell_indices[k];
                        if (!(i < j)) continue;
                        const float* pj = pos + 3 * j;
                        float ddx = grid_wrap(pj[0] - pi[0], L, invL);
                        float ddy = grid_wrap(pj[1] - pi[1], L, invL);
                        float ddz = grid_wrap(pj[2] - pi[2], L, invL);
                        float dist = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz + eps);
                        float td = ri + rad[j];
                        if (dist < td) lm = fmaxf(lm, td - dist);
                    }
                }
        local_max[i] = lm;
        if (lm > gmax) gmax = lm;
    }
    return gmax;
}

/* hash_func (dynamics.py:1436-1451), wrapping int32 arithmetic */
static inline int32_t hash_func(int32_t i, int32_t frame) {
    uint32_t t = (uint32_t)i + 12345u * (uint32_t)frame;
    uint32_t h = 1103515245u * t + 12345u;
    return (int32_t)(h & 0x7fffffffu);
}

/* equilibrate_pressure (dynamics.py:1454-1557): one Jacobi sweep.  Reads the
 * first fsc[i] slots of face_ids[i] starting at a hashed rotation; entries <0,
 * >=n or ==i are skipped.  Returns max |dr|; *changed gets the count of
 * |dr| > 1e-12. */
float orc_pressure(int n, int frame, float* rad, float* delta_r, const int32_t* face_ids,
                   const int32_t* fsc, float k, float P, float cap, int max_nei, float rmin,
                   float rmax, int* changed) {
    for (int i = 0; i < n; ++i) delta_r[i] = 0.0f;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        float Vi = powf(rad[i], P);
        int fc = fsc[i];
        if (fc <= 0) continue;
        int an = fc < max_nei ? fc : max_nei;
        int st = hash_func(i, frame) % fc;
        float acc = 0.0f;
        for (int kk = 0; kk < an; ++kk) {
            int ni = (st + kk) % fc;
            int j = face_ids[(size_t)i * ORC_S + ni];
            if (j < 0 || j >= n || j == i) continue;
            float Vj = powf(rad[j], P);
            float dvr = k * (Vi - Vj);
            float vmin = fminf(Vi, Vj);
            float dv = fmaxf(-cap * vmin, fminf(cap * vmin, dvr));
            float vn = Vi - dv;
            acc += powf(vn, 1.0f / P) - rad[i];
        }
        delta_r[i] = acc;
    }
    float mx = 0.0f;
    int ch = 0;
    for (int i = 0; i < n; ++i) {
        float d = delta_r[i];
        if (fabsf(d) > 1e-12f) {
            ch++;
            if (fabsf(d) > mx) mx = fabsf(d);
        }
        rad[i] = fmaxf(rmin, fminf(rmax, rad[i] + d));
    }
    if (changed) *changed = ch;
    return mx;
}

/* -------------------------------------------------------------- Philox4x32-10
 * Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11.  Replaces ti.random() so host and device draw identical jitter. */
static void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
        uint32_t h0 = (uint32_t)(p0 >> 32), l0 = (uint32_t)p0;
        uint32_t h1 = (uint32_t)(p1 >> 32), l1 = (uint32_t)p1;
        uint32_t n0 = h1 ^ ctr[1] ^ k0;
        uint32_t n2 = h0 ^ ctr[3] ^ k1;
        ctr[0] = n0; ctr[1] = l1; ctr[2] = n2; ctr[3] = l0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

void orc_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                uint32_t* out4) {
    uint32_t c[4] = {c0, c1, c2, c3};
    philox4x32_10(c, k0, k1);
    memcpy(out4, c, sizeof(c));
}

#define ORC_BROWNIAN_STREAM 0x42524f57u

/* apply_brownian_motion (dynamics.py:1596-1634) with the Philox draw
 * u = (x >> 8) * 2^-24 per axis, counter (i, frame, stream, 0), key = seed. */
void orc_brownian(float* pos, int n, float strength, float domain, uint64_t seed, uint32_t frame) {
    float halfL = domain * 0.5f;
    for (int i = 0; i < n; ++i) {
        uint32_t c[4] = {(uint32_t)i, frame, ORC_BROWNIAN_STREAM, 0u};
        philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        for (int d = 0; d < 3; ++d) {
            float u = (float)(c[d] >> 8) * 0x1p-24f;
            float dd = (u - 0.5f) * 2.0f * strength;
            float p = pos[3 * i + d] + dd;
            if (p < -halfL) p += domain;
            else if (p >= halfL) p -= domain;
            pos[3 * i + d] = p;
        }
    }
}

/* ---------------------------------------------------------- dirty tiles
 * mark_dirty_tiles / count_dirty_tiles (jfa.py:966-1024); tiles of 16^3
 * voxels, dirty[t][t][t] uint8; pos_thr / rad_thr already scaled by
 * VOXEL_SIZE (folded in double, rounded to float32). */
void orc_dirty_mark(const float* pos, const float* rad, const float* pos_prev,
                    const float* rad_prev, int n, int R, float halfL, float L, float pos_thr,
                    float rad_thr, int halo, uint8_t* dirty) {
    int t = (R + 15) / 16;
    for (int i = 0; i < n; ++i) {
        const float* p = &pos[3 * i];
        const float* q = &pos_prev[3 * i];
        float dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
        float dpos = sqrtf(dx * dx + dy * dy + dz * dz);
        float drad = fabsf(rad[i] - rad_prev[i]);
        int tc[3], moved = 0;
        for (int k = 0; k < 3; ++k) {
            tc[k] = w2v(p[k], halfL, L, R) / 16;
            moved |= tc[k] != w2v(q[k], halfL, L, R) / 16;
        }
        if (!(dpos > pos_thr || drad > rad_thr || moved)) continue;
        for (int oz = -halo; oz <= halo; ++oz)
            for (int oy = -halo; oy <= halo; ++oy)
                for (int ox = -halo; ox <= halo; ++ox)
                    dirty[((size_t)wrapi(tc[0] + ox, t) * t + wrapi(tc[1] + oy, t)) * t +
                          wrapi(tc[2] + oz, t)] = 1;
    }
}

int orc_dirty_count(const uint8_t* dirty, int R) {
    int t = (R + 15) / 16, c = 0;
    for (int k = 0; k < t * t * t; ++k) c += dirty[k] == 1;
    return c;
}

/* ------------------------------------------------------------- topology
 * topology.py restated with serial semantics.  Grid arguments are the CSR
 * arrays of orc_grid_build (each cell's particles ascending). */

/* grid.pdelta (grid.py:51-66): wrapP(b - a) */
static inline void topo_pdelta(const float* a, const float* b, float L, float invL, float d[3]) {
    for (int k = 0; k < 3; ++k) d[k] = grid_wrap(b[k] - a[k], L, invL);
}

static inline float topo_dot(const float d[3]) { return d[0] * d[0] + d[1] * d[1] + d[2] * d[2]; }

/* build_topo_candidates (topology.py:68-135) */
void orc_topo_candidates(const float* pos, const float* rad, const int32_t* cs, const int32_t* cc,
                         const int32_t* ci, int n, int G, float L, float invL, float halfL,
                         float mult, int cap, int32_t* pairs, int32_t* pcount, int32_t* trunc) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        pcount[i] = 0;
        trunc[i] = 0;
        int h[3];
        home_cell(&pos[3 * i], L, invL, halfL, G, h);
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    int c = (wrapi(h[0] + dx, G) * G + wrapi(h[1] + dy, G)) * G + wrapi(h[2] + dz, G);
                    for (int k = cs[c]; k < cs[c] + cc[c]; ++k) {
                        int j = ci[k];
                        if (j <= i) continue;
                        float d[3];
                        topo_pdelta(&pos[3 * i], &pos[3 * j], L, invL, d);
                        float th = mult * (rad[i] + rad[j]);
                        if (topo_dot(d) <= th * th) {
                            if (pcount[i] < cap) {
                                pairs[(size_t)i * cap + pcount[i]] = j;
                                pcount[i] += 1;
                            } else {
                                trunc[i] = 1;
                                break;
                            }
                        }
                    }
                }
    }
}

/* the witness search of topology.py:218-253 (rev = 0) / 407-443 (rev = 1) */
static int topo_is_gabriel(const float* pos, const int32_t* cs, const int32_t* cc,
                           const int32_t* ci, int i, int j, float d2, int G, float L, float invL,
                           float halfL, float cell_size, int rev) {
    float d[3], m[3];
    topo_pdelta(&pos[3 * i], &pos[3 * j], L, invL, d);
    for (int k = 0; k < 3; ++k) m[k] = grid_wrap(pos[3 * i + k] + 0.5f * d[k], L, invL);
    float r_sq = 0.25f * d2;
    int mc[3];
    for (int k = 0; k < 3; ++k) mc[k] = wrapi((int)(((m[k] + halfL) * invL) * (float)G), G);
    float r_d = sqrtf(d2) * 0.5f;
    int sc = (int)ceilf(r_d / cell_size);
    sc = sc < 1 ? 1 : (sc > 3 ? 3 : sc);
    if (sc > G / 2) sc = G / 2;
    float eps = fmaxf(1e-12f, 1e-6f * r_sq);
    for (int dx = -sc; dx <= sc; ++dx)
        for (int dy = -sc; dy <= sc; ++dy)
            for (int dz = -sc; dz <= sc; ++dz) {
                int c = (wrapi(mc[0] + dx, G) * G + wrapi(mc[1] + dy, G)) * G + wrapi(mc[2] + dz, G);
                for (int q = cs[c]; q < cs[c] + cc[c]; ++q) {
                    int k = ci[q];
                    if (k == i || k == j) continue;
                    float e[3];
                    if (rev) topo_pdelta(m, &pos[3 * k], L, invL, e);
                    else topo_pdelta(&pos[3 * k], m, L, invL, e);
                    if (topo_dot(e) < r_sq - eps) return 0;
                }
            }
    return 1;
}

static inline int topo_keep(int i, int j, int frame, int q) {
    uint32_t h = ((uint32_t)i * 73856093u) ^ ((uint32_t)j * 19349663u) ^ ((uint32_t)frame * 83492791u);
    return q <= 1 || ((int32_t)h % q) == 0;
}

/* gabriel_test_topological_degree (topology.py:140-262) */
void orc_topo_gabriel(const float* pos, const int32_t* cs, const int32_t* cc, const int32_t* ci,
                      int n, int G, float L, float invL, float halfL, float cell_size, int frame,
                      int stride, int early_exit, float deg_high, int cap, const int32_t* pairs,
                      const int32_t* pcount, const float* deg_ema, int32_t* deg) {
    for (int i = 0; i < n; ++i) deg[i] = 0;
    for (int i = 0; i < n; ++i) {
        for (int p = 0; p < pcount[i]; ++p) {
            int j = pairs[(size_t)i * cap + p];
            if (!topo_keep(i, j, frame, stride)) continue;
            if (early_exit && deg_ema[i] >= deg_high && deg_ema[j] >= deg_high) continue;
            float d[3];
            topo_pdelta(&pos[3 * i], &pos[3 * j], L, invL, d);
            float d2 = topo_dot(d);
            if (d2 < 1e-16f) continue;
            if (topo_is_gabriel(pos, cs, cc, ci, i, j, d2, G, L, invL, halfL, cell_size, 0) && j > i) {
                deg[i] += 1;
                deg[j] += 1;
            }
        }
    }
}

/* gabriel_update_batched (topology.py:335-446); only the `cap` stored
 * candidates are tested (the reference's count runs past the row) */
void orc_topo_batched(const float* pos, const float* rad, const int32_t* cs, const int32_t* cc,
                      const int32_t* ci, int n, int G, float L, float invL, float halfL,
                      float mult, float cell_size, int batch, int num_batches, int q, int frame,
                      int cap, int32_t* pairs, int32_t* pcount, int32_t* trunc, int32_t* deg) {
    for (int i = 0; i < n; ++i) {
        if (i % num_batches != batch) continue;
        pcount[i] = 0;
        trunc[i] = 0;
        int h[3];
        home_cell(&pos[3 * i], L, invL, halfL, G, h);
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    int c = (wrapi(h[0] + dx, G) * G + wrapi(h[1] + dy, G)) * G + wrapi(h[2] + dz, G);
                    for (int k = cs[c]; k < cs[c] + cc[c]; ++k) {
                        int j = ci[k];
                        if (j <= i || !topo_keep(i, j, frame, q)) continue;
                        float d[3];
                        topo_pdelta(&pos[3 * i], &pos[3 * j], L, invL, d);
                        float th = mult * (rad[i] + rad[j]);
                        if (topo_dot(d) <= th * th) {
                            int cur = pcount[i]++;
                            if (cur < cap) pairs[(size_t)i * cap + cur] = j;
                            else trunc[i] = 1;
                        }
                    }
                }
        int pc = pcount[i] < cap ? pcount[i] : cap;
        for (int p = 0; p < pc; ++p) {
            int j = pairs[(size_t)i * cap + p];
            float d[3];
            topo_pdelta(&pos[3 * i], &pos[3 * j], L, invL, d);
            float d2 = topo_dot(d);
            if (d2 < 1e-16f) continue;
            if (topo_is_gabriel(pos, cs, cc, ci, i, j, d2, G, L, invL, halfL, cell_size, 1)) {
                deg[i] += 1;
                deg[j] += 1;
            }
        }
    }
}

/* knn_topo_degree (topology.py:458-505) */
void orc_topo_knn(const float* pos, const float* rad, const int32_t* cs, const int32_t* cc,
                  const int32_t* ci, int n, int G, float L, float invL, float halfL, float mult,
                  int kmax, int32_t* deg) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        int cnt = 0;
        float lim = mult * rad[i];
        float lim2 = lim * lim;
        int h[3];
        home_cell(&pos[3 * i], L, invL, halfL, G, h);
        for (int dx = -1; dx <= 1 && cnt < kmax; ++dx)
            for (int dy = -1; dy <= 1 && cnt < kmax; ++dy)
                for (int dz = -1; dz <= 1 && cnt < kmax; ++dz) {
                    int c = (wrapi(h[0] + dx, G) * G + wrapi(h[1] + dy, G)) * G + wrapi(h[2] + dz, G);
                    for (int k = cs[c]; k < cs[c] + cc[c]; ++k) {
                        int j = ci[k];
                        if (j == i) continue;
                        float d[3];
                        topo_pdelta(&pos[3 * i], &pos[3 * j], L, invL, d);
                        if (topo_dot(d) <= lim2) {
                            cnt += 1;
                            if (cnt >= kmax) break;
                        }
                    }
                }
        deg[i] = cnt < kmax ? cnt : kmax;
    }
}

/* update_topo_ema / commit_topo_to_ema (topology.py:265-283, 448-455) */
void orc_topo_ema(const int32_t* deg, float* ema, float alpha, int n) {
    for (int i = 0; i < n; ++i) ema[i] = alpha * (float)deg[i] + (1.0f - alpha) * ema[i];
}

/* update_radii_topological (topology.py:286-322) */
void orc_topo_radii(float* rad, const float* deg_eff, float lo, float hi, float grow, float shrink,
                    float rmin, float rmax, int n) {
    for (int i = 0; i < n; ++i) {
        float d = deg_eff[i], r = rad[i];
        if (d < lo) r = r * (1.0f + grow);
        else if (d > hi) r = r * (1.0f - shrink);
        rad[i] = fmaxf(rmin, fminf(rmax, r));
    }
}

#define ORC_OU_STREAM 0x4f554a54u

/* compute_mean_radius (dynamics.py:675-689) as run.py:860-861 uses it: the
 * exact sum of the radii (each one a 2^-40 fixed-point integer), divided by
 * max(1, n) in double and rounded once to float32. */
float orc_mean_radius(const float* rad, int n) {
    long long s = 0;
    for (int i = 0; i < n; ++i) s += llrintf(rad[i] * 0x1p40f);
    return (float)((double)s * 0x1p-40 / (double)(n > 1 ? n : 1));
}

/* apply_brownian + integrate_jitter (dynamics.py:607-660), the frame's step
 * 6B (run.py:855-867).  ti.random() - 0.5 per axis is u - 0.5 with
 * u = (x >> 8) * 2^-24 from Philox-4x32-10 (i, frame, 'OUJT', 0), key = seed.
 * Python-level constants fold in double and round once to float32. */
void orc_ou_jitter(float* pos, float* v_jit, const float* rad, int n, float mean_r, float dt,
                   double rms, double tau, double max_drift, double gap, float L, float invL,
                   uint64_t seed, uint32_t frame) {
    const double t = tau > 1e-6 ? tau : 1e-6;
    const float tau_f = (float)t, sq2 = (float)sqrt(2.0 / t), rms_f = (float)rms;
    const float capk = (float)(max_drift * gap);
    const float sigma = (rms_f * mean_r) * sq2;
    const float kick = sigma * sqrtf(dt);
    for (int i = 0; i < n; ++i) {
        uint32_t c[4] = {(uint32_t)i, frame, ORC_OU_STREAM, 0u};
        philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        float v[3];
        for (int d = 0; d < 3; ++d) {
            float r = (float)(c[d] >> 8) * 0x1p-24f - 0.5f;
            float vd = v_jit[3 * i + d];
            v[d] = vd + ((-vd / tau_f) * dt + kick * r);
        }
        float cap = capk * (rad[i] + rad[i]);
        float len = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * dt;
        if (len > cap) {
            float sc = (cap / fmaxf(1e-6f, len)) / dt;
            for (int d = 0; d < 3; ++d) v[d] = v[d] * sc;
        }
        for (int d = 0; d < 3; ++d) {
            v_jit[3 * i + d] = v[d];
            pos[3 * i + d] = grid_wrap(pos[3 * i + d] + v[d] * dt, L, invL);
        }
    }
}

/* smoothstep (dynamics.py:1226-1240) */
static inline float smoothstep(float e0, float e1, float x) {
    float t = fminf(1.0f, fmaxf(0.0f, (x - e0) / (e1 - e0)));
    return t * t * (3.0f - 2.0f * t);
}

/* set_fsc_targets (dynamics.py:1242-1320) */
void orc_set_targets(const float* rad, float* rad_target, const int32_t* fsc, const float* ema,
                     int n, int f_low, int f_high, float growth, float rmin, float rmax,
                     float deadband) {
    const float hg = 1.0f, idle = 0.003f;
    for (int i = 0; i < n; ++i) {
        float r0 = rad[i];
        float f = ema[i] > 0.0f ? ema[i] : (float)fsc[i];
        float lo = (float)f_low, hi = (float)f_high;
        float gain;
        if (f < lo - hg) {
            gain = 1.0f;
            rad_target[i] = fminf(r0 * (1.0f + growth * gain), rmax);
        } else if (f < lo) {
            gain = 1.0f - smoothstep(lo - hg - deadband, lo, f);
            rad_target[i] = fminf(r0 * (1.0f + growth * gain), rmax);
        } else if (f > hi + hg) {
            gain = 1.0f;
            rad_target[i] = fmaxf(r0 * (1.0f - growth * gain), rmin);
        } else if (f > hi) {
            gain = smoothstep(hi, hi + hg + deadband, f);
            rad_target[i] = fmaxf(r0 * (1.0f - growth * gain), rmin);
        } else {
            float bc = 0.5f * (lo + hi);
            if (f < bc) rad_target[i] = fminf(r0 * (1.0f + growth * idle), rmax);
            else rad_target[i] = fmaxf(r0 * (1.0f - growth * idle), rmin);
        }
    }
}

/* nudge_radii_adaptive_ema (dynamics.py:1366-1427); mode 0 off, 1 global, 2 local */
void orc_nudge(float* rad, const float* rad_target, const float* local_max, int n, float alpha,
               float max_step, float rmin, float rmax, float back_global, int mode,
               float contact_tol) {
    for (int i = 0; i < n; ++i) {
        float r0 = rad[i];
        float rt = fminf(rmax, fmaxf(rmin, rad_target[i]));
        float d = alpha * (rt - r0);
        float b = 1.0f;
        if (mode == 1) b = back_global;
        else if (mode == 2) {
            b = (contact_tol - local_max[i]) / contact_tol;
            b = fminf(1.0f, fmaxf(0.25f, b));
        }
        d = d * b;
        float cap = max_step * r0;
        if (d > cap) d = cap;
        if (d < -cap) d = -cap;
        rad[i] = fminf(rmax, fmaxf(rmin, r0 + d));
    }
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}
