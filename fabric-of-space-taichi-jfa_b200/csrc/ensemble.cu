// ensemble.cu -- batched ensembles: many independent periodic foams advanced
// together, one launch per stage for all of them.
//
// The foams' particles are packed into one index space of n_total particles
// held by an internal context (all particle-level buffers: face rows, pair
// table, finalize arrays, cell-ordered copy, scratch).  Particle indices are
// global everywhere -- JFA labels, face_ids, neighbour lists, the pair table
// -- so every particle-level kernel of the single-foam path (compact, rows,
// reverse lists, the cooperative finalize) runs unchanged on the packed
// arrays.  Only the stages that depend on a foam's geometry look the foam up:
//   voxel stages   the packed label grids give every foam a range starting at
//                  a multiple of 1024 voxels, so a block (<= 1024 threads)
//                  never straddles two foams; the block finds its foam by a
//                  binary search over the voxel offsets;
//   particle stages foam_of[i] gives the foam's descriptor (hash grid, cell
//                  offset, band, radius bounds, Brownian key, offsets).
// The dynamics of a frame are one persistent cooperative kernel (the same
// phases as k_frame_coop, on arrival-order cell rows) whose grid rebuilds fill
// one packed cell table with each foam's cells at its offset.  Each foam's arithmetic is exactly the
// single-foam path's, with its own local index where the reference uses one
// (the pressure rotation hash, the Brownian counter), so each foam's result
// is bit-identical to running it alone.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "coop.cuh"
#include "jfa_body.cuh"

#define ENS_VOX_ALIGN 1024

struct EnsFoamDev {
    int n, part_off;
    int R, lgR, pow2, passes, final_buf;
    long long vox_off;
    int G, cell_off;
    float vs;
    int f_low, f_high;
    float r_min, r_max;
    uint32_t k0, k1;
};

struct EnsWords {  // per-foam device words
    int settle;
    int zero_fsc;
    unsigned int omax_bits;
    unsigned int rmax_bits;      // the foam's largest radius after the pressure sweeps
    unsigned int rmax0_bits;     // the foam's largest radius at the frame's first rebuild
    int pad;
    unsigned long long rad_sum;  // OU jitter: the foam's radii, 2^-40 fixed point (exact)
    unsigned long long changes[FOS_MAX_PASSES];
};

struct FosEnsemble {
    FosCtx* c = nullptr;  // packed particle-level buffers, frame index, error word
    int nf = 0, ntot = 0, device = 0;
    FosParams p{};
    FosFrameParams fp{};
    std::vector<EnsFoamDev> hf;
    std::vector<long long> hvo;  // voxel offsets [nf + 1]
    std::vector<int> hpo, hco;   // particle / cell offsets [nf + 1]
    EnsFoamDev* df = nullptr;
    EnsWords* dw = nullptr;
    long long* dvo = nullptr;  // [nf + 1]
    int32_t* foam_of = nullptr;
    long long vtot = 0;
    int g3tot = 0, max_passes = 0;
    int32_t *labA = nullptr, *labB = nullptr, *filt = nullptr;
    float4 *recA = nullptr, *recB = nullptr;  // seed records mirroring labA / labB
    unsigned long long* slot = nullptr;
    int32_t* seedlin = nullptr;
    float *pos = nullptr, *rad = nullptr, *rad_target = nullptr, *lmd = nullptr,
          *delta_r = nullptr;
    int32_t *cc = nullptr, *cs = nullptr, *ci = nullptr;
    // OU jitter (fp.ou_jitter): packed velocities and per-foam kick, key, base
    float* vjit = nullptr;
    float* ou_kick = nullptr;
    uint2* ou_key = nullptr;
    int32_t* ou_base = nullptr;
    FosEnsembleTuning tune{256, 256, 1024, 1};
    // runs of the four-voxel record pass (k_ens_jfa_pass_recx): per pass, the
    // foams that take M voxels a thread, with their thread offsets
    struct Run {
        int pass, M, nr;
        long long foam_base, to_base, threads;
    };
    std::vector<Run> runs;
    int32_t* drfoam = nullptr;
    long long* drto = nullptr;
    int multi_voxel = 1;
    // per-foam hash-grid side, first cell and radius bound (surrogate pairs)
    int32_t *dfG = nullptr, *dfcell = nullptr;
    float* dfrmax = nullptr;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    bool gvalid[2] = {false, false};
    FosEnsembleTuning gtune[2];
    long long glaunch[2] = {0, 0};
};

// Kernels of the single-foam path reused on the packed arrays.
__global__ void k_faces_reset(FosDevState* ds, int32_t* rowcnt, int n);
__global__ void k_compact(unsigned long long* keys, unsigned int* hmin, unsigned int* hcnt,
                          const unsigned int* __restrict__ claimed, FosDevState* ds,
                          int32_t* rowcnt, uint4* rowbuf);
__global__ void k_rows(int n, const int32_t* __restrict__ rowcnt, const uint4* __restrict__ rowbuf,
                       int32_t* __restrict__ face_ids, int32_t* __restrict__ face_counts,
                       FosDevState* ds);
__global__ void k_fin_reset(FosDevState* ds, int* fin_changed, int32_t* revcnt, int32_t* revfill,
                            int n);
__global__ void k_rev_fill(int n, const int32_t* __restrict__ face_ids,
                           const float* __restrict__ score, const int32_t* __restrict__ revstart,
                           int32_t* revfill, int32_t* __restrict__ rev);
__global__ void k_rev_sort(int n, const int32_t* __restrict__ revstart, int32_t* __restrict__ rev);
__global__ void k_finalize(int n, const int32_t* __restrict__ revstart,
                           const int32_t* __restrict__ rev, uint8_t* acc0, uint8_t* acc1,
                           const float* __restrict__ score, const int32_t* __restrict__ face_ids,
                           float* prev, int32_t* nl, int32_t* used_out, int32_t* fsc, float* ema,
                           float t_add, float t_drop, float alpha, int apply_ema, FosDevState* ds,
                           int* fin_changed, int max_iters);
__global__ void k_frame_end(FosDevState* ds);
__global__ void k_frame_set(FosDevState* ds, int frame, int settle);
int fos_launch_wrap(FosCtx* c, float* pos, int n, cudaStream_t s);

// Foam owning voxel v of the packed grids: the largest f with vo[f] <= v.
__device__ __forceinline__ int ens_vox_foam(const long long* __restrict__ vo, int nf, long long v) {
    int lo = 0, hi = nf;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(&vo[mid]) <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ------------------------------------------------------------ JFA stages
__global__ void k_ens_seed_prepare(const EnsFoamDev* __restrict__ F,
                                   const int32_t* __restrict__ foam_of, const float* __restrict__ pos,
                                   const float* __restrict__ rad, int ntot, float halfL, float L,
                                   float beta, float4* __restrict__ seeds,
                                   int32_t* __restrict__ seedlin,
                                   unsigned long long* __restrict__ slot) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    const EnsFoamDev& d = F[foam_of[i]];
    const int R = d.R;
    float px = pos[3 * i + 0], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    float br = fmul(beta, rad[i]);
    seeds[i] = make_float4(px, py, pz, fmul(br, br));
    int x = world_to_voxel(px, halfL, L, R);
    int y = world_to_voxel(py, halfL, L, R);
    int z = world_to_voxel(pz, halfL, L, R);
    long long lin = d.vox_off + ((long long)x * R + y) * R + z;
    seedlin[i] = (int32_t)lin;
    slot[lin] = ~0ull;
}

template <bool UNIT_L>
__global__ void k_ens_seed_min(const EnsFoamDev* __restrict__ F, const int32_t* __restrict__ foam_of,
                               const float4* __restrict__ seeds, const int32_t* __restrict__ seedlin,
                               int ntot, float halfL, float L, unsigned long long* __restrict__ slot) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    const EnsFoamDev& d = F[foam_of[i]];
    const int R = d.R;
    long long g = seedlin[i];
    long long lin = g - d.vox_off;
    int z = (int)(lin % R), y = (int)((lin / R) % R), x = (int)(lin / ((long long)R * R));
    float dd = power_dist<UNIT_L>(voxel_centre(x, d.vs, halfL), voxel_centre(y, d.vs, halfL),
                                  voxel_centre(z, d.vs, halfL), seeds[i], L);
    unsigned long long key = ((unsigned long long)float_order_key(dd) << 32) | (unsigned int)i;
    atomicMin(&slot[g], key);
}

__global__ void k_ens_seed_write(const int32_t* __restrict__ seedlin, int ntot,
                                 const unsigned long long* __restrict__ slot,
                                 int32_t* __restrict__ labels) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    long long g = seedlin[i];
    labels[g] = (int32_t)(unsigned int)(slot[g] & 0xFFFFFFFFull);
}

// Pass `pass` of every foam that has it: step = max(1, (R/2) >> pass), the
// single-foam schedule; foams with fewer passes are idle.
template <bool UNIT_L, bool TIE_LOWER>
__global__ void __launch_bounds__(512) k_ens_jfa_pass(const long long* __restrict__ vo, int nf,
                                                      const EnsFoamDev* __restrict__ F,
                                                      int32_t* __restrict__ labA,
                                                      int32_t* __restrict__ labB,
                                                      const float4* __restrict__ seeds,
                                                      float halfL, float L, EnsWords* W,
                                                      int pass) {
    const long long v0 = (long long)blockIdx.x * blockDim.x;
    const int f = ens_vox_foam(vo, nf, v0);
    const EnsFoamDev d = F[f];
    if (pass >= d.passes) return;  // block-uniform
    int step = (d.R / 2) >> pass;
    if (step < 1) step = 1;
    const int32_t* in = ((pass & 1) ? labB : labA) + d.vox_off;
    int32_t* out = ((pass & 1) ? labA : labB) + d.vox_off;
    const long long lin = v0 + threadIdx.x - d.vox_off;
    if (d.pow2)
        jfa_pass_body<UNIT_L, true, TIE_LOWER>(in, out, seeds, d.R, d.lgR, d.vs, halfL, L, step,
                                               W[f].changes, pass, lin);
    else
        jfa_pass_body<UNIT_L, false, TIE_LOWER>(in, out, seeds, d.R, d.lgR, d.vs, halfL, L, step,
                                                W[f].changes, pass, lin);
}

// The same pass over the packed seed-record grids (jfa_pass_rec_body): the
// candidates' seeds come as coalesced record rows instead of label loads and
// seed gathers.  Records of the padding between foams are never read.  One
// candidate loop for every R (jfa_pass_rec_body_any) and 3 blocks of 512
// threads per SM keep it at 40 registers; with a loop per R kind and no
// bound it took 102, and 16 warps per SM.
template <bool UNIT_L>
__global__ void __launch_bounds__(512, UNIT_L ? 3 : 2)
    k_ens_jfa_pass_rec(const long long* __restrict__ vo, int nf,
                                                          const EnsFoamDev* __restrict__ F,
                                                          int32_t* __restrict__ labA,
                                                          int32_t* __restrict__ labB,
                                                          float4* __restrict__ recA,
                                                          float4* __restrict__ recB,
                                                          float halfL, float L, EnsWords* W,
                                                          int pass) {
    const long long v0 = (long long)blockIdx.x * blockDim.x;
    const int f = ens_vox_foam(vo, nf, v0);
    const EnsFoamDev d = F[f];
    if (pass >= d.passes) return;  // block-uniform
    int step = (d.R / 2) >> pass;
    if (step < 1) step = 1;
    const int32_t* in = ((pass & 1) ? labB : labA) + d.vox_off;
    int32_t* out = ((pass & 1) ? labA : labB) + d.vox_off;
    const float4* rin = ((pass & 1) ? recB : recA) + d.vox_off;
    float4* rout = ((pass & 1) ? recA : recB) + d.vox_off;
    const long long lin = v0 + threadIdx.x - d.vox_off;
    jfa_pass_rec_body_any<UNIT_L>(in, rin, out, rout, d.R, d.lgR, d.pow2, d.vs, halfL, L, step,
                                  W[f].changes, pass, lin);
}

// The four-voxel record pass (recx_scan) over the packed grids, unit L.
// One launch covers the foams of one run: those whose pass `pass` takes M
// voxels a thread (M = 4 where R is a multiple of 4s, 2 where it is a multiple
// of 2s, else 1; s the foam's step).  Run foam j's threads start at rto[j]
// (multiples of 256, so a block stays in one foam), R^3 / M of them; a thread
// takes x = xb + m s (m < M) at one (y, z), xb = (xi / s) M s + xi % s.
template <int M>
__global__ void __launch_bounds__(256, 4)
    k_ens_jfa_pass_recx(const long long* __restrict__ rto, const int32_t* __restrict__ rfoam,
                        int nr, const EnsFoamDev* __restrict__ F, int32_t* __restrict__ labA,
                        int32_t* __restrict__ labB, float4* __restrict__ recA,
                        float4* __restrict__ recB, float halfL, EnsWords* W, int pass) {
    const long long t0 = (long long)blockIdx.x * blockDim.x;
    const int j = ens_vox_foam(rto, nr, t0);
    const int f = __ldg(&rfoam[j]);
    const EnsFoamDev d = F[f];
    const int R = d.R;
    int step = (R / 2) >> pass;
    if (step < 1) step = 1;
    const int32_t* in = ((pass & 1) ? labB : labA) + d.vox_off;
    int32_t* out = ((pass & 1) ? labA : labB) + d.vox_off;
    const float4* rin = ((pass & 1) ? recB : recA) + d.vox_off;
    float4* rout = ((pass & 1) ? recA : recB) + d.vox_off;
    const long long V = (long long)R * R * R;
    const long long tl = t0 + threadIdx.x - rto[j];
    const bool live = tl < V / M;
    const int tt = live ? (int)tl : 0;
    const int z = tt % R, yz = tt / R, y = yz % R, xi = yz / R;
    const int g = xi / step;
    const int xb = g * M * step + (xi - g * step);
    int ys[3], zs[3], xp[M + 2];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int o = (k - 1) * step;
        ys[k] = wrap_small(y + o, R) * R;
        zs[k] = wrap_small(z + o, R);
    }
#pragma unroll
    for (int p = 0; p < M + 2; ++p) xp[p] = wrap_small(xb + (p - 1) * step, R) * R * R;
    const float vy = voxel_centre(y, d.vs, halfL), vz = voxel_centre(z, d.vs, halfL);
    float vx[M], bd[M];
    int bl[M], own[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int l = xp[m + 1] + ys[1] + zs[1];
        vx[m] = voxel_centre(xb + m * step, d.vs, halfL);
        own[m] = in[l];
        bd[m] = fminf(power_dist_unit2m(make_float2(vx[m], vy), vz, __ldg(&rin[l])), 1e10f);
        bl[m] = l;
    }
    if (M == 2 && 2 * step == R)  // block-uniform: a block covers one foam
        recx_scan<M, true>(rin, xp, ys, zs, vx, vy, vz, bd, bl);
    else
        recx_scan<M>(rin, xp, ys, zs, vx, vy, vz, bd, bl);
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int l = xp[m + 1] + ys[1] + zs[1];
        int best = own[m];
        if (bl[m] != l) best = in[bl[m]];
        if (live) {
            out[l] = best;
            rout[l] = __ldg(&rin[bl[m]]);
        }
        const int cnt = __syncthreads_count(live && best != own[m]);
        if (threadIdx.x == 0 && cnt) atomicAdd(&W[f].changes[pass], (unsigned long long)cnt);
    }
}

// Records of the packed label grids (seeds[label], NaN bits when unassigned).
__global__ void k_ens_rec_from_labels(const int32_t* __restrict__ lab,
                                      const float4* __restrict__ seeds, float4* __restrict__ rec,
                                      long long V) {
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < V;
         l += (long long)gridDim.x * blockDim.x) {
        const int v = lab[l];
        rec[l] = v >= 0 ? __ldg(&seeds[v]) : rec_none();
    }
}

__global__ void __launch_bounds__(512) k_ens_majority(const long long* __restrict__ vo, int nf,
                                                      const EnsFoamDev* __restrict__ F,
                                                      const int32_t* __restrict__ labA,
                                                      const int32_t* __restrict__ labB,
                                                      int32_t* __restrict__ filt) {
    const long long v0 = (long long)blockIdx.x * blockDim.x;
    const EnsFoamDev d = F[ens_vox_foam(vo, nf, v0)];
    const int32_t* lab = (d.final_buf ? labB : labA) + d.vox_off;
    majority_body(lab, d.R, filt + d.vox_off, v0 + threadIdx.x - d.vox_off);
}

__global__ void __launch_bounds__(512) k_ens_faces(const long long* __restrict__ vo, int nf,
                                                   const EnsFoamDev* __restrict__ F,
                                                   const int32_t* __restrict__ filt, int ntot,
                                                   unsigned long long* keys, unsigned int* hmin,
                                                   unsigned int* hcnt, unsigned int* claimed,
                                                   FosDevState* ds, unsigned long long mask) {
    __shared__ unsigned int s_slot[3 * 512];
    __shared__ int s_n;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const ClaimBuf cb{s_slot, &s_n, claimed};
    const long long v0 = (long long)blockIdx.x * blockDim.x;
    const EnsFoamDev d = F[ens_vox_foam(vo, nf, v0)];
    faces_body(filt + d.vox_off, d.R, ntot, keys, hmin, hcnt, cb, ds, mask,
               v0 + threadIdx.x - d.vox_off);
    faces_claims_flush(cb, claimed, ds);
}

// The same over voxel tiles of FACES_TILE_THREADS voxels with a per-block merge of the pairs
// (faces_tile_body), every foam's R a multiple of 8: a block of
// FACES_TILE_THREADS threads takes one tile of its foam (foam offsets are multiples of 1024 voxels); a
// block in the padding after a foam's voxels does nothing.
__global__ void __launch_bounds__(FACES_TILE_THREADS) k_ens_faces_tile(
    const long long* __restrict__ vo, int nf, const EnsFoamDev* __restrict__ F,
    const int32_t* __restrict__ filt, int ntot, unsigned long long* keys, unsigned int* hmin,
    unsigned int* hcnt, unsigned int* claimed, FosDevState* ds, unsigned long long mask) {
    __shared__ unsigned int s_slot[3 * FACES_TILE_THREADS];
    __shared__ int s_n;
    const long long v0 = (long long)blockIdx.x * FACES_TILE_THREADS;
    const EnsFoamDev d = F[ens_vox_foam(vo, nf, v0)];
    const long long tile = (v0 - d.vox_off) / FACES_TILE_THREADS;
    if (tile * FACES_TILE_THREADS >= (long long)d.R * d.R * d.R) return;  // block-uniform
    if (threadIdx.x == 0) s_n = 0;
    const ClaimBuf cb{s_slot, &s_n, claimed};
    faces_tile_body(filt + d.vox_off, d.R, ntot, keys, hmin, hcnt, cb, ds, mask, (int)tile);
    faces_claims_flush(cb, claimed, ds);
}

__global__ void k_ens_scores(int ntot, const EnsFoamDev* __restrict__ F,
                             const int32_t* __restrict__ foam_of,
                             const int32_t* __restrict__ face_ids,
                             const int32_t* __restrict__ face_counts, const float* __restrict__ rad,
                             float face_scale, float t_add, float* __restrict__ score, uint8_t* acc,
                             int32_t* revcnt) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ntot * FOS_S) return;
    const float vs = F[foam_of[t >> 5]].vs;
    score_slot(t, ntot, face_ids, face_counts, rad, vs, face_scale, t_add, score, acc, revcnt);
}

__global__ void k_ens_jfa_prep(EnsWords* W, int nf) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    W[f].zero_fsc = 0;
    for (int q = 0; q < FOS_MAX_PASSES; ++q) W[f].changes[q] = 0ull;
}

__global__ void k_ens_zero(int ntot, const int32_t* __restrict__ fsc,
                           const int32_t* __restrict__ foam_of, EnsWords* W) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ntot && fsc[i] == 0) atomicAdd(&W[foam_of[i]].zero_fsc, 1);
}

// Warm-start gate + set_fsc_targets per foam (k_set_targets' logic with each
// foam's own zero-FSC fraction, band and radius bounds).
__global__ void k_ens_targets(int ntot, const EnsFoamDev* __restrict__ F,
                              const int32_t* __restrict__ foam_of, EnsWords* W,
                              const FosDevState* __restrict__ ds, const float* __restrict__ rad,
                              float* __restrict__ rt, const int32_t* __restrict__ fsc,
                              const float* __restrict__ ema, float growth, float db,
                              int warm_frames, double zero_thresh, int adjust_frames) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    const int f = foam_of[i];
    const EnsFoamDev& d = F[f];
    double f0 = (double)W[f].zero_fsc / (double)(d.n > 0 ? d.n : 1);
    bool warm = (ds->frame < warm_frames) || (f0 > zero_thresh);
    if (warm) return;
    if (i == d.part_off) W[f].settle = adjust_frames;
    rt[i] = target_one(rad[i], ema[i], fsc[i], d.f_low, d.f_high, growth, d.r_min, d.r_max, db);
}

// ------------------------------------------------------------ dynamics
// Loads of the PBD and max-overlap sweeps: L1-allocating (LdL1) or L2 only
// (LdL2).  Every phase reads what earlier phases wrote behind a grid barrier,
// whose acquire makes those writes visible to the block's plain loads.
#ifndef ENS_SWEEP_LD
#define ENS_SWEEP_LD LdL1
#endif
// Rounds of 8-lane groups in flight in the pressure sweeps: their loads are
// all issued before the first sum.
#ifndef ENS_PRESS_ROUNDS
#define ENS_PRESS_ROUNDS 2
#endif

struct EnsGeo {
    const EnsFoamDev* F;
    const int32_t* foam_of;
    float L, invL, halfL;
    __device__ __forceinline__ int cell(int i, float wx, float wy, float wz) const {
        const EnsFoamDev& d = F[foam_of[i]];
        return d.cell_off + cell_of_wrapped(wx, wy, wz, invL, halfL, d.G);
    }
};

struct EnsArgs {
    // coop_grid fields
    int n, G3, chunk, small_grid;
    int32_t* cc;
    int32_t* cs;
    int32_t* ci;
    int32_t* cellof;
    int32_t* rank;
    int32_t* ci_tmp;
    int32_t* cnt;
    int32_t* cnt2;
    int32_t* cfix;
    int32_t* idsort;
    float4* spfix;
    float4* spst;
    int32_t* slot_of;
    int32_t* part;
    int32_t* bsum;
    float4* sp;
    FosDevState* ds;
    unsigned long long* trace;
    int trace_cap;
    // ensemble
    const EnsFoamDev* F;
    const int32_t* foam_of;
    EnsWords* W;
    int nf, mode, pbd_iters, sweeps, warmup, bp_mode;
    float* pos;
    float* pos_tmp;
    float* rad;
    float* rad_tmp;
    const float* rad_target;
    float* lmd;
    float* delta_r;
    float* vol0;  // [n] r^P ping-pong of the pressure sweeps
    float* vol1;
    int32_t* pnbr;  // [16 n] the frame's pressure neighbours (pressure_nbr_fill)
    float gap1, mdf, dmul, eps, contact_tol;
    double contact_tol_d;
    float alpha, max_step;
    PressureArgs pa;
    float strength, domain, L, invL, halfL;
    // OU jitter (dynamics.py:607-660, run.py:855-867) per foam
    int ou;
    float* vjit;
    float* ou_kick;
    const uint2* ou_key;
    const int32_t* ou_base;
    OuParams ou_p;
};

// One PBD sweep over every particle of every foam on layout `lay`, into
// pos_tmp; with p1, each new position also enters the histogram of the next
// rebuild (count buffer par), wrapped into pos.
__device__ __forceinline__ void ens_pbd(const EnsArgs& a, const EnsGeo& geo, const CoopLayout& lay,
                                        int wid, int W_, int lane, bool p1, int par,
                                        const OuStep* ou = nullptr) {
    const int rounds = (a.n + W_ - 1) / W_;
    P1Defer d1;
    int kk_next = wid < a.n ? __ldcg(&a.slot_of[wid]) : 0;
    for (int r = 0; r < rounds; ++r) {
        const int i = r * W_ + wid;
        const int kk = kk_next;
        kk_next = i + W_ < a.n ? __ldcg(&a.slot_of[i + W_]) : 0;
        if (i < a.n) {  // warp-uniform
            const int f = a.foam_of[i];
            const EnsFoamDev& d = a.F[f];
            const GridGeom g{d.G, a.L, a.invL, a.halfL};
            // the stencil skips the cells beyond reach of the foam's largest
            // radius (set in the Brownian phase; radii are fixed during PBD)
            const float rmax = d.G >= 5 ? __uint_as_float(__ldcg(&a.W[f].rmax_bits)) : 0.f;
            float4 nv = make_float4(0.f, 0.f, 0.f, 0.f);
            int pi = pbd_warp<LdL2>(kk, lane, lay.sp, lay.ci, a.pos_tmp, g,
                                    lay.cs ? lay.cs + d.cell_off : nullptr, lay.cc + d.cell_off,
                                    a.gap1, a.mdf, a.dmul, &nv, lay.cap, d.cell_off, rmax,
                                    a.L / (float)d.G);
            if (p1) d1.put(a, geo, lane, pi, nv, a.pos, coop_p1_par(a, par), ou);
        }
    }
    if (p1) d1.flush(a, geo, a.pos, coop_p1_par(a, par), ou);
}

// A frame's rebuilds on arrival-order rows, as the single-foam frame kernel
// runs them: rebuild r (0 before max overlap, 1..pbd_iters before each PBD
// sweep, pbd_iters + 1 the final CSR one) drops its particles into count
// buffer r % 3 (a.cnt holds three of a.G3 cells), row set r & 1 and overflow
// bit r % 3 of ds->grid_ovf; its P1 runs in the phase that produced the
// positions.  No phase sorts the rows: max overlap does not depend on the
// order, and the PBD sweeps add their hits in (stencil cell, particle index)
// order themselves (pbd_warp_rows).
__device__ __forceinline__ P1Dst ens_p1_dst(const EnsArgs& a, int r) {
    return P1Dst{a.cnt + (size_t)(r % 3) * a.G3, a.cfix ? ((r & 1) ? a.idsort : a.cfix) : nullptr,
                 (r & 1) ? a.spfix : a.spst, a.slot_of, (unsigned int*)&a.ds->grid_ovf,
                 1u << (r % 3)};
}

// Layout of rebuild r for the phase that reads it (its P1 is behind a grid
// barrier): the rows when none overflowed, else the CSR form, whose phases
// run first.  Also clears count buffer and overflow bit (r + 2) % 3 for
// rebuild r + 2, whose P1 comes one phase later (their last reader, of
// rebuild r - 1, is done).
__device__ __forceinline__ bool ens_layout(const EnsArgs& a, const EnsGeo& geo, int r, int& tk,
                                           unsigned int& ep, CoopLayout& lay, bool& rows) {
    const int T = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t* zc = a.cnt + (size_t)((r + 2) % 3) * a.G3;
    for (int c = tid; c < a.G3; c += T) zc[c] = 0;
    const bool ovf = ((*((volatile int*)&a.ds->grid_ovf)) >> (r % 3)) & 1;
    if (tid == 0) atomicAnd(&a.ds->grid_ovf, ~(1 << ((r + 2) % 3)));
    const int32_t* cnt = a.cnt + (size_t)(r % 3) * a.G3;
    rows = a.cfix != nullptr && !ovf;
    if (rows) {
        lay = CoopLayout{(r & 1) ? a.idsort : a.cfix, (r & 1) ? a.spfix : a.spst, nullptr, cnt,
                         COOP_CAP};
        return true;
    }
    lay = CoopLayout{a.ci, a.sp, a.cs, a.cc, 0};
    return coop_csr(a, geo, cnt, a.pos, a.rad, false, tk, ep);
}

// One PBD sweep over every particle of every foam on layout `lay` (rows or
// CSR), into pos_tmp; each new position also enters rebuild `next` (P1).
__device__ __forceinline__ void ens_pbd_frame(const EnsArgs& a, const EnsGeo& geo,
                                              const CoopLayout& lay, bool rows, int wid, int W_,
                                              int lane, const P1Dst& next,
                                              const OuStep* ou = nullptr) {
    const int rounds = (a.n + W_ - 1) / W_;
    P1Defer d1;
    // the next round's slot and foam are loaded one round ahead
    int kk_next = wid < a.n ? __ldcg(&a.slot_of[wid]) : 0;
    int f_next = wid < a.n ? a.foam_of[wid] : 0;
    for (int r = 0; r < rounds; ++r) {
        const int i = r * W_ + wid;
        const int kk = kk_next;
        const int f = f_next;
        kk_next = i + W_ < a.n ? __ldcg(&a.slot_of[i + W_]) : 0;
        f_next = i + W_ < a.n ? a.foam_of[i + W_] : 0;
        if (i < a.n) {  // warp-uniform
            const EnsFoamDev& d = a.F[f];
            const GridGeom g{d.G, a.L, a.invL, a.halfL};
            // the stencil skips the cells beyond reach of the foam's largest
            // radius (set in the Brownian phase; radii are fixed during PBD)
            const float rmax = d.G >= 5 ? __uint_as_float(a.W[f].rmax_bits) : 0.f;
            const float cw = a.L / (float)d.G;
            float4 nv = make_float4(0.f, 0.f, 0.f, 0.f);
            const int pi =
                rows ? pbd_warp_rows<ENS_SWEEP_LD>(kk, lane, lay.sp, lay.ci, a.pos_tmp, g,
                                           lay.cc + d.cell_off, COOP_CAP, a.gap1, a.mdf, a.dmul,
                                           &nv, rmax, cw, d.cell_off)
                     : pbd_warp<ENS_SWEEP_LD>(kk, lane, lay.sp, lay.ci, a.pos_tmp, g, lay.cs + d.cell_off,
                                      lay.cc + d.cell_off, a.gap1, a.mdf, a.dmul, &nv, 0,
                                      d.cell_off, rmax, cw);
            d1.put(a, geo, lane, pi, nv, a.pos, next, ou);
        }
    }
    d1.flush(a, geo, a.pos, next, ou);
}

// The largest radius of each foam into *bits (w: the foam's word): one
// atomic per warp when the warp's particles share a foam (foams are
// contiguous index ranges), else one per particle.  Positive floats order as
// their bits.  Called by every active lane of the warp.
__device__ __forceinline__ void ens_foam_max(unsigned int* bits, int f, float r_i, int lane) {
    const unsigned int am = __activemask();
    const unsigned int rb = __float_as_uint(r_i);
    const int f0 = __shfl_sync(am, f, __ffs(am) - 1);
    if (__all_sync(am, f == f0)) {
        const unsigned int wm = __reduce_max_sync(am, rb);
        if (lane == __ffs(am) - 1 && wm > __ldcg(bits)) atomicMax(bits, wm);
    } else {
        atomicMax(bits, rb);
    }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_ens_coop(EnsArgs a) {
    const int T = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int W_ = T >> 5;
    const int wid = tid >> 5;
    const EnsGeo geo{a.F, a.foam_of, a.L, a.invL, a.halfL};
    int tk = 0;
    unsigned int ep = 0;
    if (a.trace && threadIdx.x == 0) atomicMax(&a.trace[a.trace_cap - 2], ~global_ns());
    trace_mark(a, tk);
    CoopLayout lay;
    int gk = 0;  // the warm-up form's rebuild gk uses count buffer gk & 1 (coop_grid)
    if (a.mode == 1) {
        // warmup_pbd of initialize_simulation (run.py:293-318): grid + PBD + copy-back
        for (int k = 0; k < a.warmup; ++k) {
            if (!coop_grid(a, geo, a.pos, a.pos, a.rad, false, tk, ep, false, gk & 1, false, &lay))
                return;
            ++gk;
            ens_pbd(a, geo, lay, wid, W_, lane, false, 0);
            if (!grid_barrier(a.ds, ep)) return;
            for (int i = tid; i < 3 * a.n; i += T) a.pos[i] = __ldcg(&a.pos_tmp[i]);
            if (!grid_barrier(a.ds, ep)) return;
        }
        return;
    }
    // (1) rebuild_grid: rebuild 0's P1, with each foam's largest radius for
    // the max-overlap stencils
    {
        const P1Dst t = ens_p1_dst(a, 0);
        for (int i = spread_tid(); i < a.n; i += T) {
            const float r_i = __ldcg(&a.rad[i]);
            ens_foam_max(&a.W[a.foam_of[i]].rmax0_bits, a.foam_of[i], r_i, lane);
            coop_p1_val(a, geo, i,
                        make_float3(__ldcg(&a.pos[3 * i + 0]), __ldcg(&a.pos[3 * i + 1]),
                                    __ldcg(&a.pos[3 * i + 2])),
                        r_i, a.pos, t);
        }
    }
    if (!grid_barrier(a.ds, ep)) return;
    trace_mark(a, tk);
    // (2) compute_max_overlap: per-foam maxima; the stencils visit only the
    // cells that can hold a positive depth
    bool rows = false;
    if (!ens_layout(a, geo, 0, tk, ep, lay, rows)) return;
    {
        const int rounds = (a.n + W_ - 1) / W_;
        int kk_next = wid < a.n ? __ldcg(&a.slot_of[wid]) : 0;
        int f_next = wid < a.n ? a.foam_of[wid] : 0;
        for (int r = 0; r < rounds; ++r) {
            const int i = r * W_ + wid;
            const int kk = kk_next;
            const int f = f_next;
            kk_next = i + W_ < a.n ? __ldcg(&a.slot_of[i + W_]) : 0;
            f_next = i + W_ < a.n ? a.foam_of[i + W_] : 0;
            if (i < a.n) {
                const EnsFoamDev& d = a.F[f];
                const GridGeom g{d.G, a.L, a.invL, a.halfL};
                const float rmax0 = d.G >= 5 ? __uint_as_float(a.W[f].rmax0_bits) : 0.f;
                unsigned int b = maxov_warp<ENS_SWEEP_LD>(kk, lane, lay.sp, lay.ci, g,
                                                  lay.cs ? lay.cs + d.cell_off : nullptr,
                                                  lay.cc + d.cell_off, a.eps, a.lmd, lay.cap,
                                                  d.cell_off, rmax0, a.L / (float)d.G);
                if (lane == 0 && b > __ldcg(&a.W[f].omax_bits)) atomicMax(&a.W[f].omax_bits, b);
            }
        }
    }
    if (!grid_barrier(a.ds, ep)) return;
    trace_mark(a, tk);
    // (3) settle nudge of the foams whose settle counter is > 0; each final
    // radius's power r^P seeds the pressure sweeps, and each particle's
    // neighbours of the sweeps go to the table (its foam's hash offset)
    const int frame = *((volatile int*)&a.ds->frame);
    for (int i = tid; i < a.n; i += T) {
        const int f = a.foam_of[i];
        if (a.sweeps > 0) {
            PressureArgs pa = a.pa;
            pa.frame = frame;
            pa.hoff = a.F[f].part_off;
            pressure_nbr_fill<LdL2>(i, pa, a.pnbr);
        }
        float r = __ldcg(&a.rad[i]);
        if (*((volatile int*)&a.W[f].settle) > 0) {
            const EnsFoamDev& d = a.F[f];
            float bg = back_global_from_bits(*((volatile unsigned int*)&a.W[f].omax_bits),
                                             a.contact_tol_d);
            r = nudge_one(r, __ldcg(&a.rad_target[i]), __ldcg(&a.lmd[i]), a.alpha, a.max_step,
                          d.r_min, d.r_max, bg, a.bp_mode, a.contact_tol);
            a.rad[i] = r;
        }
        if (a.sweeps > 0) a.vol0[i] = pow_P(r, a.pa.P);
    }
    if (!grid_barrier(a.ds, ep)) return;
    trace_mark(a, tk);
    // (4) pressure sweeps with each foam's bounds, on the neighbour table; two
    // rounds at a time, both groups' loads before either sum
    {
        const int groups_per_round = T / 8;
        const int p_rounds = (a.n + groups_per_round - 1) / groups_per_round;
        for (int w = 0; w < a.sweeps; ++w) {
            const float* rin = (w & 1) ? a.rad_tmp : a.rad;
            float* rout = (w & 1) ? a.rad : a.rad_tmp;
            const float* vin = (w & 1) ? a.vol1 : a.vol0;
            float* vout = (w == a.sweeps - 1) ? nullptr : ((w & 1) ? a.vol0 : a.vol1);
            constexpr int NR = ENS_PRESS_ROUNDS;
            for (int r = 0; r < p_rounds; r += NR) {
                int ii[NR];
                PressureIn pin[NR];
                float2 bnd[NR];
#pragma unroll
                for (int h = 0; h < NR; ++h) {
                    ii[h] = (r + h) * groups_per_round + tid / 8;
                    pin[h] = pressure_in8x2n<PRESS_LD>(ii[h], lane, a.n, a.pnbr, rin, vin);
                    bnd[h] = make_float2(0.f, 0.f);
                    if (ii[h] < a.n) {
                        const EnsFoamDev& d = a.F[a.foam_of[ii[h]]];
                        bnd[h] = make_float2(d.r_min, d.r_max);
                    }
                }
#pragma unroll
                for (int h = 0; h < NR; ++h)
                    pressure_out8x2n(ii[h], lane, a.n, a.pa, pin[h], bnd[h].x, bnd[h].y, rout, vout,
                                     a.delta_r);
            }
            if (!grid_barrier(a.ds, ep)) return;
            trace_mark(a, tk);
        }
    }
    // (5) Brownian jitter with each foam's key and local counter; settle -= 1.
    // With the OU jitter on, each foam's final radii are also summed exactly
    // for its mean radius (run.py:860-861).
    for (int i = tid; i < a.n; i += T) {
        if (a.sweeps & 1) a.rad[i] = __ldcg(&a.rad_tmp[i]);
        const int f = a.foam_of[i];
        const EnsFoamDev& d = a.F[f];
        const float r_i = __ldcg(&a.rad[i]);
        if (a.ou) atomicAdd(&a.W[f].rad_sum, (unsigned long long)rad_fixed(r_i));
        ens_foam_max(&a.W[f].rmax_bits, f, r_i, lane);  // for the PBD stencils
        brownian_one<LdL2>(i, (unsigned int)(i - d.part_off), a.pos, a.strength, a.domain, a.halfL,
                           d.k0, d.k1, (unsigned int)frame);
        coop_p1_one(a, geo, i, a.pos, a.rad, a.pos, ens_p1_dst(a, 1));
    }
    for (int f = tid; f < a.nf; f += T)
        if (a.W[f].settle > 0) a.W[f].settle -= 1;
    if (!grid_barrier(a.ds, ep)) return;
    trace_mark(a, tk);
    // (6) PBD sweeps, each on a fresh grid; (7) final rebuild.  The OU jitter
    // (run.py:855-867) runs inside the last sweep's P1 with each foam's kick
    // (from its mean radius, written here, read after the layout phase's
    // barrier), key and local counter, as the single-foam frame does.
    if (a.ou)
        for (int f = tid; f < a.nf; f += T)
            a.ou_kick[f] = ou_kick(a.ou_p, mean_from_fixed(
                                                *((volatile unsigned long long*)&a.W[f].rad_sum),
                                                a.F[f].n));
    OuStep ous{a.vjit, a.rad, a.ou_p, 0.f, (unsigned int)frame, 0,
               a.foam_of, a.ou_kick, a.ou_key, a.ou_base};
    for (int k = 0; k < a.pbd_iters; ++k) {
        if (!ens_layout(a, geo, k + 1, tk, ep, lay, rows)) return;
        ens_pbd_frame(a, geo, lay, rows, wid, W_, lane, ens_p1_dst(a, k + 2),
                      a.ou && k == a.pbd_iters - 1 ? &ous : nullptr);
        if (!grid_barrier(a.ds, ep)) return;
        trace_mark(a, tk);
    }
    coop_csr(a, geo, a.cnt + (size_t)((a.pbd_iters + 1) % 3) * a.G3, a.pos, nullptr, true, tk, ep);
    if (a.trace) {
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(&a.trace[a.trace_cap - 1], global_ns());
    }
}

__global__ void k_ens_coop_prep(FosDevState* ds, EnsWords* W, int nf) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < nf) {
        W[f].omax_bits = 0u;
        W[f].rmax_bits = 0u;
        W[f].rmax0_bits = 0u;
        W[f].rad_sum = 0ull;
    }
    if (f == 0) {
        ds->grid_ovf = 0;
        ds->bar_count = 0u;
        ds->omax_bits = 0u;
        ds->maxabs_dr_bits = 0u;
        ds->changed = 0;
    }
}

// ------------------------------------------------------------ host
static int ilog2i(int v) {
    int r = 0;
    while ((1 << r) < v) ++r;
    return r;
}

extern "C" int fos_ensemble_destroy(FosEnsemble* e) {
    if (!e) return FOS_OK;
    cudaSetDevice(e->device);
    for (int k = 0; k < 2; ++k)
        if (e->gexec[k]) cudaGraphExecDestroy(e->gexec[k]);
    void* ptrs[] = {e->df,  e->dw,  e->dvo,        e->foam_of, e->labA, e->labB, e->filt,
                    e->recA, e->recB,
                    e->slot, e->seedlin, e->pos,   e->rad,     e->rad_target, e->lmd,
                    e->delta_r, e->cc, e->cs,      e->ci,      e->vjit, e->ou_kick, e->ou_key,
                    e->ou_base, e->drfoam, e->drto, e->dfG, e->dfcell, e->dfrmax};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (e->c) fos_ctx_destroy(e->c);
    delete e;
    return FOS_OK;
}

static int ens_check_foam(const FosEnsembleFoam& f) {
    FOS_REQUIRE(f.n >= 1, FOS_E_ARG, "every foam needs n >= 1");
    FOS_REQUIRE(f.jfa_res >= 2 && f.jfa_res <= 512, FOS_E_ARG, "jfa_res must be in [2, 512]");
    FOS_REQUIRE(f.grid_res >= 3 && f.grid_res <= 1024, FOS_E_ARG, "grid_res must be in [3, 1024]");
    FOS_REQUIRE(f.r_min > 0.0 && f.r_max >= f.r_min, FOS_E_ARG, "need 0 < r_min <= r_max");
    return FOS_OK;
}

static int ens_create_impl(FosEnsemble* e, const FosEnsembleFoam* foams) {
    const int nf = e->nf;
    e->hf.resize(nf);
    e->hvo.assign(nf + 1, 0);
    e->hpo.assign(nf + 1, 0);
    e->hco.assign(nf + 1, 0);
    const double L = e->p.domain_size;
    long long ntot = 0, vtot = 0, g3 = 0;
    int maxp = 0;
    for (int f = 0; f < nf; ++f) {
        const FosEnsembleFoam& in = foams[f];
        EnsFoamDev& d = e->hf[f];
        memset(&d, 0, sizeof(d));
        d.n = in.n;
        d.part_off = (int)ntot;
        d.R = in.jfa_res;
        d.lgR = ilog2i(in.jfa_res);
        d.pow2 = (in.jfa_res & (in.jfa_res - 1)) == 0;
        d.passes = ilog2i(in.jfa_res) + 1;  // ceil(log2 R) + 1 (jfa.py:207-227)
        d.final_buf = d.passes & 1;
        d.vox_off = vtot;
        d.G = in.grid_res;
        d.cell_off = (int)g3;
        d.vs = (float)(L / (double)in.jfa_res);  // VOXEL_SIZE = L / R, folded once
        d.f_low = in.f_low;
        d.f_high = in.f_high;
        d.r_min = (float)in.r_min;
        d.r_max = (float)in.r_max;
        d.k0 = (uint32_t)in.seed;
        d.k1 = (uint32_t)(in.seed >> 32);
        e->hvo[f] = vtot;
        e->hpo[f] = (int)ntot;
        e->hco[f] = (int)g3;
        ntot += in.n;
        long long V = (long long)in.jfa_res * in.jfa_res * in.jfa_res;
        vtot += (V + ENS_VOX_ALIGN - 1) / ENS_VOX_ALIGN * ENS_VOX_ALIGN;
        g3 += (long long)in.grid_res * in.grid_res * in.grid_res;
        maxp = std::max(maxp, d.passes);
    }
    FOS_REQUIRE(ntot <= (1 << 24), FOS_E_CAPACITY, "more than 2^24 particles in the ensemble");
    FOS_REQUIRE(vtot < (1LL << 31), FOS_E_CAPACITY, "packed voxel grids exceed 2^31 voxels");
    FOS_REQUIRE(g3 < (1LL << 31), FOS_E_CAPACITY, "packed cell tables exceed 2^31 cells");
    e->hvo[nf] = vtot;
    e->hpo[nf] = (int)ntot;
    e->hco[nf] = (int)g3;
    e->ntot = (int)ntot;
    e->vtot = vtot;
    e->g3tot = (int)g3;
    e->max_passes = maxp;
    {
        // runs of the four-voxel pass: foam f's step at pass q is
        // max(1, (R/2) >> q); M = 4 where R is a multiple of 4 steps, 2 where
        // it is a multiple of 2, else 1
        std::vector<int32_t> rf;
        std::vector<long long> rt;
        for (int q = 0; q < maxp; ++q)
            for (int M : {4, 2, 1}) {
                FosEnsemble::Run run{q, M, 0, (long long)rf.size(), (long long)rt.size(), 0};
                long long off = 0;
                for (int f = 0; f < nf; ++f) {
                    const EnsFoamDev& d = e->hf[f];
                    if (q >= d.passes) continue;
                    int st = (d.R / 2) >> q;
                    if (st < 1) st = 1;
                    const int m = d.R % (4 * st) == 0 ? 4 : d.R % (2 * st) == 0 ? 2 : 1;
                    if (m != M) continue;
                    rf.push_back(f);
                    rt.push_back(off);
                    const long long T = (long long)d.R * d.R * d.R / M;
                    off += (T + 255) / 256 * 256;
                    ++run.nr;
                }
                if (!run.nr) continue;
                rt.push_back(off);
                run.threads = off;
                e->runs.push_back(run);
            }
        FOS_CUDA(cudaMalloc(&e->drfoam, rf.size() * 4));
        FOS_CUDA(cudaMalloc(&e->drto, rt.size() * sizeof(long long)));
        FOS_CUDA(cudaMemcpy(e->drfoam, rf.data(), rf.size() * 4, cudaMemcpyHostToDevice));
        FOS_CUDA(cudaMemcpy(e->drto, rt.data(), rt.size() * sizeof(long long),
                            cudaMemcpyHostToDevice));
        std::vector<int32_t> fg(nf), fc(nf);
        std::vector<float> fr(nf);
        for (int f = 0; f < nf; ++f) {
            fg[f] = e->hf[f].G;
            fc[f] = e->hf[f].cell_off;
            fr[f] = e->hf[f].r_max;
        }
        FOS_CUDA(cudaMalloc(&e->dfG, nf * 4));
        FOS_CUDA(cudaMalloc(&e->dfcell, nf * 4));
        FOS_CUDA(cudaMalloc(&e->dfrmax, nf * 4));
        FOS_CUDA(cudaMemcpy(e->dfG, fg.data(), nf * 4, cudaMemcpyHostToDevice));
        FOS_CUDA(cudaMemcpy(e->dfcell, fc.data(), nf * 4, cudaMemcpyHostToDevice));
        FOS_CUDA(cudaMemcpy(e->dfrmax, fr.data(), nf * 4, cudaMemcpyHostToDevice));
    }
    // internal context for the packed particle-level buffers: its cell
    // scratch must hold the packed cell table, its own voxel grid is unused
    FosParams cp = e->p;
    int gc = 3;
    while ((long long)gc * gc * gc < g3) ++gc;
    FOS_REQUIRE(gc <= 1024, FOS_E_CAPACITY, "packed cell table too large");
    cp.grid_res = gc;
    int rc = fos_ctx_create(&cp, (int)ntot, 2, e->device, &e->c);
    if (rc) return rc;
    std::vector<int32_t> fo(ntot);
    for (int f = 0; f < nf; ++f)
        for (int i = 0; i < foams[f].n; ++i) fo[e->hpo[f] + i] = f;
    FOS_CUDA(cudaMalloc(&e->df, nf * sizeof(EnsFoamDev)));
    FOS_CUDA(cudaMalloc(&e->dw, nf * sizeof(EnsWords)));
    FOS_CUDA(cudaMalloc(&e->dvo, (nf + 1) * sizeof(long long)));
    FOS_CUDA(cudaMalloc(&e->foam_of, ntot * 4));
    FOS_CUDA(cudaMemcpy(e->df, e->hf.data(), nf * sizeof(EnsFoamDev), cudaMemcpyHostToDevice));
    FOS_CUDA(cudaMemset(e->dw, 0, nf * sizeof(EnsWords)));
    FOS_CUDA(cudaMemcpy(e->dvo, e->hvo.data(), (nf + 1) * sizeof(long long),
                        cudaMemcpyHostToDevice));
    FOS_CUDA(cudaMemcpy(e->foam_of, fo.data(), ntot * 4, cudaMemcpyHostToDevice));
    FOS_CUDA(cudaMalloc(&e->labA, vtot * 4));
    FOS_CUDA(cudaMalloc(&e->labB, vtot * 4));
    FOS_CUDA(cudaMalloc(&e->filt, vtot * 4));
    FOS_CUDA(cudaMalloc(&e->recA, vtot * sizeof(float4)));
    FOS_CUDA(cudaMalloc(&e->recB, vtot * sizeof(float4)));
    FOS_CUDA(cudaMalloc(&e->slot, vtot * 8));
    FOS_CUDA(cudaMalloc(&e->seedlin, ntot * 4));
    FOS_CUDA(cudaMemset(e->labA, 0xFF, vtot * 4));
    FOS_CUDA(cudaMemset(e->labB, 0xFF, vtot * 4));
    FOS_CUDA(cudaMemset(e->filt, 0xFF, vtot * 4));
    float** fbufs[] = {&e->pos, &e->rad, &e->rad_target, &e->lmd, &e->delta_r};
    size_t fsz[] = {(size_t)ntot * 12, (size_t)ntot * 4, (size_t)ntot * 4, (size_t)ntot * 4,
                    (size_t)ntot * 4};
    for (int k = 0; k < 5; ++k) {
        FOS_CUDA(cudaMalloc(fbufs[k], fsz[k]));
        FOS_CUDA(cudaMemset(*fbufs[k], 0, fsz[k]));
    }
    FOS_CUDA(cudaMalloc(&e->cc, (size_t)g3 * 4));
    FOS_CUDA(cudaMalloc(&e->cs, (size_t)g3 * 4));
    FOS_CUDA(cudaMalloc(&e->ci, (size_t)ntot * 4));
    FOS_CUDA(cudaMemset(e->cc, 0, (size_t)g3 * 4));
    FOS_CUDA(cudaMemset(e->cs, 0, (size_t)g3 * 4));
    FOS_CUDA(cudaMemset(e->ci, 0, (size_t)ntot * 4));
    if (e->fp.ou_jitter) {
        std::vector<uint2> key(nf);
        for (int f = 0; f < nf; ++f) key[f] = make_uint2(e->hf[f].k0, e->hf[f].k1);
        FOS_CUDA(cudaMalloc(&e->vjit, (size_t)ntot * 12));
        FOS_CUDA(cudaMemset(e->vjit, 0, (size_t)ntot * 12));
        FOS_CUDA(cudaMalloc(&e->ou_kick, nf * sizeof(float)));
        FOS_CUDA(cudaMalloc(&e->ou_key, nf * sizeof(uint2)));
        FOS_CUDA(cudaMalloc(&e->ou_base, nf * sizeof(int32_t)));
        FOS_CUDA(cudaMemcpy(e->ou_key, key.data(), nf * sizeof(uint2), cudaMemcpyHostToDevice));
        FOS_CUDA(cudaMemcpy(e->ou_base, e->hpo.data(), nf * sizeof(int32_t),
                            cudaMemcpyHostToDevice));
    }
    return FOS_OK;
}

extern "C" int fos_ensemble_create(const FosParams* p, const FosFrameParams* fp,
                                   const FosEnsembleFoam* foams, int nfoams, int device,
                                   FosEnsemble** out) {
    FOS_REQUIRE(out != nullptr, FOS_E_ARG, "out is NULL");
    *out = nullptr;
    FOS_REQUIRE(p && fp && foams, FOS_E_ARG, "NULL argument");
    FOS_REQUIRE(nfoams >= 1 && nfoams <= 65536, FOS_E_ARG, "nfoams must be in [1, 65536]");
    FOS_REQUIRE(p->early_exit == 0, FOS_E_ARG, "ensembles run every pass: early_exit must be 0");
    FOS_REQUIRE(fp->max_eq_nei <= 16, FOS_E_ARG, "ensembles need max_eq_nei <= 16");
    FOS_REQUIRE(!fp->ou_jitter || fp->pbd_iters >= 1, FOS_E_ARG,
                "ensembles run the OU jitter inside a PBD sweep: pbd_iters >= 1");
    for (int f = 0; f < nfoams; ++f) {
        int rc = ens_check_foam(foams[f]);
        if (rc) return rc;
    }
    FOS_CUDA(cudaSetDevice(device));
    FosEnsemble* e = new FosEnsemble();
    e->nf = nfoams;
    e->device = device;
    e->p = *p;
    e->fp = *fp;
    int rc = ens_create_impl(e, foams);
    if (rc) {
        fos_ensemble_destroy(e);
        return rc;
    }
    *out = e;
    return FOS_OK;
}

extern "C" int fos_ensemble_view(FosEnsemble* e, FosEnsembleView* v) {
    FOS_REQUIRE(e && v, FOS_E_ARG, "NULL argument");
    v->nfoams = e->nf;
    v->n_total = e->ntot;
    v->pos = e->pos;
    v->rad = e->rad;
    v->rad_target = e->rad_target;
    v->local_max_depth = e->lmd;
    v->delta_r = e->delta_r;
    v->fsc = e->c->fsc;
    v->fsc_ema = e->c->ema;
    v->face_ids = e->c->face_ids;
    v->face_counts = e->c->face_counts;
    v->neighbor_list = e->c->nl;
    v->labels_a = e->labA;
    v->labels_b = e->labB;
    v->foam_of = e->foam_of;
    return FOS_OK;
}

extern "C" int fos_ensemble_offsets(FosEnsemble* e, int* part_off, long long* vox_off,
                                    int* cell_off) {
    FOS_REQUIRE(e != nullptr, FOS_E_ARG, "ensemble is NULL");
    for (int f = 0; f <= e->nf; ++f) {
        if (part_off) part_off[f] = e->hpo[f];
        if (vox_off) vox_off[f] = e->hvo[f];
        if (cell_off) cell_off[f] = e->hco[f];
    }
    return FOS_OK;
}

extern "C" int fos_ensemble_set_tuning(FosEnsemble* e, const FosEnsembleTuning* t) {
    FOS_REQUIRE(e && t, FOS_E_ARG, "NULL argument");
    auto ok_blk = [](int b) { return b == 128 || b == 256 || b == 512; };
    FOS_REQUIRE(ok_blk(t->pass_block) && ok_blk(t->voxel_block), FOS_E_ARG,
                "pass_block / voxel_block must be 128, 256 or 512");
    FOS_REQUIRE(t->coop_threads == 512 || t->coop_threads == 1024, FOS_E_ARG,
                "coop_threads must be 512 or 1024");
    FOS_REQUIRE(t->coop_blocks_per_sm == 1 || t->coop_blocks_per_sm == 2, FOS_E_ARG,
                "coop_blocks_per_sm must be 1 or 2");
    e->tune = *t;
    return FOS_OK;
}

extern "C" int fos_ensemble_get_tuning(FosEnsemble* e, FosEnsembleTuning* t) {
    FOS_REQUIRE(e && t, FOS_E_ARG, "NULL argument");
    *t = e->tune;
    return FOS_OK;
}

extern "C" long long fos_ensemble_launch_count(FosEnsemble* e) { return e ? e->c->launches : 0; }

extern "C" int fos_ensemble_frame_index(FosEnsemble* e, int* frame, fos_stream_t s) {
    FOS_REQUIRE(e && frame, FOS_E_ARG, "NULL argument");
    int settle = 0;
    return fos_sim_counters(e->c, frame, &settle, s);
}

// Resident blocks of the dynamics kernel for a (threads, blocks/SM) shape, 0
// when it cannot be resident.
static int ens_coop_blocks(FosEnsemble* e, int threads, int per_sm_want) {
    int per_sm = 0;
    const size_t smem = e->g3tot <= COOP_SMALL_G3 ? (size_t)(e->g3tot + 1) * 4 : 0;
    cudaError_t err =
        threads == 1024
            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_coop<1024>, 1024, smem)
            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_coop<512>, 512, smem);
    if (err != cudaSuccess || per_sm < per_sm_want) return 0;
    int blocks = per_sm_want * e->c->num_sms;
    return blocks > 1024 ? 1024 : blocks;
}

static int ens_coop_launch(FosEnsemble* e, int mode, cudaStream_t s,
                           unsigned long long* trace = nullptr, int trace_cap = 0) {
    FosCtx* c = e->c;
    int threads = e->tune.coop_threads;
    int blocks = ens_coop_blocks(e, threads, e->tune.coop_blocks_per_sm);
    if (blocks == 0) {  // the tuned shape is not resident here: fall back to one block per SM
        threads = 1024;
        blocks = ens_coop_blocks(e, 1024, 1);
    }
    FOS_REQUIRE(blocks > 0, FOS_E_CUDA, "ensemble dynamics kernel cannot be resident");
    const FosFrameParams* fp = &e->fp;
    EnsArgs a;
    memset(&a, 0, sizeof(a));
    a.n = e->ntot;
    a.G3 = e->g3tot;
    a.chunk = (e->g3tot + blocks - 1) / blocks;
    a.small_grid = e->g3tot <= COOP_SMALL_G3 ? 1 : 0;
    a.cc = e->cc;
    a.cs = e->cs;
    a.ci = e->ci;
    a.cellof = c->cellof;
    a.rank = c->rank;
    a.ci_tmp = c->ci_tmp;
    a.cnt = c->coop_cnt;
    a.cnt2 = c->coop_cnt2;
    a.cfix = c->coop_fixed ? c->coop_cfix : nullptr;
    a.idsort = c->coop_idsort;
    a.spfix = c->coop_spfix;
    a.spst = c->coop_spst;
    a.slot_of = c->coop_slot;
    a.part = c->coop_part;
    a.bsum = c->coop_bsum;
    a.sp = c->sorted;
    a.ds = c->ds;
    a.F = e->df;
    a.foam_of = e->foam_of;
    a.W = e->dw;
    a.nf = e->nf;
    a.mode = mode;
    a.pbd_iters = fp->pbd_iters;
    a.sweeps = fp->pressure_iters;
    a.warmup = fp->warmup_pbd;
    a.bp_mode = fp->bp_mode;
    a.pos = e->pos;
    a.pos_tmp = c->pos_tmp;
    a.rad = e->rad;
    a.rad_tmp = c->rad_tmp;
    a.rad_target = e->rad_target;
    a.lmd = e->lmd;
    a.delta_r = e->delta_r;
    a.vol0 = c->pvol;
    a.vol1 = c->pvol + c->max_n;
    a.pnbr = c->pnbr;
    a.gap1 = c->gap1;
    a.mdf = c->mdf;
    a.dmul = c->dmul;
    a.eps = c->eps;
    a.contact_tol = c->contact_tol;
    a.contact_tol_d = c->p.contact_tol;
    const int af = fp->adjustment_frames > 1 ? fp->adjustment_frames : 1;
    a.alpha = (float)(1.0 - pow(0.05, 1.0 / (double)af));
    a.max_step = (float)fp->max_step_pct;
    a.pa = PressureArgs{e->ntot, 0, fp->max_eq_nei, (float)fp->pressure_k, (float)fp->pressure_exp,
                        (float)fp->pressure_pair_cap, 0.f, 0.f, c->face_ids, c->fsc, 0};
    a.strength = (float)fp->brownian_strength;
    a.domain = c->L;
    a.L = c->L;
    a.invL = c->invL;
    a.halfL = (float)(0.5 * (double)c->L);
    a.ou = fp->ou_jitter ? 1 : 0;
    a.vjit = e->vjit;
    a.ou_kick = e->ou_kick;
    a.ou_key = e->ou_key;
    a.ou_base = e->ou_base;
    a.ou_p = ou_params(fp->jitter_rms, fp->jitter_tau, fp->max_drift_fraction, c->p.gap_fraction,
                       (float)fp->dt, c->L, c->invL, 0);
    a.trace = trace;
    a.trace_cap = trace_cap;
    k_ens_coop_prep<<<fos_blocks(e->nf > 0 ? e->nf : 1, 256), 256, 0, s>>>(c->ds, e->dw, e->nf);
    FOS_LAUNCHED(c);
    // count buffers 0 and 1 of the frame's rebuilds (the kernel clears buffer 2
    // itself; the warm-up form uses buffer 0 and coop_cnt2)
    FOS_CUDA(cudaMemsetAsync(c->coop_cnt, 0, 2 * (size_t)e->g3tot * sizeof(int32_t), s));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = a.small_grid ? (size_t)(e->g3tot + 1) * 4 : 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (threads == 1024) FOS_CUDA(cudaLaunchKernelEx(&cfg, k_ens_coop<1024>, a));
    else FOS_CUDA(cudaLaunchKernelEx(&cfg, k_ens_coop<512>, a));
    FOS_LAUNCHED(c);
    return FOS_OK;
}

static int ens_kernel_attributes() {
    static bool done = false;
    if (done) return FOS_OK;
    FOS_CUDA(cudaFuncSetAttribute(k_ens_coop<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (COOP_SMALL_G3 + 1) * 4));
    FOS_CUDA(cudaFuncSetAttribute(k_ens_coop<512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (COOP_SMALL_G3 + 1) * 4));
    done = true;
    return FOS_OK;
}

extern "C" int fos_ensemble_init(FosEnsemble* e, int frame0, fos_stream_t s_) {
    FOS_REQUIRE(e != nullptr, FOS_E_ARG, "ensemble is NULL");
    cudaStream_t s = (cudaStream_t)s_;
    FosCtx* c = e->c;
    FOS_CUDA(cudaSetDevice(e->device));
    int rc = ens_kernel_attributes();
    if (rc) return rc;
    const size_t n = e->ntot, NS = n * FOS_S;
    FOS_CUDA(cudaMemsetAsync(c->fsc, 0, n * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->used, 0, n * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->ema, 0, n * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->face_ids, 0, NS * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->face_counts, 0, NS * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->prev, 0, NS * 4, s));
    FOS_CUDA(cudaMemsetAsync(c->nl, 0xFF, NS * 4, s));
    FOS_CUDA(cudaMemsetAsync(e->lmd, 0, n * 4, s));
    FOS_CUDA(cudaMemsetAsync(e->delta_r, 0, n * 4, s));
    FOS_CUDA(cudaMemsetAsync(e->dw, 0, e->nf * sizeof(EnsWords), s));
    if (e->vjit) FOS_CUDA(cudaMemsetAsync(e->vjit, 0, n * 12, s));
    FOS_CUDA(cudaMemcpyAsync(e->rad_target, e->rad, n * 4, cudaMemcpyDeviceToDevice, s));
    k_frame_set<<<1, 1, 0, s>>>(c->ds, frame0, 0);
    FOS_LAUNCHED(c);
    rc = fos_launch_wrap(c, e->pos, e->ntot, s);
    if (rc) return rc;
    if (e->fp.warmup_pbd > 0) {
        rc = ens_coop_launch(e, 1, s);
        if (rc) return rc;
    }
    return FOS_OK;
}

// jfa_init + every pass index (one launch each for all foams).
static int ens_seed_passes(FosEnsemble* e, cudaStream_t s) {
    FosCtx* c = e->c;
    const int n = e->ntot;
    const int nb = fos_blocks(n, 256);
    FOS_CUDA(cudaMemsetAsync(e->labA, 0xFF, (size_t)e->vtot * 4, s));
    k_ens_seed_prepare<<<nb, 256, 0, s>>>(e->df, e->foam_of, e->pos, e->rad, n, c->halfL, c->L,
                                          c->beta, c->seeds, e->seedlin, e->slot);
    FOS_LAUNCHED(c);
    if (c->L == 1.0f)
        k_ens_seed_min<true><<<nb, 256, 0, s>>>(e->df, e->foam_of, c->seeds, e->seedlin, n,
                                                c->halfL, c->L, e->slot);
    else
        k_ens_seed_min<false><<<nb, 256, 0, s>>>(e->df, e->foam_of, c->seeds, e->seedlin, n,
                                                 c->halfL, c->L, e->slot);
    FOS_LAUNCHED(c);
    k_ens_seed_write<<<nb, 256, 0, s>>>(e->seedlin, n, e->slot, e->labA);
    FOS_LAUNCHED(c);
    const bool ul = c->L == 1.0f, tie = c->p.tie_lower_index != 0;
    const int pb = e->tune.pass_block;
    const int pgrid = (int)(e->vtot / pb);
    if (!tie) {
        // the reference's scan-order tie rule runs over the seed records
        int rb = fos_blocks(e->vtot, 256);
        if (rb > 8 * c->num_sms) rb = 8 * c->num_sms;
        k_ens_rec_from_labels<<<rb, 256, 0, s>>>(e->labA, c->seeds, e->recA, e->vtot);
        FOS_LAUNCHED(c);
        if (ul && e->multi_voxel) {
            for (const FosEnsemble::Run& r : e->runs) {
                const unsigned grid = (unsigned)(r.threads / 256);
                const long long* to = e->drto + r.to_base;
                const int32_t* rf = e->drfoam + r.foam_base;
                if (r.M == 4)
                    k_ens_jfa_pass_recx<4><<<grid, 256, 0, s>>>(to, rf, r.nr, e->df, e->labA,
                                                                e->labB, e->recA, e->recB,
                                                                c->halfL, e->dw, r.pass);
                else if (r.M == 2)
                    k_ens_jfa_pass_recx<2><<<grid, 256, 0, s>>>(to, rf, r.nr, e->df, e->labA,
                                                                e->labB, e->recA, e->recB,
                                                                c->halfL, e->dw, r.pass);
                else
                    k_ens_jfa_pass_recx<1><<<grid, 256, 0, s>>>(to, rf, r.nr, e->df, e->labA,
                                                                e->labB, e->recA, e->recB,
                                                                c->halfL, e->dw, r.pass);
                FOS_LAUNCHED(c);
            }
            return FOS_OK;
        }
        for (int p = 0; p < e->max_passes; ++p) {
            if (ul)
                k_ens_jfa_pass_rec<true><<<pgrid, pb, 0, s>>>(e->dvo, e->nf, e->df, e->labA,
                                                              e->labB, e->recA, e->recB, c->halfL,
                                                              c->L, e->dw, p);
            else
                k_ens_jfa_pass_rec<false><<<pgrid, pb, 0, s>>>(e->dvo, e->nf, e->df, e->labA,
                                                               e->labB, e->recA, e->recB,
                                                               c->halfL, c->L, e->dw, p);
            FOS_LAUNCHED(c);
        }
        return FOS_OK;
    }
    for (int p = 0; p < e->max_passes; ++p) {
        if (ul && !tie)
            k_ens_jfa_pass<true, false><<<pgrid, pb, 0, s>>>(e->dvo, e->nf, e->df, e->labA, e->labB,
                                                             c->seeds, c->halfL, c->L, e->dw, p);
        else if (ul && tie)
            k_ens_jfa_pass<true, true><<<pgrid, pb, 0, s>>>(e->dvo, e->nf, e->df, e->labA, e->labB,
                                                            c->seeds, c->halfL, c->L, e->dw, p);
        else if (!tie)
            k_ens_jfa_pass<false, false><<<pgrid, pb, 0, s>>>(e->dvo, e->nf, e->df, e->labA,
                                                              e->labB, c->seeds, c->halfL, c->L,
                                                              e->dw, p);
        else
            k_ens_jfa_pass<false, true><<<pgrid, pb, 0, s>>>(e->dvo, e->nf, e->df, e->labA, e->labB,
                                                             c->seeds, c->halfL, c->L, e->dw, p);
        FOS_LAUNCHED(c);
    }
    return FOS_OK;
}

// Majority filter + face pairs into the candidate rows (not the rows' sort).
static int ens_filter_faces(FosEnsemble* e, cudaStream_t s) {
    FosCtx* c = e->c;
    const int n = e->ntot;
    const int vb = e->tune.voxel_block;
    const int vgrid = (int)(e->vtot / vb);
    k_ens_majority<<<vgrid, vb, 0, s>>>(e->dvo, e->nf, e->df, e->labA, e->labB, e->filt);
    FOS_LAUNCHED(c);
    k_faces_reset<<<fos_blocks(n, 256), 256, 0, s>>>(c->ds, c->rowcnt, n);
    FOS_LAUNCHED(c);
    bool tiles = true;  // every foam's R a multiple of 8
    for (const EnsFoamDev& d : e->hf) tiles = tiles && d.R % 8 == 0;
    if (tiles && e->vtot % FACES_TILE_THREADS == 0)
        k_ens_faces_tile<<<(unsigned)(e->vtot / FACES_TILE_THREADS), FACES_TILE_THREADS, 0, s>>>(
            e->dvo, e->nf, e->df, e->filt, n, c->hkeys, c->hmin, c->hcnt, c->claimed, c->ds,
            (unsigned long long)(c->H - 1));
    else
        k_ens_faces<<<vgrid, vb, 0, s>>>(e->dvo, e->nf, e->df, e->filt, n, c->hkeys, c->hmin,
                                         c->hcnt, c->claimed, c->ds,
                                         (unsigned long long)(c->H - 1));
    FOS_LAUNCHED(c);
    k_compact<<<c->num_sms * 8, 256, 0, s>>>(c->hkeys, c->hmin, c->hcnt, c->claimed, c->ds,
                                             c->rowcnt, c->rowbuf);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// Rows, the cooperative finalize + EMA, per-foam zero counts, gate + targets.
static int ens_finalize_targets(FosEnsemble* e, cudaStream_t s) {
    FosCtx* c = e->c;
    const int n = e->ntot;
    const int nb = fos_blocks(n, 256);
    k_rows<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(n, c->rowcnt, c->rowbuf, c->face_ids,
                                                     c->face_counts, c->ds);
    FOS_LAUNCHED(c);
    k_fin_reset<<<nb, 256, 0, s>>>(c->ds, c->fin_changed, c->revcnt, c->revfill, n);
    FOS_LAUNCHED(c);
    k_ens_scores<<<fos_blocks((long long)n * FOS_S, 256), 256, 0, s>>>(
        n, e->df, e->foam_of, c->face_ids, c->face_counts, e->rad, c->face_scale, c->t_add,
        c->face_score, c->acc0, c->revcnt);
    FOS_LAUNCHED(c);
    int rc = fos_scan_exclusive(c, c->revcnt, c->revstart, n, true, s);
    if (rc) return rc;
    k_rev_fill<<<fos_blocks((long long)n * FOS_S, 256), 256, 0, s>>>(n, c->face_ids, c->face_score,
                                                                     c->revstart, c->revfill, c->rev);
    FOS_LAUNCHED(c);
    k_rev_sort<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(n, c->revstart, c->rev);
    FOS_LAUNCHED(c);
    int per_sm = 0;
    FOS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_finalize, FIN_THREADS, 0));
    int grid = fos_blocks(32LL * n, FIN_THREADS), cap = per_sm * c->num_sms;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    const int max_it = n + 2 < FOS_FIN_MAXIT ? n + 2 : FOS_FIN_MAXIT;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(FIN_THREADS);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FOS_CUDA(cudaLaunchKernelEx(&cfg, k_finalize, n, (const int32_t*)c->revstart,
                                (const int32_t*)c->rev, c->acc0, c->acc1,
                                (const float*)c->face_score, (const int32_t*)c->face_ids, c->prev,
                                c->nl, c->used, c->fsc, c->ema, c->t_add, c->t_drop, c->ema_alpha, 1,
                                c->ds, c->fin_changed, max_it));
    FOS_LAUNCHED(c);
    k_ens_zero<<<nb, 256, 0, s>>>(n, c->fsc, e->foam_of, e->dw);
    FOS_LAUNCHED(c);
    const FosFrameParams* fp = &e->fp;
    k_ens_targets<<<nb, 256, 0, s>>>(n, e->df, e->foam_of, e->dw, c->ds, e->rad, e->rad_target,
                                     c->fsc, c->ema, (float)fp->growth_pct, c->deadband,
                                     fp->warmstart_frames, fp->zero_rate_thresh,
                                     fp->adjustment_frames);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

static int ens_jfa(FosEnsemble* e, cudaStream_t s) {
    k_ens_jfa_prep<<<fos_blocks(e->nf, 256), 256, 0, s>>>(e->dw, e->nf);
    FOS_LAUNCHED(e->c);
    int rc = ens_seed_passes(e, s);
    if (rc) return rc;
    rc = ens_filter_faces(e, s);
    if (rc) return rc;
    return ens_finalize_targets(e, s);
}

extern "C" int fos_ensemble_trace(FosEnsemble* e, long long* ns_host, int cap, int* count,
                                  fos_stream_t s_) {
    FOS_REQUIRE(e && ns_host && count && cap >= 3, FOS_E_ARG, "NULL argument or cap < 3");
    cudaStream_t s = (cudaStream_t)s_;
    int rc = ens_kernel_attributes();
    if (rc) return rc;
    unsigned long long* d = nullptr;
    FOS_CUDA(cudaMalloc(&d, (size_t)cap * 8));
    cudaError_t e0 = cudaMemsetAsync(d, 0, (size_t)cap * 8, s);
    rc = e0 == cudaSuccess ? ens_coop_launch(e, 0, s, d, cap)
                           : fos_cuda_fail(e0, "cudaMemsetAsync", __FILE__, __LINE__);
    if (rc == FOS_OK) {
        cudaError_t e1 = cudaMemcpyAsync(ns_host, d, (size_t)cap * 8, cudaMemcpyDeviceToHost, s);
        if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(s);
        if (e1 != cudaSuccess) rc = fos_cuda_fail(e1, "trace readback", __FILE__, __LINE__);
    }
    cudaFree(d);
    int k = 0;
    while (rc == FOS_OK && k < cap - 2 && ns_host[k] != 0) ++k;
    *count = k;
    return rc;
}

extern "C" int fos_ensemble_frame(FosEnsemble* e, int jfa_frame, fos_stream_t s_) {
    FOS_REQUIRE(e != nullptr, FOS_E_ARG, "ensemble is NULL");
    cudaStream_t s = (cudaStream_t)s_;
    int rc = ens_kernel_attributes();
    if (rc) return rc;
    rc = ens_coop_launch(e, 0, s);
    if (rc) return rc;
    if (jfa_frame) {
        rc = ens_jfa(e, s);
        if (rc) return rc;
    }
    k_frame_end<<<1, 1, 0, s>>>(e->c->ds);
    FOS_LAUNCHED(e->c);
    return FOS_OK;
}

// A frame of every foam with the learned FSC surrogate (fos_frame_surrogate's
// order per foam): the dynamics, then on a non-JFA frame the surrogate's FSC,
// its EMA and the targets from it; on a JFA frame the surrogate's estimate
// for the same positions, the JFA and its targets, then the judging.  Pairs
// are searched on each foam's own grid, so each foam's FSC is the one the
// same foam gets alone.  No reference counterpart.
extern "C" int fos_ensemble_frame_surrogate(FosEnsemble* e, const FosSurrogate* m, int jfa_frame,
                                            fos_stream_t s_) {
    FOS_REQUIRE(e != nullptr && m != nullptr, FOS_E_ARG, "ensemble or surrogate model is NULL");
    cudaStream_t s = (cudaStream_t)s_;
    FosCtx* c = e->c;
    int rc = ens_kernel_attributes();
    if (rc) return rc;
    rc = fos_sur_prepare(c);
    if (rc) return rc;
    rc = ens_coop_launch(e, 0, s);
    if (rc) return rc;
    const SurEnsGrid g{e->ntot, e->pos,     e->rad, e->cs,     e->cc,
                       e->ci,   e->foam_of, e->dfG, e->dfcell, e->dfrmax};
    if (!jfa_frame) {
        rc = fos_sur_ens_between(c, m, g, s);
        if (rc) return rc;
        const FosFrameParams* fp = &e->fp;
        k_ens_targets<<<fos_blocks(e->ntot, 256), 256, 0, s>>>(
            e->ntot, e->df, e->foam_of, e->dw, c->ds, e->rad, e->rad_target, fos_sur_fsc_int(c),
            c->ema, (float)fp->growth_pct, c->deadband, fp->warmstart_frames,
            fp->zero_rate_thresh, fp->adjustment_frames);
        FOS_LAUNCHED(c);
    } else {
        rc = fos_sur_ens_before_jfa(c, m, g, s);
        if (rc) return rc;
        rc = ens_jfa(e, s);
        if (rc) return rc;
        rc = fos_sur_frame_judge(c, e->ntot, s);
        if (rc) return rc;
    }
    k_frame_end<<<1, 1, 0, s>>>(c->ds);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// The surrogate mode (FOS_SUR_ABSOLUTE / FOS_SUR_ANCHORED) and the counters
// of the last pair build and judged JFA frame, over all foams.
extern "C" int fos_ensemble_surrogate_mode(FosEnsemble* e, int mode) {
    FOS_REQUIRE(e != nullptr, FOS_E_ARG, "ensemble is NULL");
    return fos_surrogate_set_mode(e->c, mode);
}

extern "C" int fos_ensemble_surrogate_stats(FosEnsemble* e, FosSurrogateStats* out,
                                            fos_stream_t s) {
    FOS_REQUIRE(e != nullptr, FOS_E_ARG, "ensemble is NULL");
    return fos_surrogate_stats(e->c, out, s);
}

extern "C" int fos_ensemble_frame_graph(FosEnsemble* e, int jfa_frame, fos_stream_t s_) {
    FOS_REQUIRE(e != nullptr, FOS_E_ARG, "ensemble is NULL");
    cudaStream_t s = (cudaStream_t)s_;
    FOS_CUDA(cudaSetDevice(e->device));
    int rc = ens_kernel_attributes();
    if (rc) return rc;
    const int g = jfa_frame ? 1 : 0;
    if (!e->gvalid[g] || memcmp(&e->gtune[g], &e->tune, sizeof(e->tune)) != 0) {
        if (e->gexec[g]) {
            cudaGraphExecDestroy(e->gexec[g]);
            e->gexec[g] = nullptr;
            e->gvalid[g] = false;
        }
        cudaStream_t cap;
        FOS_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        long long before = e->c->launches;
        cudaError_t err = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (err != cudaSuccess) {
            cudaStreamDestroy(cap);
            return fos_cuda_fail(err, "cudaStreamBeginCapture", __FILE__, __LINE__);
        }
        rc = fos_ensemble_frame(e, jfa_frame, cap);
        cudaGraph_t graph = nullptr;
        err = cudaStreamEndCapture(cap, &graph);
        cudaStreamDestroy(cap);
        long long captured = e->c->launches - before;
        e->c->launches = before;
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (err != cudaSuccess) return fos_cuda_fail(err, "cudaStreamEndCapture", __FILE__, __LINE__);
        err = cudaGraphInstantiate(&e->gexec[g], graph, 0);
        cudaGraphDestroy(graph);
        if (err != cudaSuccess) return fos_cuda_fail(err, "cudaGraphInstantiate", __FILE__, __LINE__);
        e->gtune[g] = e->tune;
        e->gvalid[g] = true;
        e->glaunch[g] = captured;
    }
    FOS_CUDA(cudaGraphLaunch(e->gexec[g], s));
    e->c->launches += e->glaunch[g];
    return FOS_OK;
}

// ------------------------------------------------------------ autotuner
// Mean milliseconds of `reps` runs of fn after one untimed run.
template <class Fn>
static int ens_time(cudaStream_t s, int reps, Fn fn, float* ms_out) {
    cudaEvent_t a, b;
    FOS_CUDA(cudaEventCreate(&a));
    FOS_CUDA(cudaEventCreate(&b));
    int rc = fn();
    if (rc == FOS_OK) {
        cudaEventRecord(a, s);
        for (int r = 0; r < reps && rc == FOS_OK; ++r) rc = fn();
        cudaEventRecord(b, s);
        cudaError_t err = cudaEventSynchronize(b);
        float ms = 0.f;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, a, b);
        if (err != cudaSuccess && rc == FOS_OK) rc = fos_cuda_fail(err, "autotune timing", __FILE__, __LINE__);
        *ms_out = ms / (float)(reps > 0 ? reps : 1);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

extern "C" int fos_ensemble_autotune(FosEnsemble* e, int reps, FosEnsembleTuning* best,
                                     float* report_ms, int report_cap, fos_stream_t s_) {
    FOS_REQUIRE(e != nullptr, FOS_E_ARG, "ensemble is NULL");
    FOS_REQUIRE(reps >= 1 && reps <= 1000, FOS_E_ARG, "reps must be in [1, 1000]");
    cudaStream_t s = (cudaStream_t)s_;
    FOS_CUDA(cudaSetDevice(e->device));
    int rc = ens_kernel_attributes();
    if (rc) return rc;
    FosCtx* c = e->c;
    const FosEnsembleTuning keep = e->tune;
    FosEnsembleTuning t = keep;
    std::vector<float> rep;
    const int blocks[3] = {128, 256, 512};
    const int n = e->ntot;
    const int nb = fos_blocks(n, 256);
    // (a) JFA passes: seed + every pass (idempotent: the seed resets buffer A)
    float best_ms = 1e30f;
    for (int k = 0; k < 3; ++k) {
        e->tune.pass_block = blocks[k];
        float ms = 0.f;
        rc = ens_time(s, reps, [&]() -> int { return ens_seed_passes(e, s); }, &ms);
        if (rc) break;
        rep.push_back(ms);
        if (ms < best_ms) {
            best_ms = ms;
            t.pass_block = blocks[k];
        }
    }
    // (b) majority filter + face extraction (reset, faces, compact: idempotent)
    best_ms = 1e30f;
    for (int k = 0; k < 3 && rc == FOS_OK; ++k) {
        e->tune.voxel_block = blocks[k];
        float ms = 0.f;
        rc = ens_time(s, reps, [&]() -> int { return ens_filter_faces(e, s); }, &ms);
        if (rc) break;
        rep.push_back(ms);
        if (ms < best_ms) {
            best_ms = ms;
            t.voxel_block = blocks[k];
        }
    }
    // (c) dynamics from a snapshot of the mutable state, restored after each run
    if (rc == FOS_OK) {
        const size_t nn = (size_t)n;
        struct Buf {
            void* p;
            size_t bytes;
        } bufs[] = {{e->pos, nn * 12},          {e->rad, nn * 4},   {e->lmd, nn * 4},
                    {e->delta_r, nn * 4},       {e->dw, e->nf * sizeof(EnsWords)},
                    {c->ds, sizeof(FosDevState)}};
        const int nbuf = 6;
        std::vector<void*> snap(nbuf, nullptr);
        for (int k = 0; k < nbuf && rc == FOS_OK; ++k) {
            cudaError_t err = cudaMalloc(&snap[k], bufs[k].bytes);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(snap[k], bufs[k].p, bufs[k].bytes, cudaMemcpyDeviceToDevice, s);
            if (err != cudaSuccess) rc = fos_cuda_fail(err, "autotune snapshot", __FILE__, __LINE__);
        }
        const int shapes[4][2] = {{512, 1}, {512, 2}, {1024, 1}, {1024, 2}};
        best_ms = 1e30f;
        for (int k = 0; k < 4 && rc == FOS_OK; ++k) {
            if (ens_coop_blocks(e, shapes[k][0], shapes[k][1]) == 0) {
                rep.push_back(-1.f);
                continue;
            }
            e->tune.coop_threads = shapes[k][0];
            e->tune.coop_blocks_per_sm = shapes[k][1];
            float ms = 0.f;
            rc = ens_time(s, reps, [&]() -> int {
                for (int q = 0; q < nbuf; ++q)
                    FOS_CUDA(cudaMemcpyAsync(bufs[q].p, snap[q], bufs[q].bytes,
                                             cudaMemcpyDeviceToDevice, s));
                return ens_coop_launch(e, 0, s);
            }, &ms);
            if (rc) break;
            rep.push_back(ms);
            if (ms < best_ms) {
                best_ms = ms;
                t.coop_threads = shapes[k][0];
                t.coop_blocks_per_sm = shapes[k][1];
            }
        }
        for (int q = 0; q < nbuf; ++q) {
            if (snap[q] && rc == FOS_OK)
                cudaMemcpyAsync(bufs[q].p, snap[q], bufs[q].bytes, cudaMemcpyDeviceToDevice, s);
        }
        cudaStreamSynchronize(s);
        for (int q = 0; q < nbuf; ++q)
            if (snap[q]) cudaFree(snap[q]);
    }
    if (rc) {
        e->tune = keep;
        return rc;
    }
    e->tune = t;
    if (best) *best = t;
    if (report_ms)
        for (int k = 0; k < report_cap && k < (int)rep.size(); ++k) report_ms[k] = rep[k];
    return FOS_OK;
}

// Record passes of the batched ensemble with four voxels a thread (on, the
// default) or one; no reference counterpart.  Both give the same labels.
extern "C" int fos_ensemble_set_multi_voxel(FosEnsemble* e, int on) {
    FOS_REQUIRE(e, FOS_E_ARG, "ensemble is NULL");
    e->multi_voxel = on ? 1 : 0;
    e->gvalid[0] = e->gvalid[1] = false;  // the graphs are recaptured on next use
    return FOS_OK;
}
