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
#include <cuda.h>
#include <math.h>
#include <string.h>

#include "jfa_body.cuh"

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

template <bool UNIT_L, bool POW2, bool TIE_LOWER>
__global__ void __launch_bounds__(256) k_jfa_pass(const int32_t* __restrict__ in,
                                                  int32_t* __restrict__ out,
                                                  const float4* __restrict__ seeds, int R, int lgR,
                                                  float vs, float halfL, float L, int step,
                                                  FosDevState* ds, int pass, int early_exit,
                                                  int min_passes, double th) {
    // Programmatic dependent launch (passes after the first): the next pass's
    // blocks may be scheduled once every block of this one has started, and
    // each block waits here until the previous pass has completed and its
    // labels and change counts are visible.  Without the launch attribute both
    // instructions return at once.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const long long V = (long long)R * R * R;
    if (early_exit && jfa_exited_before(ds, pass, (double)V, min_passes, th)) return;
    jfa_pass_body<UNIT_L, POW2, TIE_LOWER>(in, out, seeds, R, lgR, vs, halfL, L, step, ds->changes,
                                           pass, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Pass over the record grid (jfa_pass_rec_body); the same launch protocol as
// k_jfa_pass.  Six blocks per SM (at most 40 registers): the pass waits on
// record-load latency, so residency pays (stress passes 3.91 -> 3.73 ms).  The
// general-L distance needs more registers: four blocks per SM (64) for it,
// where six spilled 340 bytes per thread.
template <bool UNIT_L, bool POW2>
__global__ void __launch_bounds__(256, UNIT_L ? 6 : 4) k_jfa_pass_rec(const int32_t* __restrict__ in,
                                                      const float4* __restrict__ rin,
                                                      int32_t* __restrict__ out,
                                                      float4* __restrict__ rout, int R, int lgR,
                                                      float vs, float halfL, float L, int step,
                                                      FosDevState* ds, int pass, int early_exit,
                                                      int min_passes, double th) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const long long V = (long long)R * R * R;
    if (early_exit && jfa_exited_before(ds, pass, (double)V, min_passes, th)) return;
    jfa_pass_rec_body<UNIT_L, POW2>(in, rin, out, rout, R, lgR, vs, halfL, L, step, ds->changes,
                                    pass, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// ------------------------------------------------ M voxels a thread along x
// The record pass with M voxels a thread at x = xb, xb + s, ..., xb + (M-1)s
// (s the step; unit L, power-of-two R >= 16, R / s >= M).  Voxel m's
// candidates lie in the x-planes xb + (m-1)s .. xb + (m+1)s, so the thread
// reads the 9 rows of each of M + 2 planes once and every row serves up to
// three of its voxels: 9 (M + 2) + M record loads for M voxels instead of
// 27 M (M = 4: 58 against 108).  Lanes run along z, so each load is still a
// coalesced 512-byte row.  Planes are visited in increasing x and rows in
// (dy, dz) order, so each voxel sees its own record first and then the 26
// others in the reference's (dx, dy, dz) order, with the same arithmetic as
// jfa_rec_core.  HALF: the step is R / 2, where only the offsets {-1, 0}^3
// give distinct candidates (recx_scan).
template <int M, bool HALF = false>
__global__ void __launch_bounds__(256, 4)
    k_jfa_pass_recx(const int32_t* __restrict__ in, const float4* __restrict__ rin,
                    int32_t* __restrict__ out, float4* __restrict__ rout, int lgR, int lgS,
                    float vs, float halfL, FosDevState* ds, int pass, int early_exit,
                    int min_passes, double th) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int R = 1 << lgR, step = 1 << lgS;
    const long long V = (long long)R * R * R;
    if (early_exit && jfa_exited_before(ds, pass, (double)V, min_passes, th)) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;  // < R^3 / M
    const int z = t & (R - 1), y = (t >> lgR) & (R - 1), xi = t >> (2 * lgR);
    const int xb = ((xi >> lgS) * M << lgS) + (xi & (step - 1));
    int ys[3], zs[3], xp[M + 2];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int o = (k - 1) * step;
        ys[k] = ((y + o) & (R - 1)) << lgR;
        zs[k] = (z + o) & (R - 1);
    }
#pragma unroll
    for (int p = 0; p < M + 2; ++p) xp[p] = ((xb + (p - 1) * step) & (R - 1)) << (2 * lgR);
    const float vy = voxel_centre(y, vs, halfL), vz = voxel_centre(z, vs, halfL);
    float vx[M], bd[M];
    int bl[M], own[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int l = xp[m + 1] + ys[1] + zs[1];
        vx[m] = voxel_centre(xb + m * step, vs, halfL);
        own[m] = in[l];
        bd[m] = fminf(power_dist_unit2m(make_float2(vx[m], vy), vz, __ldg(&rin[l])), 1e10f);
        bl[m] = l;
    }
    recx_scan<M, HALF>(rin, xp, ys, zs, vx, vy, vz, bd, bl);
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int l = xp[m + 1] + ys[1] + zs[1];
        int best = own[m];
        if (bl[m] != l) best = in[bl[m]];
        out[l] = best;
        rout[l] = __ldg(&rin[bl[m]]);
        const int cnt = __syncthreads_count(best != own[m]);
        if (threadIdx.x == 0 && cnt) atomicAdd(&ds->changes[pass], (unsigned long long)cnt);
    }
}

// The same for any R (unit L, R / s >= M and R a multiple of M s): coordinates
// by division, wraps by compare-and-add, a tail of threads past R^3 / M.
template <int M, bool HALF = false>
__global__ void __launch_bounds__(256, 4)
    k_jfa_pass_recx_any(const int32_t* __restrict__ in, const float4* __restrict__ rin,
                        int32_t* __restrict__ out, float4* __restrict__ rout, int R, int step,
                        float vs, float halfL, FosDevState* ds, int pass, int early_exit,
                        int min_passes, double th) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const long long V = (long long)R * R * R;
    if (early_exit && jfa_exited_before(ds, pass, (double)V, min_passes, th)) return;
    const long long tl = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
    const float vy = voxel_centre(y, vs, halfL), vz = voxel_centre(z, vs, halfL);
    float vx[M], bd[M];
    int bl[M], own[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int l = xp[m + 1] + ys[1] + zs[1];
        vx[m] = voxel_centre(xb + m * step, vs, halfL);
        own[m] = in[l];
        bd[m] = fminf(power_dist_unit2m(make_float2(vx[m], vy), vz, __ldg(&rin[l])), 1e10f);
        bl[m] = l;
    }
    recx_scan<M, HALF>(rin, xp, ys, zs, vx, vy, vz, bd, bl);
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
        if (threadIdx.x == 0 && cnt) atomicAdd(&ds->changes[pass], (unsigned long long)cnt);
    }
}

// ------------------------------------------------ pass with staged record rows
// The same pass with the records a block needs staged in shared memory by
// the tensor memory accelerator (cp.async.bulk.tensor, no multicast), for
// unit L and power-of-two R in [32, 256].  A block takes TY = 256 / R
// consecutive (x, y) rows of R voxels; every candidate of its voxels lies in
// one of the 9 * TY whole z-rows (x + {-s, 0, s}, y + {-s, 0, s}), wrapped, so
// each is one tile copy of R records (a tensor map over the record grid as a
// [R][R][R][4] float array, box 1 x 1 x R x 4) and any step needs the same
// 36,864 bytes.  The z offsets wrap inside a row.  Candidates, their order and
// the arithmetic are those of jfa_rec_core; the winner's label is read from
// the global label grid and its record from the staged rows.  Off by
// default: 8 passes at 128^3 took 0.643 ms against 0.436 ms for the global
// rows (9 at 256^3: 5.26 against 3.73 ms).  The pass is held by the L1 /
// shared-memory data path (27 16-byte records a voxel either way) and FP32
// issue; the staging adds 144 bytes a voxel of shared-memory writes on that
// path and a load-then-compute bubble per block.
#define JFA_TMA_SMEM (9 * 256 * 16)

__device__ __forceinline__ unsigned int smem_addr(const void* p) {
    return (unsigned int)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_try_wait(unsigned int bar, unsigned int parity) {
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

// Waits for phase `parity` of the barrier for at most ~1 s of clock; false
// (and FOS_E_TIMEOUT in the error word) when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned int bar, unsigned int parity,
                                                  FosDevState* ds) {
    const long long t0 = clock64();
    for (unsigned int it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63u) == 0u && clock64() - t0 > FOS_BAR_CYCLE_LIMIT) {
            atomicCAS(&ds->error, 0, (int)FOS_E_TIMEOUT);
            return false;
        }
    }
}

__global__ void __launch_bounds__(256, 6)
    k_jfa_pass_tma(const __grid_constant__ CUtensorMap tmap, const int32_t* __restrict__ in,
                   const float4* __restrict__ rin, int32_t* __restrict__ out,
                   float4* __restrict__ rout, int lgR, float vs, float halfL, int step,
                   FosDevState* ds, int pass, int early_exit, int min_passes, double th) {
    extern __shared__ __align__(128) float4 srow[];
    __shared__ __align__(8) unsigned long long s_bar;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int R = 1 << lgR;
    const long long V = (long long)R * R * R;
    if (early_exit && jfa_exited_before(ds, pass, (double)V, min_passes, th)) return;
    const int TY = 256 >> lgR;
    const int NR = 9 * TY;
    const int q0 = blockIdx.x * TY;
    const int x0 = q0 >> lgR, y0 = q0 & (R - 1);
    const unsigned int bar = smem_addr(&s_bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"((unsigned int)(NR * R * 16))
                     : "memory");
    }
    __syncthreads();
    if ((int)threadIdx.x < NR) {  // row r: x offset ix, block row ty, y offset iy
        const int r = threadIdx.x;
        const int ix = r / (3 * TY), rem = r - ix * 3 * TY, ty = rem / 3, iy = rem - ty * 3;
        const int xr = (x0 + (ix - 1) * step) & (R - 1);
        const int yr = (y0 + ty + (iy - 1) * step) & (R - 1);
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(srow + (size_t)r * R)),
            "l"(reinterpret_cast<unsigned long long>(&tmap)), "r"(0), "r"(0), "r"(yr), "r"(xr),
            "r"(bar)
            : "memory");
    }
    if (!mbar_wait_bounded(bar, 0u, ds)) {
        mbar_wait_bounded(bar, 0u, ds);  // copies still in flight: give them one more bound
        return;
    }
    const int ty = threadIdx.x >> lgR, z = threadIdx.x & (R - 1);
    const int x = x0, y = y0 + ty;
    const int l = (x << (2 * lgR)) | (y << lgR) | z;
    int xs[3], ys[3], zs[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int o = (k - 1) * step;
        xs[k] = ((x + o) & (R - 1)) << (2 * lgR);
        ys[k] = ((y + o) & (R - 1)) << lgR;
        zs[k] = (z + o) & (R - 1);
    }
    const int own = in[l];
    const float4 orec = srow[(3 * TY + ty * 3 + 1) * R + z];
    const float vx = voxel_centre(x, vs, halfL), vy = voxel_centre(y, vs, halfL),
                vz = voxel_centre(z, vs, halfL);
    const float2 vxy = make_float2(vx, vy);
    float bd = fminf(power_dist_unit2m(vxy, vz, orec), 1e10f);
    int bl = l, bsm = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float4 r[9];
        int sm[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            sm[k] = (a * 3 * TY + ty * 3 + k / 3) * R + zs[k % 3];
            if (!(a == 1 && k == 4)) r[k] = srow[sm[k]];
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            if (a == 1 && k == 4) continue;  // the voxel itself
            const float d = power_dist_unit2m(vxy, vz, r[k]);
            if (d < bd) {
                bd = d;
                bl = xs[a] + ys[k / 3] + zs[k % 3];
                bsm = sm[k];
            }
        }
    }
    int best = own;
    float4 brec = orec;
    if (bl != l) {
        best = in[bl];
        brec = srow[bsm];
    }
    out[l] = best;
    rout[l] = brec;
    const int cnt = __syncthreads_count(best != own);
    if (threadIdx.x == 0 && cnt) atomicAdd(&ds->changes[pass], (unsigned long long)cnt);
}

// The record grid of a label grid: record v = seeds[label v], or NaN bits for
// an unassigned voxel.  Run before every sequence of record passes, so a grid
// from jfa_init, a warm start or loaded labels all start consistent with the
// current seed table.
__global__ void k_rec_from_labels(const int32_t* __restrict__ lab,
                                  const float4* __restrict__ seeds, float4* __restrict__ rec,
                                  long long V) {
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < V;
         l += (long long)gridDim.x * blockDim.x) {
        const int v = lab[l];
        rec[l] = v >= 0 ? __ldg(&seeds[v]) : rec_none();
    }
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
    majority_body(ds->final_buf ? labB : labA, R, outp,
                  (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Threads per face-extraction block: a block appends its claimed table slots
// once, after a block barrier, so smaller blocks wait on fewer warps.
#ifndef FACES_THREADS
#define FACES_THREADS 128
#endif

__global__ void __launch_bounds__(FACES_THREADS) k_faces(const int32_t* __restrict__ filt, int R, int n,
                                               unsigned long long* keys, unsigned int* hmin,
                                               unsigned int* hcnt, unsigned int* claimed,
                                               FosDevState* ds, unsigned long long mask) {
    __shared__ unsigned int s_slot[3 * FACES_THREADS];
    __shared__ int s_n;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const ClaimBuf cb{s_slot, &s_n, claimed};
    faces_body(filt, R, n, keys, hmin, hcnt, cb, ds, mask,
               (long long)blockIdx.x * blockDim.x + threadIdx.x);
    faces_claims_flush(cb, claimed, ds);
}

// Face extraction over voxel tiles of FACES_TILE_THREADS voxels with a per-block merge of the
// pairs (faces_tile_body; R a multiple of 8).
__global__ void __launch_bounds__(FACES_TILE_THREADS) k_faces_tile(
    const int32_t* __restrict__ filt, int R, int n, unsigned long long* keys, unsigned int* hmin,
    unsigned int* hcnt, unsigned int* claimed, FosDevState* ds, unsigned long long mask) {
    __shared__ unsigned int s_slot[3 * FACES_TILE_THREADS];
    __shared__ int s_n;
    if (threadIdx.x == 0) s_n = 0;
    const ClaimBuf cb{s_slot, &s_n, claimed};
    faces_tile_body(filt, R, n, keys, hmin, hcnt, cb, ds, mask, blockIdx.x);
    faces_claims_flush(cb, claimed, ds);
}

// Moves every claimed pair into its lower particle's candidate row and resets
// the table slot for the next run.  Launched with 8 blocks of 256 per SM (the
// full 2,048 threads at 32 registers): each pair is a chain of dependent
// loads and a returning atomic, so the number of chains in flight sets the
// time at a million pairs.
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
// One warp per particle a: the row's (<= 64) candidates sit in registers,
// two per lane; each one's rank (stable, by first-touch key) comes from
// shuffles, and ranks below 32 are the slots.
__global__ void __launch_bounds__(256) k_rows(int n, const int32_t* __restrict__ rowcnt,
                                              const uint4* __restrict__ rowbuf,
                                              int32_t* __restrict__ face_ids,
                                              int32_t* __restrict__ face_counts, FosDevState* ds) {
    const int a = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (a >= n) return;  // warp-uniform
    int m = rowcnt[a];
    if (lane == 0 && m > 0) atomicMax(&ds->max_rowcnt, m);
    if (m > FOS_ROWCAP) m = FOS_ROWCAP;
    const uint4 none = make_uint4(0xFFFFFFFFu, 0u, 0u, 0u);
    const size_t rb = (size_t)a * FOS_ROWCAP;
    const uint4 e0 = lane < m ? rowbuf[rb + lane] : none;
    const uint4 e1 = lane + 32 < m ? rowbuf[rb + lane + 32] : none;
    int r0 = 0, r1 = 0;
    const int m0 = m < 32 ? m : 32;
    for (int k = 0; k < m0; ++k) {
        const unsigned int kx = __shfl_sync(0xffffffffu, e0.x, k);
        r0 += (kx < e0.x) || (kx == e0.x && k < lane);
        r1 += (kx < e1.x) || (kx == e1.x);
    }
    for (int k = 32; k < m; ++k) {
        const unsigned int kx = __shfl_sync(0xffffffffu, e1.x, k - 32);
        r0 += kx < e0.x;
        r1 += (kx < e1.x) || (kx == e1.x && k < lane + 32);
    }
    const size_t o = (size_t)a * FOS_S;
    if (lane < m && r0 < FOS_S) {
        face_ids[o + r0] = (int)e0.y;
        face_counts[o + r0] = (int)e0.z;
    }
    if (lane + 32 < m && r1 < FOS_S) {
        face_ids[o + r1] = (int)e1.y;
        face_counts[o + r1] = (int)e1.z;
    }
    if (lane >= m) {
        face_ids[o + lane] = -1;
        face_counts[o + lane] = 0;
    }
}

// finalize scores per face slot (score_slot, jfa_body.cuh).
__global__ void k_scores(int n, const int32_t* __restrict__ face_ids,
                         const int32_t* __restrict__ face_counts, const float* __restrict__ rad,
                         float vs, float face_scale, float t_add, float* __restrict__ score,
                         uint8_t* acc, int32_t* revcnt) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * FOS_S) return;
    score_slot(t, n, face_ids, face_counts, rad, vs, face_scale, t_add, score, acc, revcnt);
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

// One warp per particle j sorts its reverse list ascending (values are
// distinct): up to 64 entries by shuffle ranks in registers, longer lists by
// lane 0's insertion sort.
__global__ void __launch_bounds__(256) k_rev_sort(int n, const int32_t* __restrict__ revstart,
                                                  int32_t* __restrict__ rev) {
    const int j = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= n) return;  // warp-uniform
    const int b = revstart[j], e = revstart[j + 1], len = e - b;
    if (len <= 1) return;
    if (len <= 64) {
        const int v0 = lane < len ? rev[b + lane] : 0x7fffffff;
        const int v1 = lane + 32 < len ? rev[b + lane + 32] : 0x7fffffff;
        int r0 = 0, r1 = 0;
        const int l0 = len < 32 ? len : 32;
        for (int k = 0; k < l0; ++k) {
            const int kv = __shfl_sync(0xffffffffu, v0, k);
            r0 += kv < v0;
            r1 += kv < v1;
        }
        for (int k = 32; k < len; ++k) {
            const int kv = __shfl_sync(0xffffffffu, v1, k - 32);
            r0 += kv < v0;
            r1 += kv < v1;
        }
        __syncwarp();
        if (lane < len) rev[b + r0] = v0;
        if (lane + 32 < len) rev[b + r1] = v1;
        return;
    }
    if (lane != 0) return;
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
//
// One warp per row, lane s holding face slot s.  fin_app gathers the first
// FOS_S accepted entries of row i's reverse list (sorted ascending, the serial
// append order): lane p receives the score and the source particle of the
// p-th one.  It returns how many were appended.
__device__ __forceinline__ int fin_app(int i, int lane, const int32_t* __restrict__ revstart,
                                       const int32_t* __restrict__ rev, const uint8_t* acc,
                                       const float* __restrict__ score, float& appv, int& appi) {
    const int b = revstart[i], e = revstart[i + 1];
    int used = 0;
    for (int k0 = b; k0 < e && used < FOS_S; k0 += 32) {  // warp-uniform
        const int k = k0 + lane;
        const int t = k < e ? rev[k] : 0;
        const bool a = k < e && __ldcg(&acc[t]);
        const unsigned m = __ballot_sync(0xffffffffu, a);
        const float st = a ? score[t] : 0.0f;
        const int cnt = __popc(m), d = lane - used;
        const bool mine = d >= 0 && d < cnt;
        const int src = mine ? (int)__fns(m, 0, d + 1) : lane;
        const float v = __shfl_sync(0xffffffffu, st, src);
        const int ti = __shfl_sync(0xffffffffu, t, src);
        if (mine) {
            appv = v;
            appi = ti >> 5;
        }
        used += cnt;
    }
    return used < FOS_S ? used : FOS_S;
}

// Decisions of row i's own slots (bit s = slot s accepted) after `used`
// appended entries.  ok = sc >= t_add, or sc >= t_drop and the score at
// neighbour-list slot s is >= t_drop: the s-th appended entry while s is
// below the running count (rev entries first, then this row's accepted slots
// in slot order), else the previous frame's score.  Slots in the band
// [t_drop, t_add) depend on the acceptances below them and are decided in
// slot order; the others are fixed by their score alone.
__device__ __forceinline__ unsigned fin_decide(int used, float sc, float pv, float appv,
                                               float t_add, float t_drop) {
    unsigned okm = __ballot_sync(0xffffffffu, sc >= 0.0f && sc >= t_add);
    unsigned band = __ballot_sync(0xffffffffu, sc >= 0.0f && !(sc >= t_add) && sc >= t_drop);
    while (band) {  // warp-uniform
        const int s = __ffs(band) - 1;
        band &= band - 1u;
        const int below = __popc(okm & ((1u << s) - 1u));
        int src = s;
        float v = pv;
        if (s < used) {
            v = appv;
        } else if (s < used + below) {
            src = (int)__fns(okm, 0, s - used + 1);
            v = sc;
        }
        if (__shfl_sync(0xffffffffu, v, src) >= t_drop) okm |= 1u << s;
    }
    return okm;
}

__global__ void __launch_bounds__(FIN_THREADS, 2048 / FIN_THREADS) k_finalize(int n, const int32_t* __restrict__ revstart,
                                                  const int32_t* __restrict__ rev,
                                                  uint8_t* acc0, uint8_t* acc1,
                                                  const float* __restrict__ score,
                                                  const int32_t* __restrict__ face_ids,
                                                  float* prev, int32_t* nl, int32_t* used_out,
                                                  int32_t* fsc, float* ema, float t_add,
                                                  float t_drop, float alpha, int apply_ema,
                                                  FosDevState* ds, int* fin_changed,
                                                  int max_iters) {
    const int lane = threadIdx.x & 31;
    const int wstride = gridDim.x * (blockDim.x >> 5);
    const int w0 = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;  // rows spread over all SMs
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    uint8_t* cur = acc0;
    uint8_t* nxt = acc1;
    int it = 0;
    unsigned int epoch = 0;
    for (;;) {
        int ch = 0;
        for (int i = w0; i < n; i += wstride) {
            const size_t o = (size_t)i * FOS_S + lane;
            const float sc = score[o];
            const float pv = prev[o];
            const uint8_t was = __ldcg(&cur[o]);
            float appv = 0.0f;
            int appi = 0;
            const int used = fin_app(i, lane, revstart, rev, cur, score, appv, appi);
            const uint8_t ok = (fin_decide(used, sc, pv, appv, t_add, t_drop) >> lane) & 1u;
            __stcg(&nxt[o], ok);
            ch |= ok != was;
        }
        if (__syncthreads_or(ch) && threadIdx.x == 0) atomicOr(&fin_changed[it], 1);
        if (!grid_barrier(ds, epoch)) return;
        int any = *((volatile int*)&fin_changed[it]);
        uint8_t* t = cur;
        cur = nxt;
        nxt = t;
        ++it;
        if (!any) break;
        if (it >= max_iters) {
            if (lead) atomicCAS(&ds->error, 0, (int)FOS_E_TIMEOUT);
            return;
        }
    }
    if (lead) ds->fin_iters = it;
    // Materialise the serial result from the converged decisions `cur`.  For
    // neighbour-list slot p the serial writes are: the previous score; the
    // p-th reverse append; then, in slot order, the append of this row's own
    // accepted slot of rank p - used0 (slot sa) and the zeroing of a rejected
    // slot p.  The later of the last two wins.
    for (int i = w0; i < n; i += wstride) {
        const size_t o = (size_t)i * FOS_S + lane;
        const float sc = score[o];
        const float pv = prev[o];
        const int fid = face_ids[o];
        const bool ok = sc >= 0.0f && __ldcg(&cur[o]);
        float appv = 0.0f;
        int appi = 0;
        const int used0 = fin_app(i, lane, revstart, rev, cur, score, appv, appi);
        const unsigned okm = __ballot_sync(0xffffffffu, ok);
        const int own = __popc(okm);
        const int used = used0 + own < FOS_S ? used0 + own : FOS_S;
        const int r = lane - used0;
        const bool app = r >= 0 && r < own;
        const int sa = app ? (int)__fns(okm, 0, r + 1) : lane;
        const float va = __shfl_sync(0xffffffffu, sc, sa);
        const int ia = __shfl_sync(0xffffffffu, fid, sa);
        const bool zero = sc >= 0.0f && !ok;
        float pr = lane < used0 ? appv : pv;
        if (app) pr = (zero && sa < lane) ? 0.0f : va;
        else if (zero) pr = 0.0f;
        prev[o] = pr;
        nl[o] = lane < used0 ? appi : (app ? ia : -1);
        if (lane == 0) {
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
static cudaError_t launch_pass(FosCtx* c, const int32_t* in, int32_t* out, int step,
                               int pass, int early_exit, cudaStream_t s) {
    const int R = c->res;
    long long V = (long long)R * R * R;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)fos_blocks(V, 256));
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    // a pass that follows a pass overlaps its launch with that pass's tail
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pass > 0 ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k_jfa_pass<UL, P2, TIE>, in, out, (const float4*)c->seeds,
                              R, ilog2(R), c->vs, c->halfL, c->L, step, c->ds, pass,
                              early_exit, c->p.min_jfa_passes, c->p.th_pass_delta);
}

template <bool UL, bool P2>
static cudaError_t launch_pass_rec(FosCtx* c, int p, int step, int early_exit, cudaStream_t s) {
    const int R = c->res;
    long long V = (long long)R * R * R;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)fos_blocks(V, 256));
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = p > 0 ? 1 : 0;
    const int32_t* in = (p & 1) ? c->labB : c->labA;
    int32_t* out = (p & 1) ? c->labA : c->labB;
    const float4* rin = (p & 1) ? c->recB : c->recA;
    float4* rout = (p & 1) ? c->recA : c->recB;
    return cudaLaunchKernelEx(&cfg, k_jfa_pass_rec<UL, P2>, in, rin, out, rout, R, ilog2(R),
                              c->vs, c->halfL, c->L, step, c->ds, p, early_exit,
                              c->p.min_jfa_passes, c->p.th_pass_delta);
}

static cudaError_t launch_pass_recx(FosCtx* c, int p, int step, int early_exit,
                                    cudaStream_t s) {
    const int R = c->res;
    const int lgS = ilog2(step);
    const int M = (R >> lgS) >= 4 ? 4 : 2;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(((long long)R * R * R / M) / 256));
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = p > 0 ? 1 : 0;
    const int32_t* in = (p & 1) ? c->labB : c->labA;
    int32_t* out = (p & 1) ? c->labA : c->labB;
    const float4* rin = (p & 1) ? c->recB : c->recA;
    float4* rout = (p & 1) ? c->recA : c->recB;
    if (M == 4)
        return cudaLaunchKernelEx(&cfg, k_jfa_pass_recx<4>, in, rin, out, rout, ilog2(R), lgS,
                                  c->vs, c->halfL, c->ds, p, early_exit, c->p.min_jfa_passes,
                                  c->p.th_pass_delta);
    if (2 * step == R)  // the first pass: only 8 distinct candidates a voxel
        return cudaLaunchKernelEx(&cfg, k_jfa_pass_recx<2, true>, in, rin, out, rout, ilog2(R), lgS,
                                  c->vs, c->halfL, c->ds, p, early_exit, c->p.min_jfa_passes,
                                  c->p.th_pass_delta);
    return cudaLaunchKernelEx(&cfg, k_jfa_pass_recx<2>, in, rin, out, rout, ilog2(R), lgS, c->vs,
                              c->halfL, c->ds, p, early_exit, c->p.min_jfa_passes,
                              c->p.th_pass_delta);
}

// Voxels a thread of the multi-voxel pass at any R and step s: 4 where R is a
// multiple of 4 s, 2 where it is a multiple of 2 s (the first pass, s = R/2,
// then scans its 8 distinct candidates), else 0 (the one-voxel pass runs).
static int recx_any_m(int R, int step) {
    return R % (4 * step) == 0 ? 4 : (R % (2 * step) == 0 ? 2 : 0);
}

static cudaError_t launch_pass_recx_any(FosCtx* c, int p, int step, int early_exit,
                                        cudaStream_t s) {
    const int R = c->res;
    const int M = recx_any_m(R, step);
    const long long V = (long long)R * R * R;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)fos_blocks(V / M, 256));
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = p > 0 ? 1 : 0;
    const int32_t* in = (p & 1) ? c->labB : c->labA;
    int32_t* out = (p & 1) ? c->labA : c->labB;
    const float4* rin = (p & 1) ? c->recB : c->recA;
    float4* rout = (p & 1) ? c->recA : c->recB;
    if (M == 4)
        return cudaLaunchKernelEx(&cfg, k_jfa_pass_recx_any<4>, in, rin, out, rout, R, step, c->vs,
                                  c->halfL, c->ds, p, early_exit, c->p.min_jfa_passes,
                                  c->p.th_pass_delta);
    if (2 * step == R)
        return cudaLaunchKernelEx(&cfg, k_jfa_pass_recx_any<2, true>, in, rin, out, rout, R, step,
                                  c->vs, c->halfL, c->ds, p, early_exit, c->p.min_jfa_passes,
                                  c->p.th_pass_delta);
    return cudaLaunchKernelEx(&cfg, k_jfa_pass_recx_any<2>, in, rin, out, rout, R, step, c->vs,
                              c->halfL, c->ds, p, early_exit, c->p.min_jfa_passes,
                              c->p.th_pass_delta);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return (EncodeTiledFn)p;
    }();
    return fn;
}

static bool tma_applies(const FosCtx* c) {
    const int R = c->res;
    return c->use_tma && c->L == 1.0f && is_pow2(R) && R >= 32 && R <= 256;
}

// The two record grids as [R][R][R][4] float tensors, box 1 x 1 x R x 4
// (one z-row of records), re-encoded when the resolution changes.
static bool tma_maps(FosCtx* c) {
    if (c->tm_res == c->res) return c->tm_ok != 0;
    c->tm_res = c->res;
    c->tm_ok = 0;
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t R = (cuuint64_t)c->res;
    const cuuint64_t dims[4] = {4, R, R, R};
    const cuuint64_t strides[3] = {16, 16 * R, 16 * R * R};
    const cuuint32_t box[4] = {4, (cuuint32_t)R, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    float4* bufs[2] = {c->recA, c->recB};
    for (int b = 0; b < 2; ++b) {
        CUtensorMap tm;
        if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, bufs[b], dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
            CUDA_SUCCESS)
            return false;
        memcpy(c->tm_rec[b], &tm, sizeof(tm));
    }
    static_assert(sizeof(CUtensorMap) == 128, "tensor map size");
    c->tm_ok = 1;
    return true;
}

static cudaError_t launch_pass_tma(FosCtx* c, int p, int step, int early_exit, cudaStream_t s) {
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k_jfa_pass_tma,
                                             cudaFuncAttributePreferredSharedMemoryCarveout,
                                             (int)cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    const int R = c->res;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(((long long)R * R * R) / 256));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = JFA_TMA_SMEM;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = p > 0 ? 1 : 0;
    const int32_t* in = (p & 1) ? c->labB : c->labA;
    int32_t* out = (p & 1) ? c->labA : c->labB;
    const float4* rin = (p & 1) ? c->recB : c->recA;
    float4* rout = (p & 1) ? c->recA : c->recB;
    CUtensorMap tm;
    memcpy(&tm, c->tm_rec[p & 1], sizeof(tm));
    return cudaLaunchKernelEx(&cfg, k_jfa_pass_tma, tm, in, rin, out, rout, ilog2(R), c->vs,
                              c->halfL, step, c->ds, p, early_exit, c->p.min_jfa_passes,
                              c->p.th_pass_delta);
}

// `npass` passes from labA, steps first_step, first_step/2, ... (never below 1).
// The reference's scan-order tie rule runs over the record grid; the
// lower-index tie rule (which compares labels on equal distances) runs over
// labels and seed gathers.
static int run_passes(FosCtx* c, int first_step, int npass, int early_exit, cudaStream_t s) {
    const int R = c->res;
    long long V = (long long)R * R * R;
    FOS_CUDA(cudaMemsetAsync(c->ds->changes, 0, sizeof(c->ds->changes), s));
    bool ul = (c->L == 1.0f), p2 = is_pow2(R), tie = c->p.tie_lower_index != 0;
    int step = first_step;
    if (!tie) {
        int blocks = fos_blocks(V, 256);
        if (blocks > 8 * c->num_sms) blocks = 8 * c->num_sms;
        k_rec_from_labels<<<blocks, 256, 0, s>>>(c->labA, c->seeds, c->recA, V);
        FOS_LAUNCHED(c);
        const bool tma = tma_applies(c) && tma_maps(c);
        // several voxels a thread where the grid still fills the GPU (at 64^3,
        // 65k threads: 0.084 against 0.077 ms for 7 passes), or when forced
        const bool multi = ul && R >= 16 &&
                           (c->use_recx == 2 ||
                            (c->use_recx == 1 && V / 4 >= (long long)c->num_sms * 1024));
        const bool recx = multi && p2;
        const bool recx_any = multi && !p2;
        for (int p = 0; p < npass; ++p) {
            if (step < 1) step = 1;
            cudaError_t le;
            if (recx_any && recx_any_m(R, step) > 0)
                le = launch_pass_recx_any(c, p, step, early_exit, s);
            else if (tma) le = launch_pass_tma(c, p, step, early_exit, s);
            else if (recx) le = launch_pass_recx(c, p, step, early_exit, s);
            else if (ul && p2) le = launch_pass_rec<true, true>(c, p, step, early_exit, s);
            else if (ul) le = launch_pass_rec<true, false>(c, p, step, early_exit, s);
            else if (p2) le = launch_pass_rec<false, true>(c, p, step, early_exit, s);
            else le = launch_pass_rec<false, false>(c, p, step, early_exit, s);
            if (le != cudaSuccess) return fos_cuda_fail(le, "kernel launch", __FILE__, __LINE__);
            FOS_LAUNCHED(c);
            step /= 2;
        }
        k_jfa_finish<<<1, 1, 0, s>>>(c->ds, npass, V, early_exit, c->p.min_jfa_passes,
                                     c->p.th_pass_delta);
        FOS_LAUNCHED(c);
        return FOS_OK;
    }
    for (int p = 0; p < npass; ++p) {
        if (step < 1) step = 1;
        const int32_t* in = (p & 1) ? c->labB : c->labA;
        int32_t* out = (p & 1) ? c->labA : c->labB;
        const int ee = early_exit;
        cudaError_t le;
        if (ul && p2 && !tie) le = launch_pass<true, true, false>(c, in, out, step, p, ee, s);
        else if (ul && p2 && tie) le = launch_pass<true, true, true>(c, in, out, step, p, ee, s);
        else if (ul && !p2 && !tie) le = launch_pass<true, false, false>(c, in, out, step, p, ee, s);
        else if (ul && !p2 && tie) le = launch_pass<true, false, true>(c, in, out, step, p, ee, s);
        else if (!ul && p2 && !tie) le = launch_pass<false, true, false>(c, in, out, step, p, ee, s);
        else if (!ul && p2 && tie) le = launch_pass<false, true, true>(c, in, out, step, p, ee, s);
        else if (!ul && !p2 && !tie) le = launch_pass<false, false, false>(c, in, out, step, p, ee, s);
        else le = launch_pass<false, false, true>(c, in, out, step, p, ee, s);
        if (le != cudaSuccess) return fos_cuda_fail(le, "kernel launch", __FILE__, __LINE__);
        FOS_LAUNCHED(c);
        step /= 2;
    }
    k_jfa_finish<<<1, 1, 0, s>>>(c->ds, npass, V, early_exit, c->p.min_jfa_passes,
                                 c->p.th_pass_delta);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_jfa_passes(FosCtx* c, int n, fos_stream_t s) {
    int rc = check_n(c, n);
    if (rc) return rc;
    return run_passes(c, c->res / 2, c->passes, c->p.early_exit, s);
}

// The previous run's final owner grid into labA (the warm start's input).
__global__ void k_take_final(int32_t* __restrict__ labA, const int32_t* __restrict__ labB,
                             const FosDevState* ds, long long V) {
    if (ds->final_buf == 0) return;  // already in labA
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < V;
         l += (long long)gridDim.x * blockDim.x)
        labA[l] = labB[l];
}

extern "C" int fos_jfa_warm(FosCtx* c, const float* pos, const float* rad, int n, int first_step,
                            fos_stream_t s) {
    int rc = check_n(c, n);
    if (rc) return rc;
    FOS_REQUIRE(n == 0 || (pos && rad), FOS_E_ARG, "pos/rad is NULL");
    const int R = c->res;
    FOS_REQUIRE(first_step >= 1 && first_step <= (R > 1 ? R / 2 : 1) && is_pow2(first_step),
                FOS_E_ARG, "first_step must be a power of two in [1, res/2]");
    const long long V = (long long)R * R * R;
    int blocks = fos_blocks(V, 256);
    if (blocks > 8 * c->num_sms) blocks = 8 * c->num_sms;
    k_take_final<<<blocks, 256, 0, s>>>(c->labA, c->labB, c->ds, V);
    FOS_LAUNCHED(c);
    if (n > 0) {
        // re-plant every seed at its current voxel over the previous owners
        int nb = fos_blocks(n, 256);
        k_seed_prepare<<<nb, 256, 0, s>>>(pos, rad, n, R, c->halfL, c->L, c->beta, c->seeds,
                                          c->cellof, c->seedslot);
        FOS_LAUNCHED(c);
        if (c->L == 1.0f)
            k_seed_min<true><<<nb, 256, 0, s>>>(c->seeds, c->cellof, n, R, c->vs, c->halfL, c->L,
                                               c->seedslot);
        else
            k_seed_min<false><<<nb, 256, 0, s>>>(c->seeds, c->cellof, n, R, c->vs, c->halfL, c->L,
                                                c->seedslot);
        FOS_LAUNCHED(c);
        k_seed_write<<<nb, 256, 0, s>>>(c->cellof, n, c->seedslot, c->labA);
        FOS_LAUNCHED(c);
    }
    return run_passes(c, first_step, ilog2(first_step) + 2, 0, s);
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
#ifndef FOS_FACES_TILE
#define FOS_FACES_TILE 1
#endif
    if (FOS_FACES_TILE && c->res % 8 == 0)
        k_faces_tile<<<(unsigned)(V / FACES_TILE_THREADS), FACES_TILE_THREADS, 0, s>>>(
            c->filt, c->res, n, c->hkeys, c->hmin, c->hcnt, c->claimed, c->ds,
            (unsigned long long)(c->H - 1));
    else
        k_faces<<<fos_blocks(V, FACES_THREADS), FACES_THREADS, 0, s>>>(c->filt, c->res, n, c->hkeys, c->hmin, c->hcnt,
                                               c->claimed, c->ds, (unsigned long long)(c->H - 1));
    FOS_LAUNCHED(c);
    k_compact<<<c->num_sms * 8, 256, 0, s>>>(c->hkeys, c->hmin, c->hcnt, c->claimed, c->ds,
                                             c->rowcnt, c->rowbuf);
    FOS_LAUNCHED(c);
    k_rows<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(n, c->rowcnt, c->rowbuf, c->face_ids,
                                                     c->face_counts,
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
    k_rev_sort<<<fos_blocks(32LL * n, 256), 256, 0, s>>>(n, c->revstart, c->rev);
    FOS_LAUNCHED(c);
    // one warp per row, as many co-resident blocks as the rows fill
    int per_sm = 0;
    FOS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_finalize, FIN_THREADS, 0));
    int grid = fos_blocks(32LL * n, FIN_THREADS);
    int cap = per_sm * c->num_sms;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    int max_it = n + 2 < FOS_FIN_MAXIT ? n + 2 : FOS_FIN_MAXIT;
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

// Staged record rows in the JFA pass (k_jfa_pass_tma) on or off; no
// reference counterpart.  Both give the same labels.
extern "C" int fos_set_jfa_staging(FosCtx* c, int on) {
    FOS_REQUIRE(c, FOS_E_ARG, "ctx is NULL");
    c->use_tma = on ? 1 : 0;
    return FOS_OK;
}

// Record pass form: 0 one voxel a thread (k_jfa_pass_rec), 1 several voxels
// a thread along x (k_jfa_pass_recx) where R^3 / 4 threads fill the GPU, 2
// always several; no reference counterpart.  All give the same labels.
extern "C" int fos_set_jfa_multi_voxel(FosCtx* c, int mode) {
    FOS_REQUIRE(c, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(mode >= 0 && mode <= 2, FOS_E_ARG, "mode must be 0, 1 or 2");
    c->use_recx = mode;
    return FOS_OK;
}
