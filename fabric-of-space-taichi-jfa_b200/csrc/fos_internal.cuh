// fos_internal.cuh -- context layout, error plumbing and device arithmetic
// shared by the libfos.so translation units.
//
// Every FP32 expression that decides a label, a face or a neighbour is written
// with explicit round-to-nearest intrinsics (__fadd_rn, __fmul_rn, ...) in the
// operator order of the reference's Taichi source, so nvcc can never contract
// it into an FMA; the library is also built with -fmad=false for the rest.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "fos.h"

#define FOS_S 32          // MAX_NEIGHBORS (jfa.py:74)
#define FOS_ROWCAP 64     // candidate partners kept per particle before the 32-slot cut
#define FOS_FIN_MAXIT 4096
#define FOS_BAR_CYCLE_LIMIT 2000000000LL  // ~1 s at the B200's 1.965 GHz SM clock
#define FOS_BAR_TEST_CYCLES 2000000LL      // ~1 ms: the bound under fos_test_barrier_plan

// ----------------------------------------------------------- device state
// Small per-context block in device memory: the frame counters the frame
// graph reads, the JFA early-exit bookkeeping, and error/diagnostic words.
struct FosDevState {
    int frame;          // device frame index (pressure hash, Brownian counter, warm gate)
    int settle;         // settle_frames_left (run.py:744-750, 1231)
    int error;          // first device-side error code (FOS_E_*), 0 = none
    int passes_done;    // JFA passes actually run
    int final_buf;      // 0: labels in buffer A, 1: in buffer B
    int early_exited;
    int pair_count;     // distinct {a,b} pairs claimed in the pair table
    int row_overflow;   // particles with more than FOS_ROWCAP candidate partners
    int max_rowcnt;
    int fin_iters;      // fixed-point sweeps of the exact finalize
    int zero_fsc;       // particles with fsc == 0 after finalize
    int changed;        // pressure: particles with |dr| > 1e-12 (last sweep)
    unsigned int maxabs_dr_bits;  // pressure: max |dr| of the last sweep (float bits)
    unsigned int omax_bits;       // max overlap depth (float bits)
    unsigned int bar_count;       // grid barrier arrival counter
    unsigned int bar_gen;         // grid barrier generation
    int grid_ovf;                 // bit p: a fixed-capacity cell row of count buffer p overflowed
    unsigned long long rad_sum;   // OU jitter: sum of the radii, 2^-40 fixed point
    int tile_count;               // fos_dirty_count: marked tiles
    unsigned int coop_epoch;      // cooperative frame launches (tags of the pressure words)
    unsigned int rmax_bits;       // cooperative frame: largest radius before the PBD sweeps
    unsigned int rmax0_bits;      // cooperative frame: largest radius at the frame's start
    int bar_test;                 // fos_test_barrier_plan: 0, or the barrier a block leaves at
    unsigned long long changes[FOS_MAX_PASSES];
};

struct FosGraphKey {
    FosState st;
    FosFrameParams fp;
    const FosSurrogate* sur;
    int sur_mode;
    int jfa;
    int res;
    FosParams p;
};

struct FosSurBufs;  // surrogate.cu

// A batched ensemble's packed grid as the surrogate's pair search sees it.
struct SurEnsGrid {
    int n;
    const float* pos;
    const float* rad;
    const int32_t* cs;
    const int32_t* cc;
    const int32_t* ci;
    const int32_t* foam_of;
    const int32_t* fG;     // [nf] hash-grid cells a side
    const int32_t* fcell;  // [nf] first cell in the packed table
    const float* frmax;    // [nf] radius bound
};

#define FOS_SKIP_BLOCKS 1024
#define FOS_PTAG_MAX_N 32768  // particles the tagged pressure words are allocated for
#define FOS_PTAG_SWEEPS 64    // most sweeps they hold (one word per particle and sweep)
#define FOS_GRAPH_SLOTS 6
// block size of the cooperative finalize kernel (one warp per row); 1024
// threads at <= 32 registers keep two blocks (64 warps) on every SM and only
// 296 blocks at each grid barrier
#ifndef FIN_THREADS
#define FIN_THREADS 1024
#endif

struct FosCtx {
    int device = 0;
    int max_n = 0, max_res = 0;
    int num_sms = 0;
    FosParams p{};
    // resolution-derived (jfa.py:207-227)
    int res = 0, passes = 0;
    float vs = 0.f;
    // folded constants (Python floats -> f32 as Taichi folds them)
    float L = 1.f, halfL = 0.5f, invL = 1.f, beta = 1.f;
    float face_scale = 1.5f, t_add = 0.15f, t_drop = 0.10f, ema_alpha = 0.33f;
    float gap1 = 1.015f, mdf = 0.2f, dmul = 2.f, eps = 1e-8f, contact_tol = 0.035f;
    float deadband = 1.f;
    int G = 3;
    // JFA fields
    int32_t *labA = nullptr, *labB = nullptr, *filt = nullptr;
    float4 *recA = nullptr, *recB = nullptr;  // seed records mirroring labA / labB
    unsigned long long* seedslot = nullptr;
    float4* seeds = nullptr;
    int32_t *fsc = nullptr, *used = nullptr;
    float* ema = nullptr;
    int32_t *face_ids = nullptr, *face_counts = nullptr, *nl = nullptr;
    float *face_score = nullptr, *prev = nullptr;
    uint8_t *acc0 = nullptr, *acc1 = nullptr;
    // pair table
    size_t H = 0;
    unsigned long long* hkeys = nullptr;
    unsigned int *hmin = nullptr, *hcnt = nullptr, *claimed = nullptr;
    int32_t* rowcnt = nullptr;
    uint4* rowbuf = nullptr;
    int32_t *revcnt = nullptr, *revstart = nullptr, *revfill = nullptr, *rev = nullptr;
    // scratch
    int32_t* scan_tmp = nullptr;      // block sums for the multi-block scan
    size_t scan_tmp_n = 0;
    float* pos_tmp = nullptr;         // [max_n*3]
    float4* sorted = nullptr;         // [max_n] (x, y, z, r) in hash-cell order
    float* rad_tmp = nullptr;         // [max_n]
    int32_t *cellof = nullptr, *rank = nullptr;   // [max_n]
    int32_t* cell_tmp = nullptr;      // [G^3]  (scatter's copy of cell_write)
    int32_t *coop_cnt = nullptr, *coop_part = nullptr;  // [G^3] cooperative rebuild scratch
    int32_t* coop_cnt2 = nullptr;     // [G^3] second count buffer (rebuilds alternate)
    int32_t *coop_cfix = nullptr, *coop_idsort = nullptr;  // [G^3 * COOP_CAP] cell rows
    float4* coop_spfix = nullptr;     // [G^3 * COOP_CAP] (pos, rad) by cell row
    float4* coop_spst = nullptr;      // [G^3 * COOP_CAP] (pos, rad) in arrival order
    int coop_fixed = 0;               // the fixed-capacity rows are allocated
    int32_t* coop_slot = nullptr;     // [max_n] slot of each particle in the last rebuild
    float* pvol = nullptr;            // [2 * max_n] r^P ping-pong of the pressure sweeps
    int32_t* pnbr = nullptr;          // [16 * max_n] a frame's pressure neighbours (sweeps with barriers)
    // tagged r^P words of the cooperative frame's barrier-free pressure sweeps:
    // [(FOS_PTAG_SWEEPS + 1) * ptag_n], zeroed at creation
    unsigned long long* ptag = nullptr;
    int ptag_n = 0;
    int32_t* coop_bsum = nullptr;     // [1024]
    int32_t* ci_tmp = nullptr;        // [max_n]
    int use_coop = 1;                 // plain-frame dynamics as one cooperative kernel
    // tensor maps (CUtensorMap, 128 bytes each) over recA / recB for the
    // staged JFA pass (jfa.cu), encoded for resolution tm_res
    unsigned char tm_rec[2][128] = {};
    int tm_res = 0, tm_ok = 0;
    int use_tma = 0;                  // staged record rows in the JFA pass (off: it measured slower)
    int use_recx = 1;                 // JFA record pass with several voxels a thread along x
    int sur_tc = 1;                   // surrogate inference on tcgen05 (1) or mma.sync (0)
    int coop_blocks = -1;             // resident blocks of the cooperative kernel (-1: not queried)
    size_t cell_tmp_n = 0;
    float* stats_f = nullptr;         // device stats scratch
    int32_t* stats_i = nullptr;
    FosDevState* ds = nullptr;
    int* fin_changed = nullptr;       // [FOS_FIN_MAXIT] per-sweep change flags of the finalize
    void* pinned = nullptr;           // small host staging buffer
    void* skip_part = nullptr;        // fos_skip_signals: FOS_SKIP_BLOCKS partials + result
    FosSurBufs* sur = nullptr;        // FSC surrogate pair/inference buffers (first use)
    int sur_mode = FOS_SUR_ABSOLUTE;  // how surrogate frames use the model (fos.h)
    // graphs, indexed by jfa_frame (0 none, 1 exact, 2 warm) + 3 * (surrogate frame)
    cudaGraphExec_t gexec[FOS_GRAPH_SLOTS] = {};
    FosGraphKey gkey[FOS_GRAPH_SLOTS];
    bool gvalid[FOS_GRAPH_SLOTS] = {};
    long long glaunch[FOS_GRAPH_SLOTS] = {};  // kernels per captured frame graph
    long long launches = 0;
};

// ------------------------------------------------------------- host errors
void fos_set_error(const std::string& msg);
int fos_fail(int code, const char* what);
int fos_cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define FOS_CUDA(call)                                                         \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) return fos_cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

#define FOS_LAUNCHED(ctx)                                                      \
    do {                                                                       \
        (ctx)->launches++;                                                     \
        cudaError_t e_ = cudaPeekAtLastError();                                \
        if (e_ != cudaSuccess) return fos_cuda_fail(e_, "kernel launch", __FILE__, __LINE__); \
    } while (0)

#define FOS_REQUIRE(cond, code, msg)                                           \
    do {                                                                       \
        if (!(cond)) return fos_fail((code), (msg));                           \
    } while (0)

inline int fos_blocks(long long work, int threads) {
    long long b = (work + threads - 1) / threads;
    return (int)(b < 1 ? 1 : b);
}

// Exclusive scan of n int32 values (d_in may equal d_out); d_out[n] gets the
// total when with_total.  Launch-count aware.
int fos_scan_exclusive(FosCtx* ctx, const int32_t* d_in, int32_t* d_out, int n, bool with_total,
                       cudaStream_t s);
int fos_jfa_finalize_ema(FosCtx* c, const float* rad, int n, cudaStream_t s);
int fos_grid_init_attributes();
bool fos_coop_supported(FosCtx* c);
void fos_sur_free(FosCtx* c);
int fos_sur_prepare(FosCtx* c);
int fos_sur_frame_before_jfa(FosCtx* c, const FosSurrogate* m, const FosState* st,
                             const FosFrameParams* fp, cudaStream_t s);
int fos_sur_frame_judge(FosCtx* c, int n, cudaStream_t s);
int fos_sur_frame_between(FosCtx* c, const FosSurrogate* m, const FosState* st,
                          const FosFrameParams* fp, cudaStream_t s);
int fos_sur_ens_between(FosCtx* c, const FosSurrogate* m, const SurEnsGrid& g, cudaStream_t s);
int fos_sur_ens_before_jfa(FosCtx* c, const FosSurrogate* m, const SurEnsGrid& g, cudaStream_t s);
const int32_t* fos_sur_fsc_int(FosCtx* c);
// end_frame: the kernel is the frame's last one and advances the frame counter
// itself (k_frame_end's job).
int fos_frame_coop_dynamics(FosCtx* c, const FosState* st, const FosFrameParams* fp,
                            cudaStream_t s, unsigned long long* trace = nullptr,
                            int trace_cap = 0, int end_frame = 0);

// ------------------------------------------------------------ device math
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// jfa.wrapP (jfa.py:290-308): d - L*round(d/L).  With L == 1 the division and
// multiplication by L are exact identities, so the UNIT_L form is bit-identical.
template <bool UNIT_L>
__device__ __forceinline__ float jfa_wrap(float d, float L) {
    if (UNIT_L) return fsub(d, roundf(d));
    return fsub(d, fmul(L, roundf(fdiv(d, L))));
}

// power_distance_sq (jfa.py:450-477) against a seed (x, y, z, (beta*r)^2).
template <bool UNIT_L>
__device__ __forceinline__ float power_dist(float vx, float vy, float vz, float4 s, float L) {
    float dx = jfa_wrap<UNIT_L>(fsub(vx, s.x), L);
    float dy = jfa_wrap<UNIT_L>(fsub(vy, s.y), L);
    float dz = jfa_wrap<UNIT_L>(fsub(vz, s.z), L);
    float d2 = fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
    return fsub(d2, s.w);
}

// power_distance_sq for L == 1 using rintf (round half to even, one
// instruction) in place of roundf: the two differ only when d is exactly a
// half-integer, where d - round(d) is +-0.5 either way, and the distance uses
// only its square.  So the returned value is bit-identical to power_dist<true>.
__device__ __forceinline__ float power_dist_unit(float vx, float vy, float vz, float4 s) {
    float dx = fsub(vx, s.x);
    float dy = fsub(vy, s.y);
    float dz = fsub(vz, s.z);
    dx = fsub(dx, rintf(dx));
    dy = fsub(dy, rintf(dy));
    dz = fsub(dz, rintf(dz));
    float d2 = fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
    return fsub(d2, s.w);
}

// Packed float32 pairs (Blackwell add/sub/mul .f32x2): each half is the
// IEEE round-to-nearest result of its own pair, so a packed op equals two
// fsub / fmul bit for bit at half the issue slots.
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
    float2 o;
    asm("{\n\t.reg .b64 ra, rb, rc;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rc, ra, rb;\n\tmov.b64 {%0, %1}, rc;\n\t}"
        : "=f"(o.x), "=f"(o.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return o;
}

__device__ __forceinline__ float2 f2mul(float2 a, float2 b) {
    float2 o;
    asm("{\n\t.reg .b64 ra, rb, rc;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rc, ra, rb;\n\tmov.b64 {%0, %1}, rc;\n\t}"
        : "=f"(o.x), "=f"(o.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return o;
}

// power_dist_unit with the x and y axes in packed pairs: the same roundings
// in the same order, so the same float.
__device__ __forceinline__ float power_dist_unit2(float2 vxy, float vz, float4 s) {
    float2 d = f2sub(vxy, make_float2(s.x, s.y));
    float dz = fsub(vz, s.z);
    d = f2sub(d, make_float2(rintf(d.x), rintf(d.y)));
    dz = fsub(dz, rintf(dz));
    const float2 q = f2mul(d, d);
    float d2 = fadd(fadd(q.x, q.y), fmul(dz, dz));
    return fsub(d2, s.w);
}

__device__ __forceinline__ float2 f2add(float2 a, float2 b) {
    float2 o;
    asm("{\n\t.reg .b64 ra, rb, rc;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rc, ra, rb;\n\tmov.b64 {%0, %1}, rc;\n\t}"
        : "=f"(o.x), "=f"(o.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return o;
}

// power_dist_unit2 with each d - rint(d) done on the FMA pipe: for |d| < 2^22,
// (d + 1.5*2^23) - 1.5*2^23 is d rounded to the nearest integer with ties to
// even, which is rintf's value (only the sign of a zero result can differ, and
// d minus a zero is d either way up to the sign of zero, which squaring
// removes).  Voxel centres and seeds lie in [-L/2, L/2) with L = 1, so
// |d| < 1.  The distance is the same float as power_dist_unit2's, without the
// three XU-pipe rounds per candidate that held the record pass at 67 % of the
// XU pipe.
__device__ __forceinline__ float power_dist_unit2m(float2 vxy, float vz, float4 s) {
    const float M = 12582912.0f;
    float2 d = f2sub(vxy, make_float2(s.x, s.y));
    const float2 t = f2sub(f2add(d, make_float2(M, M)), make_float2(M, M));
    d = f2sub(d, t);
    float dz = fsub(vz, s.z);
    const float tz = fsub(fadd(dz, M), M);
    dz = fsub(dz, tz);
    const float2 q = f2mul(d, d);
    float d2 = fadd(fadd(q.x, q.y), fmul(dz, dz));
    return fsub(d2, s.w);
}

// power_dist_unit2m split for voxels that share y and z (several voxels a
// thread along x): the wrapped, squared y and z offsets of seed s once
// (pdist_yz2m), then each voxel's x term and the sum in power_dist_unit2m's
// order ((dx^2 + dy^2) + dz^2) - r^2, two voxels in packed pairs
// (pdist_x2m) or one (pdist_x1m).  The same roundings in the same order, so
// the same floats.
__device__ __forceinline__ float2 pdist_yz2m(float2 vyz, float4 s) {
    const float M = 12582912.0f;
    float2 d = f2sub(vyz, make_float2(s.y, s.z));
    const float2 t = f2sub(f2add(d, make_float2(M, M)), make_float2(M, M));
    d = f2sub(d, t);
    return f2mul(d, d);
}

__device__ __forceinline__ float2 pdist_x2m(float2 vx2, float2 qyz, float4 s) {
    const float M = 12582912.0f;
    float2 d = f2sub(vx2, make_float2(s.x, s.x));
    const float2 t = f2sub(f2add(d, make_float2(M, M)), make_float2(M, M));
    d = f2sub(d, t);
    const float2 a = f2add(f2mul(d, d), make_float2(qyz.x, qyz.x));
    const float2 b = f2add(a, make_float2(qyz.y, qyz.y));
    return f2sub(b, make_float2(s.w, s.w));
}

__device__ __forceinline__ float pdist_x1m(float vx, float2 qyz, float4 s) {
    const float M = 12582912.0f;
    float d = fsub(vx, s.x);
    const float t = fsub(fadd(d, M), M);
    d = fsub(d, t);
    return fsub(fadd(fadd(fmul(d, d), qyz.x), qyz.y), s.w);
}

// voxel_to_world (jfa.py:273-287)
__device__ __forceinline__ float voxel_centre(int idx, float vs, float halfL) {
    return fsub(fmul(fadd((float)idx, 0.5f), vs), halfL);
}

// grid.wrapP (grid.py:30-48): p - L*floor(p*INV_L + 0.5)
__device__ __forceinline__ float grid_wrap(float p, float L, float invL) {
    return fsub(p, fmul(L, floorf(fadd(fmul(p, invL), 0.5f))));
}

__device__ __forceinline__ int wrap_small(int v, int R) {  // |v| < 2R
    v += (v < 0) ? R : 0;
    v -= (v >= R) ? R : 0;
    return v;
}

__device__ __forceinline__ int wrap_mod(int v, int R) { return ((v % R) + R) % R; }

// wrap_mod for v in [-R, 2R) without integer division; anything outside
// (only a non-finite position can produce it) is clamped into [0, R).
__device__ __forceinline__ int wrap_near(int v, int R) {
    v += (v < 0) ? R : 0;
    v -= (v >= R) ? R : 0;
    return min(max(v, 0), R - 1);
}

// Order-preserving map of a float to uint32 (-0 folded onto +0 so that equal
// floats map to equal keys, matching the reference's strict '<').
__device__ __forceinline__ unsigned int float_order_key(float f) {
    f = __fadd_rn(f, 0.0f);  // -0 + +0 = +0 under round-to-nearest
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t h0 = __umulhi(0xD2511F53u, c.x), l0 = 0xD2511F53u * c.x;
        uint32_t h1 = __umulhi(0xCD9E8D57u, c.z), l1 = 0xCD9E8D57u * c.z;
        uint4 n;
        n.x = h1 ^ c.y ^ k0;
        n.y = l1;
        n.z = h0 ^ c.w ^ k1;
        n.w = l0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Software grid barrier for kernels launched cooperatively (all blocks
// co-resident).  ds->bar_count is reset to 0 before the launch and only grows:
// the e-th barrier of the launch is complete when bar_count reaches
// e*gridDim.x.  Thread 0 of each block arrives with a release reduction and
// polls with acquire loads, then releases its block; `epoch` is the caller's
// count of barriers passed (a register of thread 0, starting at 0).
// Bounded: a block that has waited ~1 s (clock64), or that sees the error word
// set, records FOS_E_TIMEOUT and returns false, so a stuck barrier ends the
// kernel instead of hanging the GPU.
// Test plan (ds->bar_test, set by fos_test_barrier_plan; 0 in normal use):
// when it holds k >= 2, the launch's last block leaves at its k-th barrier
// without arriving, and every barrier from the second on waits at most
// FOS_BAR_TEST_CYCLES, so the failure path runs in about a millisecond.
__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_gpu_add(unsigned int* p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

//
// The counter takes the low FOS_BAR_FLAG_SHIFT bits of ds->bar_count; the
// bits above are flags that a phase raises (atomicOr before its block arrives)
// for the phase after the barrier.  The poll that ends the barrier reads them
// with the count and hands them to the block in *flags, so no thread has to
// load a shared flag word of its own.
#define FOS_BAR_FLAG_SHIFT 26
#define FOS_BAR_COUNT_MASK ((1u << FOS_BAR_FLAG_SHIFT) - 1u)

//
// With nf > 0, thread 0 also loads the words *fetch[0..nf) (nf <= 4) after
// the barrier and the block gets them in fetched[]: one load per block of a
// word that every block wrote or reads, instead of one per warp of the same
// address.
__device__ __forceinline__ bool grid_barrier(FosDevState* ds, unsigned int& epoch,
                                             unsigned int* flags = nullptr,
                                             const unsigned int* const* fetch = nullptr,
                                             int nf = 0, unsigned int* fetched = nullptr) {
    __shared__ int s_ok;
    __shared__ unsigned int s_flags;
    __shared__ unsigned int s_fetch[4];
    // the launch's test plan (fos_test_barrier_plan), read by thread 0 while
    // it polls at the launch's first barrier and kept for the later ones
    __shared__ int s_test;
    __syncthreads();
    if (threadIdx.x == 0) {
        epoch += 1u;
        unsigned int target = epoch * gridDim.x;
        const bool planned = epoch >= 2u && s_test != 0;
        if (planned && (int)epoch == s_test && blockIdx.x == gridDim.x - 1) {
            // the planned failure: this block leaves without arriving, so the
            // others' bounded waits run out
            s_ok = 0;
            s_flags = 0u;
            for (int k = 0; k < nf; ++k) s_fetch[k] = 0u;
        } else {
        const long long limit = planned ? FOS_BAR_TEST_CYCLES : FOS_BAR_CYCLE_LIMIT;
        bool ok = true;
        red_release_gpu_add(&ds->bar_count, 1u);
        if (epoch == 1u) s_test = *((volatile int*)&ds->bar_test);
        long long t0 = clock64();
        unsigned int polls = 0;
        unsigned int v;
        while (((v = ld_acquire_gpu(&ds->bar_count)) & FOS_BAR_COUNT_MASK) < target) {
            // the error word and the clock are checked every 32 polls, so a
            // poll is one L2 round trip and the release is seen sooner
            if ((++polls & 31u) == 0u) {
                if (*((volatile int*)&ds->error) != 0 || clock64() - t0 > limit) {
                    atomicCAS(&ds->error, 0, (int)FOS_E_TIMEOUT);
                    ok = false;
                    break;
                }
                if (polls > 2048u) __nanosleep(32);
            }
        }
        s_ok = ok ? 1 : 0;
        s_flags = v >> FOS_BAR_FLAG_SHIFT;
        for (int k = 0; k < nf; ++k) s_fetch[k] = *((const volatile unsigned int*)fetch[k]);
        }
    }
    __syncthreads();
    if (flags) *flags = s_flags;
    for (int k = 0; k < nf; ++k) fetched[k] = s_fetch[k];
    return s_ok != 0;
}
