// fos_ctx.cu -- context lifetime, parameters, resolution, errors, scan.
//
// The context plays the role of jfa.py's module-level Taichi fields
// (jfa.py:120-204): everything is allocated once, at capacity, when the
// context is created, and nothing is allocated afterwards.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <cstdlib>
#include <string>

#include "fos_internal.cuh"

static thread_local std::string g_last_error;

void fos_set_error(const std::string& msg) { g_last_error = msg; }

int fos_fail(int code, const char* what) {
    g_last_error = std::string(fos_status_string(code)) + ": " + what;
    return code;
}

int fos_cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e),
             what, file, line);
    g_last_error = buf;
    return FOS_E_CUDA;
}

extern "C" const char* fos_last_error(void) { return g_last_error.c_str(); }

extern "C" const char* fos_status_string(int status) {
    switch (status) {
        case FOS_OK: return "FOS_OK";
        case FOS_E_ARG: return "FOS_E_ARG";
        case FOS_E_CAPACITY: return "FOS_E_CAPACITY";
        case FOS_E_CUDA: return "FOS_E_CUDA";
        case FOS_E_TIMEOUT: return "FOS_E_TIMEOUT";
        case FOS_E_DEVICE: return "FOS_E_DEVICE";
        case FOS_E_STATE: return "FOS_E_STATE";
        default: return "FOS_E_UNKNOWN";
    }
}

extern "C" void fos_params_default(FosParams* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->domain_size = 0.189;          // config.py:21
    p->grid_res = 3;
    p->power_beta = 1.0;             // config.py:143
    p->early_exit = 1;               // config.py:208
    p->min_jfa_passes = 3;           // config.py:210
    p->th_pass_delta = 0.006;        // config.py:209
    p->tie_lower_index = 0;
    p->expected_face_scale = 1.5;    // jfa.py:58
    p->t_add = 0.15;                 // jfa.py:63
    p->t_drop = 0.10;                // jfa.py:64
    p->ema_alpha = 0.33;             // config.py:81
    p->gap_fraction = 0.015;         // config.py:353
    p->max_displacement_frac = 0.2;  // config.py:349
    p->displacement_multiplier = 2.0;// config.py:350
    p->eps = 1e-8;                   // config.py:324
    p->contact_tol = 0.035;          // config.py:254
    p->fsc_deadband = 1.0;           // config.py:100
}

static void fold_params(FosCtx* c) {
    const FosParams& p = c->p;
    // Taichi folds Python-scope constant expressions in double, then bakes an f32.
    c->L = (float)p.domain_size;
    c->halfL = (float)(0.5 * p.domain_size);      // HALF_L (config.py:213) / 0.5*L
    c->invL = (float)(1.0 / p.domain_size);       // INV_L (config.py:214)
    c->beta = (float)p.power_beta;
    c->face_scale = (float)p.expected_face_scale;
    c->t_add = (float)p.t_add;
    c->t_drop = (float)p.t_drop;
    c->ema_alpha = (float)p.ema_alpha;
    c->gap1 = (float)(1.0 + p.gap_fraction);      // (1.0 + GAP_FRACTION), dynamics.py:132
    c->mdf = (float)p.max_displacement_frac;
    c->dmul = (float)p.displacement_multiplier;
    c->eps = (float)p.eps;
    c->contact_tol = (float)p.contact_tol;
    c->deadband = (float)p.fsc_deadband;
    c->G = p.grid_res;
}

// Fixed-capacity cell rows of the cooperative rebuilds (32 slots a cell) are
// allocated while they stay below this size; larger grids use the CSR form.
#define FOS_COOP_FIXED_MAX_BYTES (1ull << 31)

static int alloc_cells(FosCtx* c) {
    size_t need = (size_t)c->G * c->G * c->G;
    if (need <= c->cell_tmp_n) return FOS_OK;
    int32_t** bufs[4] = {&c->cell_tmp, &c->coop_cnt, &c->coop_part, &c->coop_cnt2};
    for (int32_t** b : bufs) {
        if (*b) cudaFree(*b);
        *b = nullptr;
    }
    void* rows[4] = {c->coop_cfix, c->coop_idsort, c->coop_spfix, c->coop_spst};
    for (void* q : rows)
        if (q) cudaFree(q);
    c->coop_cfix = c->coop_idsort = nullptr;
    c->coop_spfix = c->coop_spst = nullptr;
    c->coop_fixed = 0;
    // coop_cnt holds three count buffers: the single-foam kernel rotates them
    for (int32_t** b : bufs)
        FOS_CUDA(cudaMalloc((void**)b, (b == &c->coop_cnt ? 3 : 1) * need * sizeof(int32_t)));
    FOS_CUDA(cudaMemset(c->coop_cnt, 0, 3 * need * sizeof(int32_t)));
    FOS_CUDA(cudaMemset(c->coop_cnt2, 0, need * sizeof(int32_t)));
    const size_t slots = need * 32;
    if (slots * (4 + 4 + 2 * sizeof(float4)) <= FOS_COOP_FIXED_MAX_BYTES) {
        FOS_CUDA(cudaMalloc((void**)&c->coop_cfix, slots * 4));
        FOS_CUDA(cudaMalloc((void**)&c->coop_idsort, slots * 4));
        FOS_CUDA(cudaMalloc((void**)&c->coop_spfix, slots * sizeof(float4)));
        FOS_CUDA(cudaMalloc((void**)&c->coop_spst, slots * sizeof(float4)));
        c->coop_fixed = 1;
    }
    c->cell_tmp_n = need;
    return FOS_OK;
}

static int check_params(const FosParams* p) {
    FOS_REQUIRE(p != nullptr, FOS_E_ARG, "params is NULL");
    FOS_REQUIRE(p->domain_size > 0.0, FOS_E_ARG, "domain_size must be > 0");
    FOS_REQUIRE(p->grid_res >= 3 && p->grid_res <= 1024, FOS_E_ARG, "grid_res must be in [3, 1024]");
    FOS_REQUIRE(p->min_jfa_passes >= 1, FOS_E_ARG, "min_jfa_passes must be >= 1");
    return FOS_OK;
}

extern "C" int fos_set_params(FosCtx* c, const FosParams* p) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    int rc = check_params(p);
    if (rc) return rc;
    FOS_CUDA(cudaSetDevice(c->device));
    c->p = *p;
    fold_params(c);
    for (int k = 0; k < FOS_GRAPH_SLOTS; ++k) c->gvalid[k] = false;
    return alloc_cells(c);
}

static size_t next_pow2(size_t v) {
    size_t r = 1;
    while (r < v) r <<= 1;
    return r;
}

extern "C" int fos_ctx_create(const FosParams* p, int max_n, int max_res, int device, FosCtx** out) {
    FOS_REQUIRE(out != nullptr, FOS_E_ARG, "out is NULL");
    *out = nullptr;
    int rc = check_params(p);
    if (rc) return rc;
    FOS_REQUIRE(max_n >= 1 && max_n <= (1 << 24), FOS_E_ARG, "max_n must be in [1, 2^24]");
    FOS_REQUIRE(max_res >= 2 && max_res <= 512, FOS_E_ARG, "max_res must be in [2, 512]");
    FOS_CUDA(cudaSetDevice(device));
    FosCtx* c = new FosCtx();
    c->device = device;
    c->max_n = max_n;
    c->max_res = max_res;
    c->p = *p;
    fold_params(c);
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    size_t V = (size_t)max_res * max_res * max_res;
    size_t NS = (size_t)max_n * FOS_S;
    c->H = next_pow2((size_t)max_n * 16);
#define ALLOC(ptr, bytes)                                                     \
    do {                                                                      \
        cudaError_t e_ = cudaMalloc((void**)&(ptr), (bytes));                 \
        if (e_ != cudaSuccess) {                                              \
            fos_ctx_destroy(c);                                               \
            return fos_cuda_fail(e_, "cudaMalloc " #ptr, __FILE__, __LINE__); \
        }                                                                     \
    } while (0)
    ALLOC(c->labA, V * 4);
    ALLOC(c->labB, V * 4);
    ALLOC(c->recA, V * sizeof(float4));
    ALLOC(c->recB, V * sizeof(float4));
    ALLOC(c->filt, V * 4);
    ALLOC(c->seedslot, V * 8);
    ALLOC(c->seeds, (size_t)max_n * sizeof(float4));
    ALLOC(c->fsc, (size_t)max_n * 4);
    ALLOC(c->used, (size_t)max_n * 4);
    ALLOC(c->ema, (size_t)max_n * 4);
    ALLOC(c->face_ids, NS * 4);
    ALLOC(c->face_counts, NS * 4);
    ALLOC(c->nl, NS * 4);
    ALLOC(c->face_score, NS * 4);
    ALLOC(c->prev, NS * 4);
    ALLOC(c->acc0, NS);
    ALLOC(c->acc1, NS);
    ALLOC(c->hkeys, c->H * 8);
    ALLOC(c->hmin, c->H * 4);
    ALLOC(c->hcnt, c->H * 4);
    ALLOC(c->claimed, c->H * 4);
    ALLOC(c->rowcnt, (size_t)max_n * 4);
    ALLOC(c->rowbuf, (size_t)max_n * FOS_ROWCAP * sizeof(uint4));
    ALLOC(c->revcnt, ((size_t)max_n + 1) * 4);
    ALLOC(c->revstart, ((size_t)max_n + 1) * 4);
    ALLOC(c->revfill, (size_t)max_n * 4);
    ALLOC(c->rev, NS * 4);
    c->scan_tmp_n = 4096;
    ALLOC(c->scan_tmp, c->scan_tmp_n * 4);
    ALLOC(c->pos_tmp, (size_t)max_n * 3 * 4);
    ALLOC(c->sorted, (size_t)max_n * sizeof(float4));
    ALLOC(c->ci_tmp, (size_t)max_n * 4);
    ALLOC(c->coop_bsum, 1024 * 4);
    ALLOC(c->rad_tmp, (size_t)max_n * 4);
    ALLOC(c->cellof, (size_t)max_n * 4);
    ALLOC(c->rank, (size_t)max_n * 4);
    ALLOC(c->coop_slot, (size_t)max_n * 4);
    ALLOC(c->pvol, (size_t)max_n * 8);
    ALLOC(c->pnbr, (size_t)max_n * 16 * 4);
    c->ptag_n = max_n < FOS_PTAG_MAX_N ? max_n : FOS_PTAG_MAX_N;
    ALLOC(c->ptag, (size_t)(FOS_PTAG_SWEEPS + 1) * c->ptag_n * 8);
    {
        cudaError_t e_ = cudaMemset(c->ptag, 0, (size_t)(FOS_PTAG_SWEEPS + 1) * c->ptag_n * 8);
        if (e_ != cudaSuccess) {
            fos_ctx_destroy(c);
            return fos_cuda_fail(e_, "cudaMemset ptag", __FILE__, __LINE__);
        }
    }
    ALLOC(c->stats_f, 64 * 4);
    ALLOC(c->stats_i, 64 * 4);
    ALLOC(c->ds, sizeof(FosDevState));
    ALLOC(c->fin_changed, FOS_FIN_MAXIT * sizeof(int));
    ALLOC(c->skip_part, FOS_SKIP_BLOCKS * 64 + 256);
#undef ALLOC
    if (cudaMallocHost(&c->pinned, 4096) != cudaSuccess) {
        fos_ctx_destroy(c);
        return fos_fail(FOS_E_CUDA, "cudaMallocHost staging buffer");
    }
    // Taichi fields start zeroed (fsc, fsc_ema, face_ids, prev scores ...).
    cudaMemset(c->fsc, 0, (size_t)max_n * 4);
    cudaMemset(c->used, 0, (size_t)max_n * 4);
    cudaMemset(c->ema, 0, (size_t)max_n * 4);
    cudaMemset(c->face_ids, 0, NS * 4);
    cudaMemset(c->face_counts, 0, NS * 4);
    cudaMemset(c->prev, 0, NS * 4);
    cudaMemset(c->nl, 0xFF, NS * 4);
    cudaMemset(c->hkeys, 0xFF, c->H * 8);
    cudaMemset(c->hmin, 0xFF, c->H * 4);
    cudaMemset(c->hcnt, 0, c->H * 4);
    cudaMemset(c->labA, 0xFF, V * 4);
    cudaMemset(c->labB, 0xFF, V * 4);
    cudaMemset(c->filt, 0xFF, V * 4);
    cudaMemset(c->ds, 0, sizeof(FosDevState));
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        fos_ctx_destroy(c);
        return fos_cuda_fail(e, "context init", __FILE__, __LINE__);
    }
    rc = alloc_cells(c);
    if (rc == FOS_OK) rc = fos_grid_init_attributes();
    if (rc) {
        fos_ctx_destroy(c);
        return rc;
    }
    rc = fos_set_resolution(c, max_res < 128 ? max_res : 128);
    if (rc) {
        fos_ctx_destroy(c);
        return rc;
    }
    *out = c;
    return FOS_OK;
}

extern "C" int fos_ctx_destroy(FosCtx* c) {
    if (!c) return FOS_OK;
    cudaSetDevice(c->device);
    for (int k = 0; k < FOS_GRAPH_SLOTS; ++k)
        if (c->gexec[k]) cudaGraphExecDestroy(c->gexec[k]);
    fos_sur_free(c);
    void* ptrs[] = {c->labA, c->labB, c->recA, c->recB, c->filt, c->seedslot, c->seeds, c->fsc, c->used, c->ema,
                    c->face_ids, c->face_counts, c->nl, c->face_score, c->prev, c->acc0, c->acc1,
                    c->hkeys, c->hmin, c->hcnt, c->claimed, c->rowcnt, c->rowbuf, c->revcnt,
                    c->revstart, c->revfill, c->rev, c->scan_tmp, c->pos_tmp, c->rad_tmp,
                    c->cellof, c->rank, c->cell_tmp, c->stats_f, c->stats_i, c->ds,
                    c->fin_changed, c->sorted, c->ci_tmp, c->coop_bsum, c->coop_cnt,
                    c->coop_part, c->coop_cnt2, c->coop_cfix, c->coop_idsort, c->coop_spfix,
                    c->coop_spst,
                    c->coop_slot, c->skip_part, c->pvol, c->pnbr, c->ptag};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (c->pinned) cudaFreeHost(c->pinned);
    delete c;
    return FOS_OK;
}

extern "C" int fos_set_resolution(FosCtx* c, int res) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(res >= 2 && res <= c->max_res, FOS_E_CAPACITY, "res outside [2, max_res]");
    c->res = res;
    c->vs = (float)(c->p.domain_size / (double)res);      // VOXEL_SIZE = L / JFA_RES
    c->passes = (int)ceil(log2((double)res)) + 1;         // ceil(log2 R) + 1
    if (c->passes > FOS_MAX_PASSES) c->passes = FOS_MAX_PASSES;
    for (int k = 0; k < FOS_GRAPH_SLOTS; ++k) c->gvalid[k] = false;
    return FOS_OK;
}

extern "C" int fos_get_resolution(FosCtx* c, int* res, int* num_passes, float* voxel_size) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    if (res) *res = c->res;
    if (num_passes) *num_passes = c->passes;
    if (voxel_size) *voxel_size = c->vs;
    return FOS_OK;
}

extern "C" int fos_jfa_fields(FosCtx* c, FosJfaFields* o) {
    FOS_REQUIRE(c != nullptr && o != nullptr, FOS_E_ARG, "NULL argument");
    o->fsc = c->fsc;
    o->fsc_ema = c->ema;
    o->face_ids = c->face_ids;
    o->face_counts = c->face_counts;
    o->neighbor_list = c->nl;
    o->neighbor_used_count = c->used;
    o->neighbor_prev_scores = c->prev;
    // final owner grid: buffer A or B by the passes actually run (device word)
    int fb = 0;
    FOS_CUDA(cudaDeviceSynchronize());
    FOS_CUDA(cudaMemcpy(&fb, &c->ds->final_buf, sizeof(int), cudaMemcpyDeviceToHost));
    o->labels = fb ? c->labB : c->labA;
    o->label_filtered = c->filt;
    return FOS_OK;
}

extern "C" long long fos_launch_count(FosCtx* c) { return c ? c->launches : -1; }

extern "C" int fos_device_error(FosCtx* c, int* word, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr && word != nullptr, FOS_E_ARG, "NULL argument");
    int* h = (int*)c->pinned;
    FOS_CUDA(cudaMemcpyAsync(h, &c->ds->error, sizeof(int), cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaStreamSynchronize(s));
    *word = *h;
    return FOS_OK;
}

__global__ void k_set_dev_int(int* p, int v) { *p = v; }

extern "C" int fos_device_error_clear(FosCtx* c, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    k_set_dev_int<<<1, 1, 0, s>>>(&c->ds->error, 0);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_test_barrier_plan(FosCtx* c, int leave_at_barrier, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(leave_at_barrier == 0 || leave_at_barrier >= 2, FOS_E_ARG,
                "leave_at_barrier must be 0 (off) or >= 2");
    k_set_dev_int<<<1, 1, 0, s>>>(&c->ds->bar_test, leave_at_barrier);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// ------------------------------------------------------------------- scan
// Block-wide exclusive scan of 4 consecutive items per thread (1024 threads,
// 4096 items per tile) using warp shuffles.
__device__ __forceinline__ int block_excl_scan(int v, int* s_warp, int* total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        int t = lane < nw ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) s_warp[lane] = t;
    }
    __syncthreads();
    int base = w > 0 ? s_warp[w - 1] : 0;
    *total = s_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return base + x - v;
}

// Single block; loops over tiles of 4096 with a running carry.
__global__ void k_scan_single(const int32_t* __restrict__ in, int32_t* __restrict__ out, int n,
                              int with_total) {
    __shared__ int s_warp[32];
    int carry = 0;
    for (int base = 0; base < n; base += 4096) {
        int i0 = base + threadIdx.x * 4;
        int v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = (i0 + k < n) ? in[i0 + k] : 0;
        int sum = v[0] + v[1] + v[2] + v[3];
        int tot;
        int ex = block_excl_scan(sum, s_warp, &tot);
        int run = carry + ex;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (i0 + k < n) out[i0 + k] = run;
            run += v[k];
        }
        carry += tot;
    }
    if (with_total && threadIdx.x == 0) out[n] = carry;
}

__global__ void k_scan_reduce(const int32_t* __restrict__ in, int32_t* __restrict__ bsum, int n) {
    __shared__ int s_warp[32];
    int i0 = blockIdx.x * 4096 + threadIdx.x * 4;
    int sum = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) sum += (i0 + k < n) ? in[i0 + k] : 0;
    int tot;
    block_excl_scan(sum, s_warp, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void k_scan_apply(const int32_t* __restrict__ in, int32_t* __restrict__ out,
                             const int32_t* __restrict__ bpre, int n, int with_total, int nb) {
    __shared__ int s_warp[32];
    int i0 = blockIdx.x * 4096 + threadIdx.x * 4;
    int v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = (i0 + k < n) ? in[i0 + k] : 0;
    int tot;
    int ex = block_excl_scan(v[0] + v[1] + v[2] + v[3], s_warp, &tot);
    int run = bpre[blockIdx.x] + ex;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (i0 + k < n) out[i0 + k] = run;
        run += v[k];
    }
    if (with_total && blockIdx.x == nb - 1 && threadIdx.x == 0) out[n] = bpre[nb - 1] + tot;
}

int fos_scan_exclusive(FosCtx* c, const int32_t* d_in, int32_t* d_out, int n, bool with_total,
                       cudaStream_t s) {
    if (n <= 0) {
        if (with_total) FOS_CUDA(cudaMemsetAsync(d_out, 0, 4, s));
        return FOS_OK;
    }
    if (n <= 4 * 4096) {
        k_scan_single<<<1, 1024, 0, s>>>(d_in, d_out, n, with_total ? 1 : 0);
        FOS_LAUNCHED(c);
        return FOS_OK;
    }
    int nb = (n + 4095) / 4096;
    FOS_REQUIRE((size_t)nb + 1 <= c->scan_tmp_n, FOS_E_CAPACITY, "scan too large");
    // block sums into scan_tmp[0..nb), exclusive scan of them in place, then apply.
    k_scan_reduce<<<nb, 1024, 0, s>>>(d_in, c->scan_tmp, n);
    FOS_LAUNCHED(c);
    k_scan_single<<<1, 1024, 0, s>>>(c->scan_tmp, c->scan_tmp, nb, 0);
    FOS_LAUNCHED(c);
    k_scan_apply<<<nb, 1024, 0, s>>>(d_in, d_out, c->scan_tmp, n, with_total ? 1 : 0, nb);
    FOS_LAUNCHED(c);
    return FOS_OK;
}
