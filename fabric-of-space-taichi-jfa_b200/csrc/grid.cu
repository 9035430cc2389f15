// grid.cu -- periodic spatial hash grid built by counting sort.
//
// Reference: grid.py:145-309 and rebuild_grid (run.py:476-504).  The
// reference scatters with an atomic fetch-add, so the order of particles
// inside a cell depends on scheduling; serial semantics (particles in index
// order) make each cell's slice of cell_indices ascending, and that is what
// these kernels produce: histogram with per-particle rank -> exclusive scan ->
// rank scatter -> per-cell sort of the (short) slices.
#include "phases.cuh"

// count_particles_per_cell (grid.py:186-222).  Optionally also writes the
// wrapped position to dst (scatter_particles' write-back, grid.py:287-288)
// and records each particle's cell and arrival rank for the rank scatter.
__global__ void k_grid_count(const float* src, float* dst, int n, int G, float L, float invL,
                             float halfL, int32_t* __restrict__ cell_count,
                             int32_t* __restrict__ cellof, int32_t* __restrict__ rank) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float wx = grid_wrap(src[3 * i + 0], L, invL);
    float wy = grid_wrap(src[3 * i + 1], L, invL);
    float wz = grid_wrap(src[3 * i + 2], L, invL);
    int c = cell_of_wrapped(wx, wy, wz, invL, halfL, G);
    int r = atomicAdd(&cell_count[c], 1);
    if (cellof) {
        cellof[i] = c;
        rank[i] = r;
    }
    if (dst) {
        dst[3 * i + 0] = wx;
        dst[3 * i + 1] = wy;
        dst[3 * i + 2] = wz;
    }
}

__global__ void k_grid_scatter_ranked(int n, const int32_t* __restrict__ cellof,
                                      const int32_t* __restrict__ rank,
                                      const int32_t* __restrict__ cell_start,
                                      int32_t* __restrict__ cell_indices) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cell_indices[cell_start[cellof[i]] + rank[i]] = i;
}

// scatter_particles (grid.py:268-309) for a caller-provided cell_write.
__global__ void k_grid_scatter_atomic(float* pos, int n, int G, float L, float invL, float halfL,
                                      int32_t* cell_write, int32_t* __restrict__ cell_indices) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float wx = grid_wrap(pos[3 * i + 0], L, invL);
    float wy = grid_wrap(pos[3 * i + 1], L, invL);
    float wz = grid_wrap(pos[3 * i + 2], L, invL);
    pos[3 * i + 0] = wx;
    pos[3 * i + 1] = wy;
    pos[3 * i + 2] = wz;
    int c = cell_of_wrapped(wx, wy, wz, invL, halfL, G);
    int p = atomicAdd(&cell_write[c], 1);
    cell_indices[p] = i;
}

// Sorts each cell's slice ascending.  Slice c is [begin[c], begin[c]+count[c])
// or, with end != NULL, [begin[c], end[c]).  With sp != NULL it also writes
// the cell-ordered copy sp[k] = (pos[idx[k]], rad[idx[k]]) that the
// neighbour-gather kernels read.
__global__ void k_grid_sort_cells(int ncells, const int32_t* __restrict__ begin,
                                  const int32_t* __restrict__ count, const int32_t* __restrict__ end,
                                  int32_t* __restrict__ idx, const float* __restrict__ pos,
                                  const float* __restrict__ rad, float4* __restrict__ sp) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int b = begin[c];
    int e = end ? end[c] : b + count[c];
    for (int k = b + 1; k < e; ++k) {
        int v = idx[k];
        int q = k - 1;
        while (q >= b && idx[q] > v) {
            idx[q + 1] = idx[q];
            --q;
        }
        idx[q + 1] = v;
    }
    if (sp) {
        for (int k = b; k < e; ++k) {
            int j = idx[k];
            sp[k] = make_float4(pos[3 * j + 0], pos[3 * j + 1], pos[3 * j + 2], rad[j]);
        }
    }
}

// sp[k] = (pos[idx[k]], rad[idx[k]]) for a grid built elsewhere.
__global__ void k_grid_gather_sorted(int n, const int32_t* __restrict__ idx,
                                     const float* __restrict__ pos, const float* __restrict__ rad,
                                     float4* __restrict__ sp) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int j = idx[k];
    sp[k] = make_float4(pos[3 * j + 0], pos[3 * j + 1], pos[3 * j + 2], rad[j]);
}

int fos_grid_gather_sorted(FosCtx* c, const int32_t* idx, const float* pos, const float* rad,
                           int n, cudaStream_t s) {
    if (n == 0) return FOS_OK;
    k_grid_gather_sorted<<<fos_blocks(n, 256), 256, 0, s>>>(n, idx, pos, rad, c->sorted);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

int fos_grid_init_attributes() { return FOS_OK; }

static int check_grid(FosCtx* c, int n) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(n >= 0 && n <= c->max_n, FOS_E_CAPACITY, "n outside [0, max_n]");
    return FOS_OK;
}

extern "C" int fos_grid_clear(FosCtx* c, int32_t* cell_count, fos_stream_t s) {
    FOS_REQUIRE(c != nullptr && cell_count != nullptr, FOS_E_ARG, "NULL argument");
    size_t G3 = (size_t)c->G * c->G * c->G;
    FOS_CUDA(cudaMemsetAsync(cell_count, 0, G3 * 4, s));
    return FOS_OK;
}

extern "C" int fos_grid_count(FosCtx* c, const float* pos, int32_t* cell_count, int n,
                              fos_stream_t s) {
    int rc = check_grid(c, n);
    if (rc) return rc;
    FOS_REQUIRE(cell_count && (n == 0 || pos), FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    k_grid_count<<<fos_blocks(n, 256), 256, 0, s>>>(pos, nullptr, n, c->G, c->L, c->invL, c->halfL,
                                                    cell_count, nullptr, nullptr);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_grid_prefix_sum(FosCtx* c, const int32_t* cell_count, int32_t* cell_start,
                                   fos_stream_t s) {
    FOS_REQUIRE(c && cell_count && cell_start, FOS_E_ARG, "NULL argument");
    return fos_scan_exclusive(c, cell_count, cell_start, c->G * c->G * c->G, false, s);
}

extern "C" int fos_grid_copy_pointers(FosCtx* c, const int32_t* cell_start, int32_t* cell_write,
                                      fos_stream_t s) {
    FOS_REQUIRE(c && cell_start && cell_write, FOS_E_ARG, "NULL argument");
    size_t G3 = (size_t)c->G * c->G * c->G;
    FOS_CUDA(cudaMemcpyAsync(cell_write, cell_start, G3 * 4, cudaMemcpyDeviceToDevice, s));
    return FOS_OK;
}

extern "C" int fos_grid_scatter(FosCtx* c, float* pos, int32_t* cell_write, int32_t* cell_indices,
                                int n, fos_stream_t s) {
    int rc = check_grid(c, n);
    if (rc) return rc;
    FOS_REQUIRE(cell_write && cell_indices && (n == 0 || pos), FOS_E_ARG, "NULL argument");
    if (n == 0) return FOS_OK;
    int G3 = c->G * c->G * c->G;
    FOS_REQUIRE((size_t)G3 <= c->cell_tmp_n, FOS_E_CAPACITY, "cell scratch too small");
    FOS_CUDA(cudaMemcpyAsync(c->cell_tmp, cell_write, (size_t)G3 * 4, cudaMemcpyDeviceToDevice, s));
    k_grid_scatter_atomic<<<fos_blocks(n, 256), 256, 0, s>>>(pos, n, c->G, c->L, c->invL, c->halfL,
                                                             cell_write, cell_indices);
    FOS_LAUNCHED(c);
    k_grid_sort_cells<<<fos_blocks(G3, 256), 256, 0, s>>>(G3, c->cell_tmp, nullptr, cell_write,
                                                          cell_indices, nullptr, nullptr, nullptr);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

// Fused rebuild reading positions from src and writing the wrapped positions
// to dst (src may equal dst).  With rad != NULL the cell-ordered (pos, rad)
// copy ctx->sorted is refreshed as well.
int fos_grid_build_from(FosCtx* c, const float* src, float* dst, int n, int32_t* cell_count,
                        int32_t* cell_start, int32_t* cell_indices, const float* rad,
                        cudaStream_t s) {
    int G3 = c->G * c->G * c->G;
    FOS_CUDA(cudaMemsetAsync(cell_count, 0, (size_t)G3 * 4, s));
    if (n > 0) {
        k_grid_count<<<fos_blocks(n, 256), 256, 0, s>>>(src, dst, n, c->G, c->L, c->invL, c->halfL,
                                                        cell_count, c->cellof, c->rank);
        FOS_LAUNCHED(c);
    }
    int rc = fos_scan_exclusive(c, cell_count, cell_start, G3, false, s);
    if (rc) return rc;
    if (n == 0) return FOS_OK;
    k_grid_scatter_ranked<<<fos_blocks(n, 256), 256, 0, s>>>(n, c->cellof, c->rank, cell_start,
                                                             cell_indices);
    FOS_LAUNCHED(c);
    k_grid_sort_cells<<<fos_blocks(G3, 256), 256, 0, s>>>(G3, cell_start, cell_count, nullptr,
                                                          cell_indices, dst, rad,
                                                          rad ? c->sorted : nullptr);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_grid_build(FosCtx* c, float* pos, int n, int32_t* cell_count,
                              int32_t* cell_start, int32_t* cell_indices, fos_stream_t s) {
    int rc = check_grid(c, n);
    if (rc) return rc;
    FOS_REQUIRE(cell_count && cell_start && cell_indices && (n == 0 || pos), FOS_E_ARG,
                "NULL argument");
    return fos_grid_build_from(c, pos, pos, n, cell_count, cell_start, cell_indices, nullptr, s);
}
