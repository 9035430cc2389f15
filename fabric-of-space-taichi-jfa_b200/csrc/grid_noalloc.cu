// grid_noalloc.cu -- a hash-grid rebuild that allocates no device memory.
//
// fos_grid_build needs a context, and creating a context allocates.  Some
// callers cannot allocate at the point where they need the grid:
//   - a host that has handed all device memory to its own pool or caching
//     allocator, and forbids allocation outside it;
//   - a frame loop where cudaMalloc/cudaFree are unacceptable because they can
//     synchronise the device and stall every other stream;
//   - plain C hosts that hold only raw buffers and want no context object.
// fos_grid_build_noalloc serves them.  The caller passes the positions and
// the three output arrays.  The only other memory it needs is the
// per-particle scratch (each particle's cell and arrival rank), and that lives
// in a fixed array compiled into the library, so there is a hard limit of
// FOS_NOALLOC_MAX_PARTICLES particles.
//
// The scratch array is a single static device array per GPU: it exists from
// when the library is loaded until the process exits.  Every call writes each
// scratch entry it uses before reading it, so nothing in it has to start at
// zero and the previous call's contents are harmless.  Calls that overlap on
// the GPU, for example on two streams, share the array and race.  Serialise
// them.
#include <mutex>

#include "fos_internal.cuh"

// Kernels shared with the context-based rebuild (grid.cu, fos_ctx.cu).
__global__ void k_grid_count(const float* src, float* dst, int n, int G, float L, float invL,
                             float halfL, int32_t* __restrict__ cell_count,
                             int32_t* __restrict__ cellof, int32_t* __restrict__ rank);
__global__ void k_grid_scatter_ranked(int n, const int32_t* __restrict__ cellof,
                                      const int32_t* __restrict__ rank,
                                      const int32_t* __restrict__ cell_start,
                                      int32_t* __restrict__ cell_indices);
__global__ void k_grid_sort_cells(int ncells, const int32_t* __restrict__ begin,
                                  const int32_t* __restrict__ count, const int32_t* __restrict__ end,
                                  int32_t* __restrict__ idx, const float* __restrict__ pos,
                                  const float* __restrict__ rad, float4* __restrict__ sp);
__global__ void k_scan_single(const int32_t* __restrict__ in, int32_t* __restrict__ out, int n,
                              int with_total);

// Scratch: [0, MAX) cell of each particle, [MAX, 2*MAX) its arrival rank.
// 2 * 65,536 * 4 bytes = 512 KiB on every GPU that loads the library.
static __device__ __align__(256) int32_t g_noalloc_scratch[2 * FOS_NOALLOC_MAX_PARTICLES];

#define FOS_NOALLOC_MAX_DEVICES 64

// Device address of g_noalloc_scratch on the current device.  In host code the
// symbol's name is only a host-side handle, never a device address, so it must
// go through cudaGetSymbolAddress with the right device current.  Outside
// stream capture the address is looked up on every call (no allocation, no
// synchronisation), so a device reset or a reloaded module never leaves a stale
// pointer behind.  During capture the lookup is not made: the address cached
// by an earlier call on this device is used, and with none cached the call
// fails with FOS_E_ARG before anything is launched.
static int32_t* scratch_for_current_device(fos_stream_t s, int* rc_out) {
    static std::mutex mu;
    static int32_t* addr[FOS_NOALLOC_MAX_DEVICES] = {nullptr};
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *rc_out = fos_cuda_fail(e, "cudaGetDevice", __FILE__, __LINE__);
        return nullptr;
    }
    if (dev < 0 || dev >= FOS_NOALLOC_MAX_DEVICES) {
        *rc_out = fos_fail(FOS_E_ARG, "device index above the supported range");
        return nullptr;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) {
        *rc_out = fos_cuda_fail(e, "cudaStreamIsCapturing", __FILE__, __LINE__);
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            *rc_out = fos_cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__,
                                    __LINE__);
            return nullptr;
        }
        addr[dev] = (int32_t*)p;
    } else if (!addr[dev]) {
        *rc_out = fos_fail(FOS_E_ARG,
                           "fos_grid_build_noalloc: the first call on a device must come before "
                           "any stream capture (it looks up the scratch array's address)");
        return nullptr;
    }
    *rc_out = FOS_OK;
    return addr[dev];
}

extern "C" int fos_grid_build_noalloc(float* pos, int n, int grid_res, double domain_size,
                                      int32_t* cell_count, int32_t* cell_start,
                                      int32_t* cell_indices, fos_stream_t s) {
    FOS_REQUIRE(n >= 0, FOS_E_ARG, "n must be >= 0");
    FOS_REQUIRE(n <= FOS_NOALLOC_MAX_PARTICLES, FOS_E_CAPACITY,
                "n exceeds FOS_NOALLOC_MAX_PARTICLES (65536): use a context and fos_grid_build");
    FOS_REQUIRE(grid_res >= 3 && grid_res <= FOS_NOALLOC_MAX_GRID_RES, FOS_E_ARG,
                "grid_res must be in [3, 256]");
    FOS_REQUIRE(domain_size > 0.0, FOS_E_ARG, "domain_size must be > 0");
    FOS_REQUIRE(cell_count && cell_start && cell_indices && (n == 0 || pos), FOS_E_ARG,
                "NULL argument");
    int rc = FOS_OK;
    int32_t* scratch = scratch_for_current_device(s, &rc);
    if (!scratch) return rc;
    int32_t* cellof = scratch;
    int32_t* rank = scratch + FOS_NOALLOC_MAX_PARTICLES;
    // the same folded constants as a context (Python floats -> f32 once)
    const float L = (float)domain_size;
    const float invL = (float)(1.0 / domain_size);
    const float halfL = (float)(0.5 * domain_size);
    const int G = grid_res;
    const int G3 = G * G * G;
    // cell_count is the histogram, so it (an output, not scratch) starts at zero
    FOS_CUDA(cudaMemsetAsync(cell_count, 0, (size_t)G3 * sizeof(int32_t), s));
    if (n > 0) {
        k_grid_count<<<fos_blocks(n, 256), 256, 0, s>>>(pos, pos, n, G, L, invL, halfL, cell_count,
                                                        cellof, rank);
        FOS_CUDA(cudaPeekAtLastError());
    }
    // single-block scan: it needs no block-sum scratch, and its time grows with
    // grid_res^3 (about a millisecond at 128, tens of milliseconds at 256)
    k_scan_single<<<1, 1024, 0, s>>>(cell_count, cell_start, G3, 0);
    FOS_CUDA(cudaPeekAtLastError());
    if (n == 0) return FOS_OK;
    k_grid_scatter_ranked<<<fos_blocks(n, 256), 256, 0, s>>>(n, cellof, rank, cell_start,
                                                             cell_indices);
    FOS_CUDA(cudaPeekAtLastError());
    k_grid_sort_cells<<<fos_blocks(G3, 256), 256, 0, s>>>(G3, cell_start, cell_count, nullptr,
                                                          cell_indices, nullptr, nullptr, nullptr);
    FOS_CUDA(cudaPeekAtLastError());
    return FOS_OK;
}
