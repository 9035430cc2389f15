// jfa_dirty.cu -- dirty-tile bookkeeping of the JFA grid (jfa.py:966-1049).
//
// The reference marks 16^3-voxel tiles whose particles moved or resized since
// the last JFA and counts them for its telemetry (run.py:1021-1047); the JFA
// itself is unchanged by it.  Here one thread per particle marks its tile and
// halo (byte stores of 1: idempotent, so the order of the stores does not
// matter) and one reduction counts the marked tiles.
#include "jfa_body.cuh"

#define FOS_TILE 16  // JFA_TILE_SIZE (config.py:182)

// world_to_tile (jfa.py:316-335) on one axis.
__device__ __forceinline__ int tile_of(float p, float halfL, float L, int R) {
    return world_to_voxel(p, halfL, L, R) / FOS_TILE;
}

// mark_dirty_tiles (jfa.py:966-1008) for particle i.
__global__ void k_dirty_mark(const float* __restrict__ pos, const float* __restrict__ rad,
                             const float* __restrict__ pos_prev, const float* __restrict__ rad_prev,
                             int n, int R, float halfL, float L, float pos_thr, float rad_thr,
                             int halo, int tiles, uint8_t* __restrict__ dirty) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float p[3], q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p[k] = __ldg(&pos[3 * i + k]);
        q[k] = __ldg(&pos_prev[3 * i + k]);
    }
    const float dx = fsub(p[0], q[0]), dy = fsub(p[1], q[1]), dz = fsub(p[2], q[2]);
    const float dpos = __fsqrt_rn(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
    const float drad = fabsf(fsub(__ldg(&rad[i]), __ldg(&rad_prev[i])));
    int tc[3];
    bool moved = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        tc[k] = tile_of(p[k], halfL, L, R);
        moved |= tc[k] != tile_of(q[k], halfL, L, R);
    }
    if (!(dpos > pos_thr || drad > rad_thr || moved)) return;
    for (int oz = -halo; oz <= halo; ++oz)
        for (int oy = -halo; oy <= halo; ++oy)
            for (int ox = -halo; ox <= halo; ++ox) {
                const int tx = wrap_mod(tc[0] + ox, tiles), ty = wrap_mod(tc[1] + oy, tiles),
                          tz = wrap_mod(tc[2] + oz, tiles);
                dirty[((size_t)tx * tiles + ty) * tiles + tz] = 1;
            }
}

// count_dirty_tiles (jfa.py:1011-1024): one atomic per warp.
__global__ void k_dirty_count(const uint8_t* __restrict__ dirty, int total, int* count) {
    int c = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x)
        c += dirty[t] == 1 ? 1 : 0;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

extern "C" int fos_dirty_mark(FosCtx* c, const float* pos, const float* rad, const float* pos_prev,
                              const float* rad_prev, int n, double pos_threshold,
                              double rad_threshold, int halo, uint8_t* tile_dirty,
                              fos_stream_t s) {
    FOS_REQUIRE(c != nullptr, FOS_E_ARG, "ctx is NULL");
    FOS_REQUIRE(n >= 0 && n <= c->max_n, FOS_E_CAPACITY, "n outside [0, max_n]");
    FOS_REQUIRE(halo >= 0 && halo <= 4, FOS_E_ARG, "halo must be in [0, 4]");
    FOS_REQUIRE(n == 0 || (pos && rad && pos_prev && rad_prev && tile_dirty), FOS_E_ARG,
                "NULL argument");
    if (n == 0) return FOS_OK;
    const int tiles = (c->res + FOS_TILE - 1) / FOS_TILE;
    // thresholds are fractions of VOXEL_SIZE = L / JFA_RES, folded in double
    const double vs = c->p.domain_size / (double)c->res;
    k_dirty_mark<<<fos_blocks(n, 256), 256, 0, s>>>(
        pos, rad, pos_prev, rad_prev, n, c->res, c->halfL, c->L, (float)(pos_threshold * vs),
        (float)(rad_threshold * vs), halo, tiles, tile_dirty);
    FOS_LAUNCHED(c);
    return FOS_OK;
}

extern "C" int fos_dirty_count(FosCtx* c, const uint8_t* tile_dirty, int* count_host,
                               fos_stream_t s) {
    FOS_REQUIRE(c && tile_dirty && count_host, FOS_E_ARG, "NULL argument");
    const int tiles = (c->res + FOS_TILE - 1) / FOS_TILE;
    const int total = tiles * tiles * tiles;
    int* d = &c->ds->tile_count;
    FOS_CUDA(cudaMemsetAsync(d, 0, sizeof(int), s));
    int blocks = fos_blocks(total, 256);
    if (blocks > 64) blocks = 64;
    k_dirty_count<<<blocks, 256, 0, s>>>(tile_dirty, total, d);
    FOS_LAUNCHED(c);
    int* h = (int*)c->pinned;
    FOS_CUDA(cudaMemcpyAsync(h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
    FOS_CUDA(cudaStreamSynchronize(s));
    *count_host = *h;
    return FOS_OK;
}
