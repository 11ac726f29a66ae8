// Error reporting and small device utilities shared by the distger sources.
#include "dg_internal.h"

#include <atomic>
#include <cstdarg>
#include <cstring>

namespace dg {

static thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(DG_ERR_NOMEM, "%s: %s", what, cudaGetErrorString(e));
    }
    return fail(DG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

void clear_error() { g_last_error.clear(); }

static std::atomic<uint64_t> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int sm_count(int device) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
    return n > 0 ? n : 1;
}

// ---------------------------------------------------------------- scan ----
// Three-phase exclusive scan: per-tile sums, one-block scan of the tile sums,
// per-tile scan plus tile offset.  Tiles are SCAN_TILE elements, one block each.
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t *total) {
    __shared__ uint64_t warp_sums[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint64_t s = lane < SCAN_THREADS / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < SCAN_THREADS / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    uint64_t before = wid ? warp_sums[wid - 1] : 0;
    *total = warp_sums[SCAN_THREADS / 32 - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void scan_tile_sums(const uint32_t *in, uint64_t n, uint64_t *tile_sums) {
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    uint64_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
        if (base + i < n) s += in[base + i];
    uint64_t total;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void scan_tile_offsets(uint64_t *tile_sums, uint64_t n_tiles) {
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < n_tiles; base += SCAN_THREADS) {
        uint64_t i = base + threadIdx.x;
        uint64_t v = i < n_tiles ? tile_sums[i] : 0;
        uint64_t total;
        uint64_t ex = block_exclusive_scan(v, &total);
        if (i < n_tiles) tile_sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

__global__ void scan_tiles(const uint32_t *in, uint64_t n, const uint64_t *tile_offsets, uint64_t *out) {
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint64_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = base + i < n ? in[base + i] : 0;
        s += v[i];
    }
    uint64_t total;
    uint64_t ex = block_exclusive_scan(s, &total) + tile_offsets[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (base + i < n) out[base + i] = ex;
        ex += v[i];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == SCAN_THREADS - 1) out[n] = ex;
}

int exclusive_scan_u32_to_u64(const uint32_t *in, uint64_t *out, uint64_t n, cudaStream_t s) {
    if (n == 0) {
        DG_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), s));
        return DG_OK;
    }
    uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    DevArray<uint64_t> sums;
    DG_CUDA(sums.alloc(tiles));
    scan_tile_sums<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, sums.p); dg::note_launch();
    scan_tile_offsets<<<1, SCAN_THREADS, 0, s>>>(sums.p, tiles); dg::note_launch();
    scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, sums.p, out); dg::note_launch();
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaStreamSynchronize(s));
    return DG_OK;
}

}  // namespace dg

extern "C" const char *dg_last_error(void) { return dg::g_last_error.c_str(); }

extern "C" const char *dg_version(void) { return "distger 0.1 sm_100a"; }

extern "C" uint64_t dg_launch_count(void) { return dg::g_launches.load(std::memory_order_relaxed); }
