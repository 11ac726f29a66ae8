// Internal declarations shared by the distger CUDA sources (not part of the C ABI).
#pragma once

#include "distger.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace dg {

// Records `msg` as the calling thread's last error and returns `code`.
int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
void clear_error();

#define DG_CUDA(call)                                              \
    do {                                                           \
        cudaError_t dg_e_ = (call);                                \
        if (dg_e_ != cudaSuccess) return dg::cuda_fail(dg_e_, #call); \
    } while (0)

#define DG_CHECK(cond, code, ...)                    \
    do {                                             \
        if (!(cond)) return dg::fail(code, __VA_ARGS__); \
    } while (0)

// Typed device allocation that frees itself.
template <typename T>
struct DevArray {
    T *p = nullptr;
    size_t n = 0;
    DevArray() = default;
    DevArray(const DevArray &) = delete;
    DevArray &operator=(const DevArray &) = delete;
    ~DevArray() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        release();
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc(reinterpret_cast<void **>(&p), count * sizeof(T));
    }
    size_t bytes() const { return n * sizeof(T); }
    void swap(DevArray &o) {
        T *tp = p;
        p = o.p;
        o.p = tp;
        const size_t tn = n;
        n = o.n;
        o.n = tn;
    }
};

// Sets the current device for the lifetime of the guard and restores the old one.
struct DeviceGuard {
    int old = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&old);
        if (dev != old) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (old >= 0 && cur != old) cudaSetDevice(old);
    }
};

// Event pair for timing work queued on one stream.
struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    EventTimer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~EventTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    void start(cudaStream_t s) { cudaEventRecord(a, s); }
    void stop(cudaStream_t s) { cudaEventRecord(b, s); }
    double ms() {
        float t = 0.f;
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&t, a, b);
        return (double)t;
    }
};

int sm_count(int device);

// Counts kernel launches issued by this library (reported by dg_launch_count).
void note_launch();
void note_launches(uint64_t n);  // kernels run by a replayed CUDA graph

// Exclusive prefix sum of n 32-bit counts into 64-bit offsets (out has n + 1
// entries; out[n] = total).  Scratch is allocated internally.
int exclusive_scan_u32_to_u64(const uint32_t *in, uint64_t *out, uint64_t n, cudaStream_t s);

}  // namespace dg

// Device-resident graph: int64 row offsets and 8-byte CSR entries
// {neighbour, acceptance threshold}.
struct dg_graph {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t v_num = 0;
    uint64_t m = 0;
    dg::DevArray<uint64_t> offsets;   // v_num + 1
    dg::DevArray<uint2> entries;      // m
    dg::DevArray<uint32_t> out_deg;   // v_num
    dg::DevArray<uint32_t> in_deg;    // v_num
    dg::DevArray<uint32_t> freq;      // cumulative visits, v_num
    dg::DevArray<double> etable;      // entropy-term table
    uint32_t etable_max_sn = 0;
    std::vector<uint32_t> h_out_deg;
    std::vector<double> entropy_history;
    uint64_t visits_total = 0;        // footprints over all rounds (sum of freq)
    double threshold_ms = 0.0;
    int walk_shape = 0;               // walk_kernel launch shape (dg_walk_autotune)
    // Per-round buffers kept between rounds, so a round allocates nothing once
    // the first has run: counters, the visit counts' backup, entropy partial
    // sums, and the walk arena of the last freed dg_paths (largest kept).
    dg::DevArray<unsigned long long> round_stats;
    dg::DevArray<uint32_t> round_ctl, freq_backup;
    dg::DevArray<double> entropy_partial;
    dg::DevArray<uint32_t> spare_verts, spare_lens;
    dg::DevArray<uint64_t> copy_at;   // dg_paths_copy: walk offsets and compacted walks,
    dg::DevArray<uint32_t> copy_flat; // kept (and grown) between calls
    ~dg_graph();
};

// One round of walks in slot layout: walk w owns vertices[w * stride, w * stride + len[w]).
struct dg_paths {
    dg_graph *g = nullptr;
    int device = 0;
    uint32_t round = 0;
    uint32_t n_walks = 0;
    uint32_t stride = 0;
    dg::DevArray<uint32_t> verts;  // n_walks * stride
    dg::DevArray<uint32_t> lens;   // n_walks
    dg_round_info info{};
};

namespace dg {
int ensure_entropy_table(dg_graph *g, uint32_t max_sn);
}

// Device-resident undirected edge list: unique keys (lo << 32 | hi), lo < hi, ascending.
struct dg_edges {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t v_num = 0;
    uint64_t n = 0;
    dg::DevArray<uint64_t> keys;
    uint64_t data_seed = 0;
    int weighted = 1;
    ~dg_edges();
};

// Link-prediction test pairs on the device: positives first, then negatives.
struct dg_lp_pairs {
    int device = 0;
    uint64_t n_pos = 0, n_neg = 0;
    dg::DevArray<uint32_t> u, v;
    dg::DevArray<uint8_t> label;
    ~dg_lp_pairs();
};

namespace dg {
// splitmix64 finaliser.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}
// Data of a generated undirected edge: uniform (0, 1] keyed by the pair, or 1.0.
__host__ __device__ __forceinline__ float edge_data(uint64_t key, uint64_t seed, int weighted) {
    if (!weighted) return 1.0f;
    return 1.0f - (float)(mix64(key ^ seed) >> 40) * (1.0f / 16777216.0f);
}
}  // namespace dg
