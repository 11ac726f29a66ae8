// Synthetic graphs, the link-prediction split and AUC scoring on the device.
//
// The reference reads graphs from disk and its gtrain tool splits them on the
// host (src/tools/gtrain.cpp:226-386); at the Twitter-shaped scale (41.6M
// vertices, 1.47B edges) neither a host generator nor a host split is
// practical, so the whole loop runs here:
//
//  * dg_edges_chung_lu: edge-sampling Chung-Lu graph.  Expected degrees
//    w_i = (i + 1)^(-1/(beta - 1)) scaled to sum 2m and capped at max_degree
//    (computed on the host in double, sequentially); each of m draws picks both
//    endpoints with probability proportional to w (a 53-bit Philox uniform
//    looked up in the CDF through a guide table); self-loops are dropped,
//    duplicate undirected pairs merged (sort + unique), and every vertex left
//    without an edge gets one edge to a w-weighted vertex.  Vertex ids are
//    permuted by a keyed Feistel bijection so that id order carries no degree
//    information.  Edge data: uniform (0, 1] keyed by the pair, or 1.0.
//  * dg_edges_split: gtrain's hold-out rule in a parallel form.  An edge is a
//    candidate when its keyed hash falls below frac; a candidate is held out
//    unless one of its endpoints would lose its last edge (deg - candidates < 1
//    at that endpoint, which keeps every vertex connected as gtrain's
//    degree > 1 test does); as many negatives are drawn as uniform vertex pairs
//    that are not edges of the full graph (Philox, up to 64 tries each).
//  * dg_lp_auc: score = sigmoid of the input-embedding dot product (cosine
//    too), AUC as the Mann-Whitney statistic with ties averaged -- the same
//    definition as the host scorer.
//
// Every step is deterministic given the seeds.
#include "dg_internal.h"
#include "dg_philox.cuh"
#include "dg_sgns.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

namespace {

constexpr uint32_t kGenTag = 0x4347454Eu;    // "CGEN": draw j
constexpr uint32_t kIsoTag = 0x4349534Fu;    // "CISO": partner of isolated vertex v
constexpr uint32_t kNegTag = 0x4C504E47u;    // "LPNG": negative pair j, try t
constexpr uint64_t kNoEdge = ~0ull;

using dg::mix64;

// Keyed bijection of [0, n): a 4-round Feistel network on 2*half bits, cycle-walked into range.
struct Perm {
    uint32_t n, half, mask;
    uint64_t key;
    __host__ __device__ uint32_t operator()(uint32_t x) const {
        do {
            uint32_t l = x >> half, r = x & mask;
            for (uint32_t k = 0; k < 4; k++) {
                const uint32_t f = (uint32_t)mix64((uint64_t)r ^ (key + (uint64_t)k * 0x9E3779B97F4A7C15ull)) & mask;
                const uint32_t t = l ^ f;
                l = r;
                r = t;
            }
            x = (l << half) | r;
        } while (x >= n);
        return x;
    }
};

Perm make_perm(uint32_t n, uint64_t seed) {
    uint32_t bits = 2;
    while (bits < 32 && (1ull << bits) < n) bits++;
    if (bits & 1) bits++;
    Perm p;
    p.n = n;
    p.half = bits / 2;
    p.mask = (1u << p.half) - 1;
    p.key = mix64(seed ^ 0x5045524D5045524Dull);
    return p;
}

// 53-bit uniform in [0, 1) from two 32-bit words.
__host__ __device__ __forceinline__ double uniform53(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// First i with cdf[i] > u (clamped to n - 1), searched inside the guide table's bucket.
__device__ __forceinline__ uint32_t sample_cdf(const double *__restrict__ cdf, const uint32_t *__restrict__ guide,
                                               uint32_t n, double u) {
    uint32_t k = (uint32_t)(u * (double)n);
    if (k >= n) k = n - 1;   // u * n can round up to n for u just below 1
    uint32_t lo = guide[k], hi = guide[k + 1];
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] > u) hi = mid;
        else lo = mid + 1;
    }
    return lo < n ? lo : n - 1;
}

__global__ void draw_keys(const double *cdf, const uint32_t *guide, uint32_t n, uint64_t m, Perm perm, uint32_t k0,
                          uint32_t k1, uint64_t *keys) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint4 x = philox4x32_10(make_uint4((uint32_t)j, (uint32_t)(j >> 32), 0u, kGenTag), k0, k1);
        const uint32_t s = sample_cdf(cdf, guide, n, uniform53(x.x, x.y));
        const uint32_t d = sample_cdf(cdf, guide, n, uniform53(x.z, x.w));
        if (s == d) {
            keys[j] = kNoEdge;
            continue;
        }
        const uint32_t a = perm(s), b = perm(d);
        keys[j] = a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
    }
}

__global__ void count_degrees(const uint64_t *keys, uint64_t n_keys, uint32_t *deg) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_keys;
         i += (uint64_t)gridDim.x * blockDim.x) {
        atomicAdd(&deg[keys[i] >> 32], 1u);
        atomicAdd(&deg[(uint32_t)keys[i]], 1u);
    }
}

// One edge for every vertex without one (the reference asserts every vertex has
// an edge, walk.hpp:709-723); appended at slots taken from a counter, order
// fixed afterwards by the sort.
__global__ void isolated_edges(const uint32_t *deg, uint32_t n, const double *cdf, const uint32_t *guide, Perm perm,
                               uint32_t k0, uint32_t k1, uint64_t *out, unsigned long long *count) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (deg[v]) continue;
        const uint4 x = philox4x32_10(make_uint4(v, 0u, 1u, kIsoTag), k0, k1);
        uint32_t p = perm(sample_cdf(cdf, guide, n, uniform53(x.x, x.y)));
        if (p == v) p = (v + 1) % n;
        const uint64_t key = v < p ? ((uint64_t)v << 32) | p : ((uint64_t)p << 32) | v;
        out[atomicAdd(count, 1ull)] = key;
    }
}

template <typename F>
int cub_run(F f) {
    size_t bytes = 0;
    DG_CUDA(f(nullptr, bytes));
    dg::DevArray<uint8_t> tmp;
    DG_CUDA(tmp.alloc(bytes ? bytes : 1));
    DG_CUDA(f(tmp.p, bytes));
    return DG_OK;
}

// Sorts keys[0, n) and removes duplicates and kNoEdge; keys is replaced, *n updated.
int sort_unique(dg::DevArray<uint64_t> &keys, uint64_t &n, cudaStream_t s) {
    dg::DevArray<uint64_t> alt;
    DG_CUDA(alt.alloc(n ? n : 1));
    cub::DoubleBuffer<uint64_t> db(keys.p, alt.p);
    const uint64_t items = n;
    int rc = cub_run([&](void *t, size_t &b) {
        return cub::DeviceRadixSort::SortKeys(t, b, db, items, 0, 64, s);
    });
    if (rc) return rc;
    uint64_t *sorted = db.Current(), *other = db.Alternate();
    dg::DevArray<uint64_t> d_count;
    DG_CUDA(d_count.alloc(1));
    rc = cub_run([&](void *t, size_t &b) {
        return cub::DeviceSelect::Unique(t, b, sorted, other, d_count.p, (int64_t)items, s);
    });
    if (rc) return rc;
    uint64_t unique = 0;
    DG_CUDA(cudaMemcpyAsync(&unique, d_count.p, 8, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    // kNoEdge sorts last: drop it.
    uint64_t last = 0;
    if (unique) {
        DG_CUDA(cudaMemcpyAsync(&last, other + unique - 1, 8, cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        if (last == kNoEdge) unique--;
    }
    // Keep the array that holds the result.
    if (other == alt.p) keys.swap(alt);
    n = unique;
    return DG_OK;
}

// Expected degrees and their normalised CDF (double, sequential sums), plus a
// guide table: guide[k] = first i with cdf[i] > k / n, k = 0..n.
void host_cdf(uint32_t n, uint64_t m, double beta, double cap, std::vector<double> &cdf, std::vector<uint32_t> &guide) {
    std::vector<double> w(n);
    const double gamma = 1.0 / (beta - 1.0);
    double total = 0.0;
    for (uint32_t i = 0; i < n; i++) {
        w[i] = std::pow((double)i + 1.0, -gamma);
        total += w[i];
    }
    const double target = 2.0 * (double)m;
    for (uint32_t i = 0; i < n; i++) w[i] *= target / total;
    if (cap > 0) {
        for (int it = 0; it < 8; it++) {
            total = 0.0;
            for (uint32_t i = 0; i < n; i++) {
                w[i] = std::min(w[i], cap);
                total += w[i];
            }
            for (uint32_t i = 0; i < n; i++) w[i] *= target / total;
        }
        for (uint32_t i = 0; i < n; i++) w[i] = std::min(w[i], cap);
    }
    cdf.resize(n);
    double acc = 0.0;
    for (uint32_t i = 0; i < n; i++) {
        acc += w[i];
        cdf[i] = acc;
    }
    for (uint32_t i = 0; i < n; i++) cdf[i] /= acc;
    guide.resize((size_t)n + 1);
    uint32_t i = 0;
    for (uint64_t k = 0; k <= n; k++) {
        const double u = (double)k / (double)n;
        while (i < n && !(cdf[i] > u)) i++;
        guide[k] = i;
    }
}

// ------------------------------------------------------------------ split

__device__ __forceinline__ bool is_candidate(uint64_t key, uint64_t seed, double frac) {
    return (double)(mix64(key ^ seed) >> 11) * (1.0 / 9007199254740992.0) < frac;
}

__global__ void split_count(const uint64_t *keys, uint64_t n, uint64_t seed, double frac, uint32_t *cand) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (!is_candidate(keys[i], seed, frac)) continue;
        atomicAdd(&cand[keys[i] >> 32], 1u);
        atomicAdd(&cand[(uint32_t)keys[i]], 1u);
    }
}

__global__ void split_flag(const uint64_t *keys, uint64_t n, uint64_t seed, double frac, const uint32_t *deg,
                           const uint32_t *cand, uint8_t *held) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = (uint32_t)(keys[i] >> 32), b = (uint32_t)keys[i];
        held[i] = is_candidate(keys[i], seed, frac) && deg[a] - cand[a] >= 1 && deg[b] - cand[b] >= 1;
    }
}

__device__ __forceinline__ bool has_key(const uint64_t *keys, uint64_t n, uint64_t key) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (keys[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && keys[lo] == key;
}

__global__ void split_negatives(const uint64_t *keys, uint64_t n_keys, uint32_t v_num, uint64_t n_neg, uint32_t k0,
                                uint32_t k1, uint32_t *u, uint32_t *v, unsigned int *fail) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_neg;
         j += (uint64_t)gridDim.x * blockDim.x) {
        bool done = false;
        for (uint32_t t = 0; t < 64 && !done; t++) {
            const uint4 x = philox4x32_10(make_uint4((uint32_t)j, (uint32_t)(j >> 32), t, kNegTag), k0, k1);
            const uint32_t a = (uint32_t)(((uint64_t)x.x * v_num) >> 32), b = (uint32_t)(((uint64_t)x.y * v_num) >> 32);
            if (a == b) continue;
            const uint64_t key = a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
            if (has_key(keys, n_keys, key)) continue;
            u[j] = a;
            v[j] = b;
            done = true;
        }
        if (!done) atomicOr(fail, 1u);
    }
}

__global__ void reverse_copy(const uint64_t *in, uint64_t n, uint64_t *out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = in[n - 1 - i];
}

__global__ void split_positives(const uint64_t *held_keys, uint64_t n, uint32_t *u, uint32_t *v) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        u[i] = (uint32_t)(held_keys[i] >> 32);
        v[i] = (uint32_t)held_keys[i];
    }
}

// -------------------------------------------------------------------- AUC

// Orderable 64-bit key of a double (ascending keys = ascending values).
__device__ __forceinline__ uint64_t order_key(double x) {
    const uint64_t b = (uint64_t)__double_as_longlong(x);
    return (b >> 63) ? ~b : b | 0x8000000000000000ull;
}

template <int V>
__global__ void lp_scores(const uint32_t *u, const uint32_t *v, uint64_t n, const int32_t *v2w, const float *f32,
                          const __nv_bfloat16 *bf, const float *master, uint32_t n_master, uint64_t *sig_key,
                          uint64_t *cos_key) {
    constexpr int D = 32 * V;
    const int lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const int32_t a = v2w[u[i]], b = v2w[v[i]];
        double dot = 0.0, na = 0.0, nb = 0.0;
        for (int c = lane * V; c < lane * V + V; c++) {
            double x = 0.0, y = 0.0;
            if (a >= 0) x = f32 ? f32[(size_t)a * D + c] : (uint32_t)a < n_master ? master[(size_t)a * D + c]
                                                                                   : __bfloat162float(bf[(size_t)a * D + c]);
            if (b >= 0) y = f32 ? f32[(size_t)b * D + c] : (uint32_t)b < n_master ? master[(size_t)b * D + c]
                                                                                   : __bfloat162float(bf[(size_t)b * D + c]);
            dot = fma(x, y, dot);
            na = fma(x, x, na);
            nb = fma(y, y, nb);
        }
        for (int o = 16; o; o >>= 1) {
            dot += __shfl_xor_sync(0xffffffffu, dot, o);
            na += __shfl_xor_sync(0xffffffffu, na, o);
            nb += __shfl_xor_sync(0xffffffffu, nb, o);
        }
        if (lane == 0) {
            sig_key[i] = order_key(1.0 / (1.0 + exp(-dot)));
            cos_key[i] = order_key(dot / fmax(sqrt(na) * sqrt(nb), 1e-30));
        }
    }
}

// For sorted keys: per element its tie group's first index (flags of group starts
// are turned into starts by a max-scan done here per element by a backward search
// bounded by the group length -- groups are walked once by their first element).
__global__ void tie_groups(const uint64_t *keys, const uint8_t *label, uint64_t n, double *pos_rank_sum) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (i > 0 && keys[i] == keys[i - 1]) {
            pos_rank_sum[i] = 0.0;
            continue;
        }
        uint64_t e = i + 1;
        uint64_t pos = label[i];
        while (e < n && keys[e] == keys[i]) pos += label[e++];
        // ranks i+1 .. e, average (i + 1 + e) / 2
        pos_rank_sum[i] = (double)pos * ((double)(i + 1) + (double)e) * 0.5;
    }
}

int auc_of(const uint64_t *keys_in, const uint8_t *labels_in, uint64_t n, uint64_t n_pos, cudaStream_t s,
           int device, double *auc) {
    dg::DevArray<uint64_t> keys;
    dg::DevArray<uint8_t> labels;
    DG_CUDA(keys.alloc(n));
    DG_CUDA(labels.alloc(n));
    int rc = cub_run([&](void *t, size_t &b) {
        return cub::DeviceRadixSort::SortPairs(t, b, keys_in, keys.p, labels_in, labels.p, n, 0, 64, s);
    });
    if (rc) return rc;
    dg::DevArray<double> part, total;
    DG_CUDA(part.alloc(n));
    DG_CUDA(total.alloc(1));
    tie_groups<<<dg::sm_count(device) * 8, 256, 0, s>>>(keys.p, labels.p, n, part.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    rc = cub_run([&](void *t, size_t &b) { return cub::DeviceReduce::Sum(t, b, part.p, total.p, (int64_t)n, s); });
    if (rc) return rc;
    double sum = 0.0;
    DG_CUDA(cudaMemcpyAsync(&sum, total.p, 8, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    const double np = (double)n_pos, nn = (double)(n - n_pos);
    *auc = (n_pos == 0 || n_pos == n) ? NAN : (sum - np * (np + 1.0) / 2.0) / (np * nn);
    return DG_OK;
}

}  // namespace

dg_edges::~dg_edges() {
    if (stream) {
        dg::DeviceGuard guard(device);
        cudaStreamSynchronize(stream);
        keys.release();
        cudaStreamDestroy(stream);
    }
}

dg_lp_pairs::~dg_lp_pairs() {
    dg::DeviceGuard guard(device);
    u.release();
    v.release();
    label.release();
}

extern "C" int dg_edges_chung_lu(const dg_chung_lu_params *p, int device, dg_edges **out) {
    DG_CHECK(p && out, DG_ERR_ARG, "dg_edges_chung_lu: NULL argument");
    *out = nullptr;
    DG_CHECK(p->n >= 2 && p->m >= 1, DG_ERR_ARG, "need n >= 2 and m >= 1");
    DG_CHECK(p->beta > 1.0, DG_ERR_ARG, "beta must exceed 1");
    int n_dev = 0;
    DG_CUDA(cudaGetDeviceCount(&n_dev));
    DG_CHECK(device >= 0 && device < n_dev, DG_ERR_ARG, "device %d out of range (%d)", device, n_dev);
    std::vector<double> cdf;
    std::vector<uint32_t> guide;
    host_cdf(p->n, p->m, p->beta, p->max_degree, cdf, guide);
    dg::DeviceGuard guard(device);
    std::unique_ptr<dg_edges> e(new dg_edges());
    e->device = device;
    e->v_num = p->n;
    e->weighted = p->weighted;
    e->data_seed = mix64(p->seed ^ 0x4441544144415441ull);
    DG_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    cudaStream_t s = e->stream;
    dg::DevArray<double> d_cdf;
    dg::DevArray<uint32_t> d_guide, deg;
    DG_CUDA(d_cdf.alloc(p->n));
    DG_CUDA(d_guide.alloc((size_t)p->n + 1));
    DG_CUDA(cudaMemcpyAsync(d_cdf.p, cdf.data(), (size_t)p->n * 8, cudaMemcpyHostToDevice, s));
    DG_CUDA(cudaMemcpyAsync(d_guide.p, guide.data(), ((size_t)p->n + 1) * 4, cudaMemcpyHostToDevice, s));
    const Perm perm = make_perm(p->n, p->seed);
    const uint32_t k0 = (uint32_t)p->seed, k1 = (uint32_t)(p->seed >> 32);
    const unsigned grid = (unsigned)dg::sm_count(device) * 8;
    // Room for the draws plus one edge per possibly isolated vertex.
    DG_CUDA(e->keys.alloc(p->m + p->n));
    draw_keys<<<grid, 256, 0, s>>>(d_cdf.p, d_guide.p, p->n, p->m, perm, k0, k1, e->keys.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    uint64_t n = p->m;
    int rc = sort_unique(e->keys, n, s);
    if (rc) return rc;
    DG_CUDA(deg.alloc(p->n));
    DG_CUDA(cudaMemsetAsync(deg.p, 0, (size_t)p->n * 4, s));
    count_degrees<<<grid, 256, 0, s>>>(e->keys.p, n, deg.p);
    dg::note_launch();
    dg::DevArray<unsigned long long> cnt;
    DG_CUDA(cnt.alloc(1));
    DG_CUDA(cudaMemsetAsync(cnt.p, 0, 8, s));
    if (e->keys.n < n + p->n) {   // sort_unique may hand back a buffer sized for the draws only
        dg::DevArray<uint64_t> bigger;
        DG_CUDA(bigger.alloc(n + p->n));
        DG_CUDA(cudaMemcpyAsync(bigger.p, e->keys.p, n * 8, cudaMemcpyDeviceToDevice, s));
        bigger.swap(e->keys);
    }
    isolated_edges<<<grid, 256, 0, s>>>(deg.p, p->n, d_cdf.p, d_guide.p, perm, k0, k1, e->keys.p + n, cnt.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    unsigned long long n_iso = 0;
    DG_CUDA(cudaMemcpyAsync(&n_iso, cnt.p, 8, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    if (n_iso) {
        n += n_iso;
        rc = sort_unique(e->keys, n, s);
        if (rc) return rc;
    }
    e->n = n;
    *out = e.release();
    return DG_OK;
}

extern "C" int dg_edges_get_info(const dg_edges *e, uint32_t *v_num, uint64_t *n_edges) {
    DG_CHECK(e, DG_ERR_ARG, "dg_edges_get_info: NULL edges");
    if (v_num) *v_num = e->v_num;
    if (n_edges) *n_edges = e->n;
    return DG_OK;
}

namespace {
__global__ void edges_unpack(const uint64_t *keys, uint64_t n, uint64_t data_seed, int weighted, uint32_t *src,
                             uint32_t *dst, float *data) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (src) src[i] = (uint32_t)(keys[i] >> 32);
        if (dst) dst[i] = (uint32_t)keys[i];
        if (data) data[i] = dg::edge_data(keys[i], data_seed, weighted);
    }
}
}  // namespace

extern "C" int dg_edges_copy(const dg_edges *e, uint32_t *src, uint32_t *dst, float *data) {
    DG_CHECK(e, DG_ERR_ARG, "dg_edges_copy: NULL edges");
    dg::DeviceGuard guard(e->device);
    if (e->n == 0) return DG_OK;
    dg::DevArray<uint32_t> a, b;
    dg::DevArray<float> c;
    if (src) DG_CUDA(a.alloc(e->n));
    if (dst) DG_CUDA(b.alloc(e->n));
    if (data) DG_CUDA(c.alloc(e->n));
    edges_unpack<<<dg::sm_count(e->device) * 8, 256, 0, e->stream>>>(e->keys.p, e->n, e->data_seed, e->weighted, a.p,
                                                                     b.p, c.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    if (src) DG_CUDA(cudaMemcpyAsync(src, a.p, e->n * 4, cudaMemcpyDeviceToHost, e->stream));
    if (dst) DG_CUDA(cudaMemcpyAsync(dst, b.p, e->n * 4, cudaMemcpyDeviceToHost, e->stream));
    if (data) DG_CUDA(cudaMemcpyAsync(data, c.p, e->n * 4, cudaMemcpyDeviceToHost, e->stream));
    DG_CUDA(cudaStreamSynchronize(e->stream));
    return DG_OK;
}

extern "C" void dg_edges_free(dg_edges *e) { delete e; }

extern "C" int dg_edges_split(dg_edges *e, double frac, uint64_t seed, dg_lp_pairs **test) {
    DG_CHECK(e && test, DG_ERR_ARG, "dg_edges_split: NULL argument");
    *test = nullptr;
    DG_CHECK(frac >= 0.0 && frac < 1.0, DG_ERR_ARG, "frac must be in [0, 1)");
    dg::DeviceGuard guard(e->device);
    cudaStream_t s = e->stream;
    const unsigned grid = (unsigned)dg::sm_count(e->device) * 8;
    const uint64_t hseed = mix64(seed ^ 0x53504C4953504C49ull);
    dg::DevArray<uint32_t> deg, cand;
    DG_CUDA(deg.alloc(e->v_num));
    DG_CUDA(cand.alloc(e->v_num));
    DG_CUDA(cudaMemsetAsync(deg.p, 0, (size_t)e->v_num * 4, s));
    DG_CUDA(cudaMemsetAsync(cand.p, 0, (size_t)e->v_num * 4, s));
    count_degrees<<<grid, 256, 0, s>>>(e->keys.p, e->n, deg.p);
    dg::note_launch();
    split_count<<<grid, 256, 0, s>>>(e->keys.p, e->n, hseed, frac, cand.p);
    dg::note_launch();
    dg::DevArray<uint8_t> held;
    DG_CUDA(held.alloc(e->n ? e->n : 1));
    split_flag<<<grid, 256, 0, s>>>(e->keys.p, e->n, hseed, frac, deg.p, cand.p, held.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    // Partition: held-out keys first (in key order), kept keys after, reversed (cub's partition layout).
    dg::DevArray<uint64_t> parted;
    dg::DevArray<int64_t> n_sel;
    DG_CUDA(parted.alloc(e->n ? e->n : 1));
    DG_CUDA(n_sel.alloc(1));
    const uint64_t n = e->n;
    int rc = cub_run([&](void *t, size_t &b) {
        return cub::DevicePartition::Flagged(t, b, e->keys.p, held.p, parted.p, n_sel.p, (int64_t)n, s);
    });
    if (rc) return rc;
    int64_t n_held = 0;
    DG_CUDA(cudaMemcpyAsync(&n_held, n_sel.p, 8, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    std::unique_ptr<dg_lp_pairs> t(new dg_lp_pairs());
    t->device = e->device;
    t->n_pos = (uint64_t)n_held;
    t->n_neg = (uint64_t)n_held;
    const uint64_t tot = t->n_pos + t->n_neg;
    DG_CUDA(t->u.alloc(tot ? tot : 1));
    DG_CUDA(t->v.alloc(tot ? tot : 1));
    DG_CUDA(t->label.alloc(tot ? tot : 1));
    split_positives<<<grid, 256, 0, s>>>(parted.p, t->n_pos, t->u.p, t->v.p);
    dg::note_launch();
    dg::DevArray<unsigned int> fail;
    DG_CUDA(fail.alloc(1));
    DG_CUDA(cudaMemsetAsync(fail.p, 0, 4, s));
    // Negatives are checked against the full graph (before the held-out edges leave it).
    split_negatives<<<grid, 256, 0, s>>>(e->keys.p, e->n, e->v_num, t->n_neg, (uint32_t)seed, (uint32_t)(seed >> 32),
                                         t->u.p + t->n_pos, t->v.p + t->n_pos, fail.p);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    if (t->n_pos) DG_CUDA(cudaMemsetAsync(t->label.p, 1, t->n_pos, s));
    if (t->n_neg) DG_CUDA(cudaMemsetAsync(t->label.p + t->n_pos, 0, t->n_neg, s));
    // The kept keys sit after the held-out ones in reverse order: restore key order.
    dg::DevArray<uint64_t> kept;
    const uint64_t n_kept = n - (uint64_t)n_held;
    DG_CUDA(kept.alloc(n_kept ? n_kept : 1));
    if (n_kept) {
        reverse_copy<<<grid, 256, 0, s>>>(parted.p + n_held, n_kept, kept.p);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
    }
    unsigned int h_fail = 0;
    DG_CUDA(cudaMemcpyAsync(&h_fail, fail.p, 4, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    DG_CHECK(h_fail == 0, DG_ERR_ARG, "could not draw a non-edge in 64 tries (graph too dense)");
    e->keys.swap(kept);
    e->n = n_kept;
    *test = t.release();
    return DG_OK;
}

extern "C" int dg_lp_pairs_get_info(const dg_lp_pairs *t, uint64_t *n_pos, uint64_t *n_neg) {
    DG_CHECK(t, DG_ERR_ARG, "dg_lp_pairs_get_info: NULL pairs");
    if (n_pos) *n_pos = t->n_pos;
    if (n_neg) *n_neg = t->n_neg;
    return DG_OK;
}

extern "C" int dg_lp_pairs_copy(const dg_lp_pairs *t, uint32_t *u, uint32_t *v, uint8_t *label) {
    DG_CHECK(t, DG_ERR_ARG, "dg_lp_pairs_copy: NULL pairs");
    dg::DeviceGuard guard(t->device);
    const uint64_t n = t->n_pos + t->n_neg;
    if (!n) return DG_OK;
    if (u) DG_CUDA(cudaMemcpy(u, t->u.p, n * 4, cudaMemcpyDeviceToHost));
    if (v) DG_CUDA(cudaMemcpy(v, t->v.p, n * 4, cudaMemcpyDeviceToHost));
    if (label) DG_CUDA(cudaMemcpy(label, t->label.p, n, cudaMemcpyDeviceToHost));
    return DG_OK;
}

extern "C" void dg_lp_pairs_free(dg_lp_pairs *t) { delete t; }

extern "C" int dg_lp_auc(const dg_sgns *s, const dg_lp_pairs *t, double *auc, double *auc_cosine) {
    DG_CHECK(s && t, DG_ERR_ARG, "dg_lp_auc: NULL argument");
    DG_CHECK(s->device == t->device, DG_ERR_ARG, "trainer and pairs live on different devices");
    dg::DeviceGuard guard(s->device);
    const uint64_t n = t->n_pos + t->n_neg;
    DG_CHECK(n > 0, DG_ERR_ARG, "no test pairs");
    dg::DevArray<uint64_t> sig, cosk;
    DG_CUDA(sig.alloc(n));
    DG_CUDA(cosk.alloc(n));
    const bool plain = dgs::fp32_rows(s);
    const unsigned grid = (unsigned)dg::sm_count(s->device) * 8;
    switch (s->p.size) {
#define DG_LP_CASE(V)                                                                                        \
    case 32 * V:                                                                                             \
        lp_scores<V><<<grid, 256, 0, s->stream>>>(t->u.p, t->v.p, n, s->v2w.p, plain ? s->syn0.p : nullptr, \
                                                  s->in_bf.p, s->in_master.p, plain ? 0u : s->n_master,     \
                                                  sig.p, cosk.p);                                           \
        break;
        DG_LP_CASE(1)
        DG_LP_CASE(2)
        DG_LP_CASE(4)
        DG_LP_CASE(8)
        DG_LP_CASE(16)
#undef DG_LP_CASE
    default:
        return dg::fail(DG_ERR_ARG, "size %d not supported", s->p.size);
    }
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    double a = 0.0, c = 0.0;
    int rc = auc_of(sig.p, t->label.p, n, t->n_pos, s->stream, s->device, &a);
    if (rc) return rc;
    rc = auc_of(cosk.p, t->label.p, n, t->n_pos, s->stream, s->device, &c);
    if (rc) return rc;
    if (auc) *auc = a;
    if (auc_cosine) *auc_cosine = c;
    return DG_OK;
}
