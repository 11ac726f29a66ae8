// Information-oriented random walk (DistGER / HuGE transition, entropy
// termination) as one persistent kernel, plus the per-round bookkeeping the
// reference does on the host (visit frequencies, relative entropy, walk files).
//
// Compiled with -fmad=false; the FP64 termination state is in addition written
// with explicit round-to-nearest intrinsics so that every operation is one IEEE
// rounding in the order of include/walk.hpp:284-354.
#include "dg_internal.h"
#include "dg_philox.cuh"

#include <cmath>
#include <cstring>
#include <memory>

namespace {

// Launch shapes of walk_kernel: walks per block (one walk per thread) and the
// first footprints of each walk cached in shared memory.  Variant 0 is the
// default; dg_walk_autotune times them all and keeps the fastest per graph.
struct WalkShape {
    int threads, steps;
};
constexpr WalkShape kWalkShapes[] = {{256, 24}, {128, 24}, {256, 16}, {256, 32}, {512, 16}, {128, 48}};
constexpr int kWalkShapeCount = (int)(sizeof(kWalkShapes) / sizeof(kWalkShapes[0]));
constexpr uint32_t kWalkTag = 0x57414C4Bu; // Philox counter word 3 for walk draws ("WALK")
constexpr uint32_t kDefaultStride = 64;

// Seeded replay: one Philox block per transition attempt, counter = (attempt,
// walker, round, tag), key = seed.

struct WalkArgs {
    const uint64_t *__restrict__ offsets;
    const uint2 *__restrict__ entries;
    const double *__restrict__ etable;
    uint32_t *__restrict__ verts;
    uint32_t *__restrict__ lens;
    uint32_t *__restrict__ freq;
    uint32_t *next;                 // work queue head
    unsigned long long *stats;      // footprints, draws, traces, overflows
    uint32_t *max_len;
    uint32_t n_walks, v_num, stride, min_len, round, seed_lo, seed_hi;
};

// Running entropy / effectiveness state of one walk (Correlation, walk.hpp:260-387).
// N equals S at every step (both start at 1 and grow by 1), so one variable serves both.
struct Corr {
    double S, H, EH, ES, EHS, EHH, ESS, R;
};

// Correlation::iterate with step_k = 1 (walk.hpp:317-354); t = log2 term from the table.
__device__ __forceinline__ void corr_iterate(Corr &c, double t) {
    const double S1 = __dadd_rn(c.S, 1.0);
    const double H1 = __ddiv_rn(__dsub_rn(__dmul_rn(c.S, c.H), t), S1);
    c.EH = __dadd_rn(c.EH, __ddiv_rn(__dsub_rn(H1, c.EH), S1));
    c.ES = __dadd_rn(c.ES, __ddiv_rn(__dsub_rn(S1, c.ES), S1));
    c.EHS = __dadd_rn(c.EHS, __ddiv_rn(__dsub_rn(__dmul_rn(H1, S1), c.EHS), S1));
    c.EHH = __dadd_rn(c.EHH, __ddiv_rn(__dsub_rn(__dmul_rn(H1, H1), c.EHH), S1));
    c.ESS = __dadd_rn(c.ESS, __ddiv_rn(__dsub_rn(__dmul_rn(S1, S1), c.ESS), S1));
    const double DH = __dsub_rn(c.EHH, __dmul_rn(c.EH, c.EH));
    const double DS = __dsub_rn(c.ESS, __dmul_rn(c.ES, c.ES));
    const double e = __dsub_rn(c.EHS, __dmul_rn(c.EH, c.ES));
    c.R = e == 0.0 ? 0.0 : __ddiv_rn(e, __dsqrt_rn(__dmul_rn(DH, DS)));
    c.H = H1;
    c.S = S1;
}

// walk.hpp:868-872: stop once step > min_len and (R^2 < 0.999 or R < 0).
__device__ __forceinline__ bool corr_stop(const Corr &c, uint32_t step, uint32_t min_len) {
    return step > min_len && (__dmul_rn(c.R, c.R) < 0.999 || c.R < 0.0);
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Persistent walk kernel: each thread pulls walker ids from a device queue and
// advances that walk to completion (walk.hpp:845-1024 with every vertex local).
// Per transition attempt: one Philox block, two loads for the row bounds, one
// 8-byte CSR entry {neighbour, acceptance threshold}; the accept test is an
// integer compare.  The walk's footprints go to its arena slot and, for the first
// kSmemSteps, to a shared-memory copy that serves the prior-visit count
// (the unordered_map of walk.hpp:816).
template <int THREADS, int STEPS>
__global__ void __launch_bounds__(THREADS) walk_kernel(WalkArgs a) {
    __shared__ uint32_t cache[STEPS][THREADS];
    const int tid = threadIdx.x;
    unsigned long long n_fp = 0, n_draw = 0, n_trace = 0, n_over = 0;
    uint32_t longest = 0;
    for (;;) {
        const uint32_t w = atomicAdd(a.next, 1u);
        if (w >= a.n_walks) break;
        uint32_t *path = a.verts + (uint64_t)w * a.stride;
        uint32_t cur = w % a.v_num;
        uint32_t n = 0;

        // Appends v and returns its prior-visit count.
        auto visit_count = [&](uint32_t v) -> uint32_t {
            uint32_t c = 0;
            const uint32_t hot = n < (uint32_t)STEPS ? n : (uint32_t)STEPS;
            for (uint32_t i = 0; i < hot; i++) c += cache[i][tid] == v;
            for (uint32_t i = STEPS; i < n; i++) c += path[i] == v;
            return c;
        };
        auto push = [&](uint32_t v) {
            if (n < (uint32_t)STEPS) cache[n][tid] = v;
            path[n] = v;
            atomicAdd(&a.freq[v], 1u);
            n++;
        };

        push(cur);
        Corr c{1.0, 0.0, 0.0, 1.0, 0.0, 0.0, 1.0, 1.0};  // walk.hpp:853-855
        uint32_t attempt = 0;
        for (;;) {
            const uint64_t row = a.offsets[cur];
            const uint32_t deg = (uint32_t)(a.offsets[cur + 1] - row);
            if (deg == 0) break;  // walk.hpp:887-892
            const uint4 x = philox4x32_10(make_uint4(attempt, w, a.round, kWalkTag), a.seed_lo, a.seed_hi);
            attempt++;
            n_draw++;
            const uint32_t slot = (uint32_t)__umul64hi(((uint64_t)x.y << 32) | x.x, (uint64_t)deg);
            if (deg == 2 && a.entries[row].x == cur) break;  // walk.hpp:900-902
            const uint2 ent = a.entries[row + slot];
            if (n == 1 && ent.x == cur) continue;          // walk.hpp:904-906 (step == 0)
            const bool trace = (x.z & 0x7fffffffu) >= ent.y; // tanh(p_accept) <= rand()/RAND_MAX
            n_trace += trace;
            const uint32_t dst = ent.x;
            if (n == a.stride) { n_over++; break; }
            uint32_t fi = visit_count(dst);
            double t = a.etable[(uint64_t)n * (n + 1) / 2 + fi - 1];
            push(dst);
            corr_iterate(c, t);
            if (corr_stop(c, n - 1, a.min_len)) break;
            if (trace) {  // walk.hpp:986-1017: step back to the current vertex
                if (n == a.stride) { n_over++; break; }
                fi = visit_count(cur);
                t = a.etable[(uint64_t)n * (n + 1) / 2 + fi - 1];
                push(cur);
                corr_iterate(c, t);
                if (corr_stop(c, n - 1, a.min_len)) break;
            } else {
                cur = dst;
            }
        }
        a.lens[w] = n;
        n_fp += n;
        longest = n > longest ? n : longest;
    }
    n_fp = warp_sum(n_fp);
    n_draw = warp_sum(n_draw);
    n_trace = warp_sum(n_trace);
    n_over = warp_sum(n_over);
#pragma unroll
    for (int o = 16; o; o >>= 1) longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, o));
    if ((tid & 31) == 0) {
        atomicAdd(&a.stats[0], n_fp);
        atomicAdd(&a.stats[1], n_draw);
        atomicAdd(&a.stats[2], n_trace);
        if (n_over) atomicAdd(&a.stats[3], n_over);
        atomicMax(a.max_len, longest);
    }
}

// Per-block partial sums of p_i * (log p_i - log q_i) (walk.hpp:706-725).
constexpr int kEntropyThreads = 256;
__global__ void entropy_partials(const uint32_t *__restrict__ deg, const uint32_t *__restrict__ freq, uint32_t v_num,
                                 double degree_sum, double words_sum, double *partial) {
    __shared__ double red[kEntropyThreads];
    double acc = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < v_num; i += (uint64_t)gridDim.x * blockDim.x) {
        const double pi = (double)deg[i] / degree_sum;
        const double qi = (double)freq[i] / words_sum;
        acc += pi * (log(pi) - log(qi));
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kEntropyThreads / 2; s; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Walk-file bytes of each walk: " %u" per vertex plus "\n".
__device__ __forceinline__ uint32_t ndigits(uint32_t v) {
    uint32_t d = 1;
    while (v >= 10) { v /= 10; d++; }
    return d;
}

__global__ void text_lengths(const uint32_t *__restrict__ verts, const uint32_t *__restrict__ lens, uint32_t n_walks,
                             uint32_t stride, uint32_t *bytes) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n_walks; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t *p = verts + w * stride;
        uint32_t b = 1;
        for (uint32_t i = 0; i < lens[w]; i++) b += 1 + ndigits(p[i]);
        bytes[w] = b;
    }
}

__global__ void text_write(const uint32_t *__restrict__ verts, const uint32_t *__restrict__ lens, uint32_t n_walks,
                           uint32_t stride, const uint64_t *__restrict__ at, char *out) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n_walks; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t *p = verts + w * stride;
        char *o = out + at[w];
        for (uint32_t i = 0; i < lens[w]; i++) {
            uint32_t v = p[i];
            const uint32_t d = ndigits(v);
            *o++ = ' ';
            for (uint32_t k = d; k > 0; k--) {
                o[k - 1] = (char)('0' + v % 10);
                v /= 10;
            }
            o += d;
        }
        *o = '\n';
    }
}

// Warp per walk: copies a slot into the compacted walker-order corpus.
__global__ void compact_walks(const uint32_t *__restrict__ verts, const uint32_t *__restrict__ lens, uint32_t n_walks,
                              uint32_t stride, const uint64_t *__restrict__ at, uint32_t *out) {
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n_walks;
         w += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint32_t *p = verts + w * stride;
        uint32_t *o = out + at[w];
        for (uint32_t i = lane; i < lens[w]; i += 32) o[i] = p[i];
    }
}

int relative_entropy(dg_graph *g, uint64_t words_sum, double *h) {
    const int blocks = dg::sm_count(g->device) * 4;
    dg::DevArray<double> &partial = g->entropy_partial;
    if (partial.n < (size_t)blocks) DG_CUDA(partial.alloc(blocks));
    entropy_partials<<<blocks, kEntropyThreads, 0, g->stream>>>(g->out_deg.p, g->freq.p, g->v_num, (double)g->m,
                                                                  (double)words_sum, partial.p); dg::note_launch();
    DG_CUDA(cudaGetLastError());
    std::vector<double> host(blocks);
    DG_CUDA(cudaMemcpyAsync(host.data(), partial.p, blocks * sizeof(double), cudaMemcpyDeviceToHost, g->stream));
    DG_CUDA(cudaStreamSynchronize(g->stream));
    double s = 0.0;
    for (double v : host) s += v;
    *h = s;
    return DG_OK;
}

// One launch of walk_kernel in launch shape I: a persistent grid of as many
// blocks as fit (each thread pulls walker ids from the queue).
template <int I>
int walk_launch_shape(dg_graph *g, const WalkArgs &a, uint32_t n_walkers) {
    constexpr int T = kWalkShapes[I].threads, S = kWalkShapes[I].steps;
    int per_sm = 0;
    DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, walk_kernel<T, S>, T, 0));
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = (uint64_t)dg::sm_count(g->device) * per_sm;
    const uint64_t needed = ((uint64_t)n_walkers + T - 1) / T;
    if (blocks > needed) blocks = needed ? needed : 1;
    walk_kernel<T, S><<<(unsigned)blocks, T, 0, g->stream>>>(a);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    return DG_OK;
}

int walk_launch(int shape, dg_graph *g, const WalkArgs &a, uint32_t n_walkers) {
    static_assert(kWalkShapeCount == 6, "dispatch below lists every shape");
    switch (shape) {
    case 0: return walk_launch_shape<0>(g, a, n_walkers);
    case 1: return walk_launch_shape<1>(g, a, n_walkers);
    case 2: return walk_launch_shape<2>(g, a, n_walkers);
    case 3: return walk_launch_shape<3>(g, a, n_walkers);
    case 4: return walk_launch_shape<4>(g, a, n_walkers);
    case 5: return walk_launch_shape<5>(g, a, n_walkers);
    default: return dg::fail(DG_ERR_ARG, "walk launch shape %d out of range", shape);
    }
}

// shape < 0: the graph's current (tuned) launch shape.
int run_round(dg_graph *g, const dg_walk_params *p, uint32_t round, uint32_t n_walkers, uint32_t stride,
              std::unique_ptr<dg_paths> &out, int shape = -1) {
    DG_CHECK(stride >= 2 && stride <= (1u << 16), DG_ERR_ARG, "max_len %u out of range [2, 65536]", stride);
    int rc = dg::ensure_entropy_table(g, stride);
    if (rc) return rc;
    std::unique_ptr<dg_paths> ps(new dg_paths());
    ps->g = g;
    ps->device = g->device;
    ps->round = round;
    ps->n_walks = n_walkers;
    ps->stride = stride;
    if (g->spare_verts.n >= (size_t)n_walkers * stride && g->spare_lens.n >= n_walkers) {
        ps->verts.swap(g->spare_verts);   // the arena of a freed round (its walks are not read again)
        ps->lens.swap(g->spare_lens);
    } else {
        DG_CUDA(ps->verts.alloc((size_t)n_walkers * stride));
        DG_CUDA(ps->lens.alloc(n_walkers));
    }

    dg::DevArray<unsigned long long> &stats = g->round_stats;
    dg::DevArray<uint32_t> &ctl = g->round_ctl;  // [0] queue head, [1] longest walk
    if (!stats.p) DG_CUDA(stats.alloc(4));
    if (!ctl.p) DG_CUDA(ctl.alloc(2));
    DG_CUDA(cudaMemsetAsync(stats.p, 0, 4 * sizeof(unsigned long long), g->stream));
    DG_CUDA(cudaMemsetAsync(ctl.p, 0, 2 * sizeof(uint32_t), g->stream));
    // Keep the pre-round visit counts so a failed (overflowing) round can be undone.
    dg::DevArray<uint32_t> &freq_backup = g->freq_backup;
    if (freq_backup.n < g->v_num) DG_CUDA(freq_backup.alloc(g->v_num));
    DG_CUDA(cudaMemcpyAsync(freq_backup.p, g->freq.p, (size_t)g->v_num * 4, cudaMemcpyDeviceToDevice, g->stream));

    WalkArgs a;
    a.offsets = g->offsets.p;
    a.entries = g->entries.p;
    a.etable = g->etable.p;
    a.verts = ps->verts.p;
    a.lens = ps->lens.p;
    a.freq = g->freq.p;
    a.next = ctl.p;
    a.stats = stats.p;
    a.max_len = ctl.p + 1;
    a.n_walks = n_walkers;
    a.v_num = g->v_num;
    a.stride = stride;
    a.min_len = p->min_len;
    a.round = round;
    a.seed_lo = (uint32_t)p->seed;
    a.seed_hi = (uint32_t)(p->seed >> 32);

    dg::EventTimer t;
    t.start(g->stream);
    rc = walk_launch(shape < 0 ? g->walk_shape : shape, g, a, n_walkers);
    if (rc) return rc;
    t.stop(g->stream);
    unsigned long long h_stats[4];
    uint32_t h_ctl[2];
    DG_CUDA(cudaMemcpyAsync(h_stats, stats.p, sizeof(h_stats), cudaMemcpyDeviceToHost, g->stream));
    DG_CUDA(cudaMemcpyAsync(h_ctl, ctl.p, sizeof(h_ctl), cudaMemcpyDeviceToHost, g->stream));
    DG_CUDA(cudaStreamSynchronize(g->stream));
    if (h_stats[3]) {
        DG_CUDA(cudaMemcpyAsync(g->freq.p, freq_backup.p, (size_t)g->v_num * 4, cudaMemcpyDeviceToDevice, g->stream));
        DG_CUDA(cudaStreamSynchronize(g->stream));
        return dg::fail(DG_ERR_OVERFLOW, "%llu walks of round %u exceeded max_len = %u footprints",
                        h_stats[3], round, stride);
    }
    dg_round_info &inf = ps->info;
    inf.n_walks = n_walkers;
    inf.footprints = h_stats[0];
    inf.steps = h_stats[0] - n_walkers;
    inf.draws = h_stats[1];
    inf.traces = h_stats[2];
    inf.max_len = h_ctl[1];
    inf.walk_ms = t.ms();

    out.swap(ps);
    return DG_OK;
}

}  // namespace

extern "C" int dg_walk_run_round(dg_graph *g, const dg_walk_params *p, uint32_t round, uint32_t n_walkers,
                                 dg_paths **out) {
    DG_CHECK(g && p && out, DG_ERR_ARG, "dg_walk_run_round: NULL argument");
    *out = nullptr;
    DG_CHECK(p->walker_num > 0 || n_walkers > 0, DG_ERR_ARG, "dg_walk_run_round: walker_num is 0");
    DG_CHECK(round > 0, DG_ERR_ARG, "dg_walk_run_round: rounds are numbered from 1");
    uint64_t n = n_walkers;
    if (n == 0) n = round == 1 ? (uint64_t)p->walker_num * (p->init_round ? p->init_round : 5) : p->walker_num;
    DG_CHECK(n > 0 && n < (1ull << 32), DG_ERR_ARG, "walker count %llu out of range", (unsigned long long)n);
    const uint32_t stride = p->max_len ? p->max_len : kDefaultStride;
    dg::DeviceGuard guard(g->device);
    std::unique_ptr<dg_paths> ps;
    int rc = run_round(g, p, round, (uint32_t)n, stride, ps);
    if (rc) return rc;

    // Relative entropy of cumulative visits vs degree share (walk.hpp:693-734).
    g->visits_total += ps->info.footprints;
    double h = 0.0;
    rc = relative_entropy(g, g->visits_total, &h);
    if (rc) return rc;
    const double prev = g->entropy_history.empty() ? 0.0 : g->entropy_history.back();
    ps->info.relative_entropy = h;
    ps->info.delta_h = g->entropy_history.empty() ? h : h - prev;
    g->entropy_history.push_back(h);
    *out = ps.release();
    return DG_OK;
}

extern "C" int dg_paths_get_info(const dg_paths *paths, dg_round_info *info) {
    DG_CHECK(paths && info, DG_ERR_ARG, "dg_paths_get_info: NULL argument");
    *info = paths->info;
    return DG_OK;
}

extern "C" int dg_paths_copy(const dg_paths *ps, uint64_t *offsets, uint32_t *vertices) {
    DG_CHECK(ps, DG_ERR_ARG, "dg_paths_copy: NULL paths");
    dg::DeviceGuard guard(ps->device);
    dg_graph *g = ps->g;
    cudaStream_t s = g->stream;
    dg::DevArray<uint64_t> &at = g->copy_at;
    if (at.n < (size_t)ps->n_walks + 1) DG_CUDA(at.alloc((size_t)ps->n_walks + 1));
    int rc = dg::exclusive_scan_u32_to_u64(ps->lens.p, at.p, ps->n_walks, s);
    if (rc) return rc;
    if (offsets) DG_CUDA(cudaMemcpyAsync(offsets, at.p, ((size_t)ps->n_walks + 1) * 8, cudaMemcpyDeviceToHost, s));
    if (vertices && ps->info.footprints) {
        dg::DevArray<uint32_t> &flat = g->copy_flat;
        if (flat.n < ps->info.footprints) DG_CUDA(flat.alloc(ps->info.footprints + ps->info.footprints / 8));
        compact_walks<<<dg::sm_count(ps->device) * 8, 256, 0, s>>>(ps->verts.p, ps->lens.p, ps->n_walks, ps->stride,
                                                                     at.p, flat.p); dg::note_launch();
        DG_CUDA(cudaGetLastError());
        DG_CUDA(cudaMemcpyAsync(vertices, flat.p, ps->info.footprints * 4, cudaMemcpyDeviceToHost, s));
    }
    DG_CUDA(cudaStreamSynchronize(s));
    return DG_OK;
}

extern "C" int dg_paths_write_text(const dg_paths *ps, const char *file_path) {
    DG_CHECK(ps && file_path, DG_ERR_ARG, "dg_paths_write_text: NULL argument");
    dg::DeviceGuard guard(ps->device);
    cudaStream_t s = ps->g->stream;
    const int blocks = dg::sm_count(ps->device) * 8;
    dg::DevArray<uint32_t> nbytes;
    dg::DevArray<uint64_t> at;
    DG_CUDA(nbytes.alloc(ps->n_walks ? ps->n_walks : 1));
    DG_CUDA(at.alloc((size_t)ps->n_walks + 1));
    text_lengths<<<blocks, 256, 0, s>>>(ps->verts.p, ps->lens.p, ps->n_walks, ps->stride, nbytes.p); dg::note_launch();
    DG_CUDA(cudaGetLastError());
    int rc = dg::exclusive_scan_u32_to_u64(nbytes.p, at.p, ps->n_walks, s);
    if (rc) return rc;
    uint64_t total = 0;
    DG_CUDA(cudaMemcpy(&total, at.p + ps->n_walks, 8, cudaMemcpyDeviceToHost));
    std::vector<char> host(total);
    if (total) {
        dg::DevArray<char> text;
        DG_CUDA(text.alloc(total));
        text_write<<<blocks, 256, 0, s>>>(ps->verts.p, ps->lens.p, ps->n_walks, ps->stride, at.p, text.p); dg::note_launch();
        DG_CUDA(cudaGetLastError());
        DG_CUDA(cudaStreamSynchronize(s));
        DG_CUDA(cudaMemcpy(host.data(), text.p, total, cudaMemcpyDeviceToHost));
    }
    FILE *f = fopen(file_path, "wb");
    DG_CHECK(f != nullptr, DG_ERR_IO, "cannot open %s for writing", file_path);
    size_t put = total ? fwrite(host.data(), 1, total, f) : 0;
    int cl = fclose(f);
    DG_CHECK(put == total && cl == 0, DG_ERR_IO, "short write to %s", file_path);
    return DG_OK;
}

extern "C" void dg_paths_free(dg_paths *ps) {
    if (!ps) return;
    dg::DeviceGuard guard(ps->device);
    cudaStreamSynchronize(ps->g->stream);
    // The graph keeps the largest freed arena for its next round.
    dg_graph *g = ps->g;
    if (ps->verts.n > g->spare_verts.n) {
        g->spare_verts.swap(ps->verts);
        g->spare_lens.swap(ps->lens);
    }
    delete ps;
}

// Times every launch shape of walk_kernel on `n_walkers` walkers of `round` and
// keeps the fastest for this graph.  Walks do not depend on the shape (each
// walker's draws are keyed by its id), so tuning changes speed only; the visit
// counts the trial rounds add are restored, and no round is recorded.
extern "C" int dg_walk_autotune(dg_graph *g, const dg_walk_params *p, uint32_t round, uint32_t n_walkers,
                                dg_tune_info *info) {
    DG_CHECK(g && p, DG_ERR_ARG, "dg_walk_autotune: NULL argument");
    DG_CHECK(round > 0, DG_ERR_ARG, "dg_walk_autotune: rounds are numbered from 1");
    uint64_t n = n_walkers ? n_walkers : p->walker_num;
    DG_CHECK(n > 0 && n < (1ull << 32), DG_ERR_ARG, "walker count %llu out of range", (unsigned long long)n);
    const uint32_t stride = p->max_len ? p->max_len : kDefaultStride;
    dg::DeviceGuard guard(g->device);
    dg::DevArray<uint32_t> saved;
    DG_CUDA(saved.alloc(g->v_num));
    DG_CUDA(cudaMemcpyAsync(saved.p, g->freq.p, (size_t)g->v_num * 4, cudaMemcpyDeviceToDevice, g->stream));
    dg_tune_info r{};
    r.n_candidates = kWalkShapeCount;
    double best = 1e300;
    for (int k = 0; k < kWalkShapeCount; k++) {
        double ms = 0.0;
        for (int rep = 0; rep < 2; rep++) {   // the first run warms caches and the queue
            std::unique_ptr<dg_paths> ps;
            int rc = run_round(g, p, round, (uint32_t)n, stride, ps, k);
            if (rc) {
                cudaMemcpyAsync(g->freq.p, saved.p, (size_t)g->v_num * 4, cudaMemcpyDeviceToDevice, g->stream);
                cudaStreamSynchronize(g->stream);
                return rc;
            }
            ms = ps->info.walk_ms;
        }
        if (k < DG_TUNE_MAX) {
            r.ms[k] = ms;
            r.shape[k][0] = kWalkShapes[k].threads;
            r.shape[k][1] = kWalkShapes[k].steps;
        }
        if (ms < best) {
            best = ms;
            r.chosen = k;
        }
    }
    DG_CUDA(cudaMemcpyAsync(g->freq.p, saved.p, (size_t)g->v_num * 4, cudaMemcpyDeviceToDevice, g->stream));
    DG_CUDA(cudaStreamSynchronize(g->stream));
    g->walk_shape = r.chosen;
    if (info) *info = r;
    return DG_OK;
}

extern "C" int dg_walk_set_shape(dg_graph *g, int shape) {
    DG_CHECK(g, DG_ERR_ARG, "dg_walk_set_shape: NULL graph");
    DG_CHECK(shape >= 0 && shape < kWalkShapeCount, DG_ERR_ARG, "walk launch shape %d out of range [0, %d)", shape,
             kWalkShapeCount);
    g->walk_shape = shape;
    return DG_OK;
}
