// Minibatch SGNS with shared negatives: the update rule of dsgl.hpp
// Train_SGNS_MPI (dsgl.hpp:783-1407) on BF16 rows with FP32 accumulation.
//
// One CTA is one dsgl worker: it owns a contiguous slice of the walks and keeps
// two sentences in flight.  Per step (one position in each sentence):
//   inputs  I <= 2 * 2 * window : context rows of both centres, same shrink b
//                                 (dsgl.hpp:1097-1127), from per-sentence caches;
//   outputs O <= negative + 2   : centre 1, the step's group of the shared
//                                 negative pool (duplicates merged with a count,
//                                 dsgl.hpp:1131-1156), centre 2;
//   corr (O x I) = outputs . inputs^T -> g = (label - sigmoid) * alpha * count,
//   row 0 positive against sentence-1 columns, row O-1 against sentence-2
//   columns (dsgl.hpp:1241-1274);
//   outputs += corr . inputs,  inputs += corr^T . outputs (dsgl.hpp:1290-1311).
// Sentence caches live in shared memory (FP32); the negative pool lives in this
// CTA's slice of a global scratch area (FP32).  Caches are written back as
// deltas when a sentence ends (inputs) or after two sentences (pool), so that
// concurrent workers do not overwrite each other.  BF16 rows are rounded
// stochastically; the hottest rows (lowest vocabulary ids) are FP32 masters
// updated with atomics.
//
// The contractions are O x I x d = 7 x 40 x 128 per step for the reference
// configuration: far below one tcgen05 tile (M >= 64), so they run as
// thread-per-dot products and thread-per-column updates on FP32 CUDA cores.
#include "dg_sgns.h"

#include <algorithm>
#include <mutex>

namespace dgs {

constexpr int kMbThreads = 128;
constexpr int kMbMaxSent = 64;              // tokens per sentence (= distinct rows per cache)
constexpr uint32_t kMbWinTag = 0x4D425749u; // "MBWI": window shrink of step s
constexpr uint32_t kMbPoolTag = 0x4D42504Fu; // "MBPO": negative pool sample j of pool p

struct MbArgs {
    float *scratch;            // per worker: pool_cur, pool_init (pool_cap x d each), sent_init (2 x 64 x d)
    uint64_t scratch_stride;   // floats per worker
    uint32_t pool_cap;         // kMbMaxSent * negative
    int max_out, max_in;
};

__device__ __forceinline__ uint32_t mix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}

// FP32 -> BF16 with stochastic rounding: add 16 random bits below the kept
// mantissa and truncate (unbiased in expectation).
__device__ __forceinline__ __nv_bfloat16 bf16_sr(float x, uint32_t noise) {
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7F800000u) != 0x7F800000u) u += noise & 0xFFFFu;
    return __ushort_as_bfloat16((unsigned short)(u >> 16));
}

struct MbRows {
    __nv_bfloat16 *bf;
    float *master;
    uint32_t n_master;
    int d;
    __device__ __forceinline__ float get(int32_t w, int k) const {
        return (uint32_t)w < n_master ? __ldcg(master + (size_t)w * d + k) : __bfloat162float(bf[(size_t)w * d + k]);
    }
    // row[w][k] += delta
    __device__ __forceinline__ void add(int32_t w, int k, float delta, uint32_t noise) const {
        if ((uint32_t)w < n_master) {
            atomicAdd(master + (size_t)w * d + k, delta);
        } else {
            __nv_bfloat16 *p = bf + (size_t)w * d + k;
            *p = bf16_sr(__bfloat162float(*p) + delta, noise);
        }
    }
};

template <int D>
__global__ void __launch_bounds__(kMbThreads) sgns_mb_kernel(SgnsArgs a, WalkSet ws, MbArgs m) {
    constexpr int LD = D + 1;                        // padded row stride (bank-conflict free)
    constexpr int CPT = D >= kMbThreads ? D / kMbThreads : 1;
    extern __shared__ float smem[];
    const int tid = threadIdx.x;
    const int MO = m.max_out, MI = m.max_in;
    float *cache = smem;                              // [2][kMbMaxSent][LD]
    float *outs = cache + 2 * kMbMaxSent * LD;        // [MO][LD]
    float *gm = outs + MO * LD;                       // [MO][MI]
    int *ip = reinterpret_cast<int *>(gm + MO * MI);
    int *sen = ip;                                    // [2][kMbMaxSent] vocabulary ids
    int *slot = sen + 2 * kMbMaxSent;                 // [2][kMbMaxSent] token -> cache row
    int *dist = slot + 2 * kMbMaxSent;                // [2][kMbMaxSent] cache row -> word
    int *in_row = dist + 2 * kMbMaxSent;              // [MI] cache row (+ kMbMaxSent for sentence 2)
    int *out_word = in_row + MI;                      // [MO]
    int *out_meta = out_word + MO;                    // [MO]
    int *out_slot = out_meta + MO;                    // [MO] pool slot, -1 for centres
    int *pool_slot = out_slot + MO;                   // [pool_cap] sample -> pool slot
    int *pool_word = pool_slot + m.pool_cap;          // [pool_cap] pool slot -> word

    __shared__ int s_len[2], s_pos[2], s_ndist[2], s_walk[2];
    __shared__ int s_npool, s_nbn, s_O, s_I, s_first;
    __shared__ unsigned long long s_words, s_trained, s_pairs;

    const uint32_t worker = blockIdx.x;
    const uint32_t W = ws.n_walks, G = gridDim.x;
    const uint32_t w_begin = (uint32_t)((uint64_t)W * worker / G), w_end = (uint32_t)((uint64_t)W * (worker + 1) / G);
    float *pool_cur = m.scratch + (uint64_t)worker * m.scratch_stride;
    float *pool_init = pool_cur + (uint64_t)m.pool_cap * D;
    float *sent_init = pool_init + (uint64_t)m.pool_cap * D;   // [2][kMbMaxSent][D]
    const uint32_t key0 = a.seed_lo ^ mix32(a.pass * 0x9E3779B9u + 0x632BE5ABu), key1 = a.seed_hi;
    const MbRows in_rows{a.in_bf, a.in_master, a.n_master, D};
    const MbRows out_rows{a.out_bf, a.out_master, a.n_master, D};
    const float alpha = a.alpha;
    const int window = a.window, negative = a.negative;

    if (tid == 0) {
        s_len[0] = s_len[1] = 0;
        s_words = s_trained = s_pairs = 0;
        s_npool = 0;
    }
    uint32_t next_walk = w_begin;   // uniform across the CTA
    uint32_t step = 0, pool_no = 0, neg_count = 0;
    int train_sen_num = 0;
    bool change_neg = true, pool_loaded = false;
    __syncthreads();

    // Writes back cache s as a delta against the rows it was loaded from.
    auto flush_sentence = [&](int s) {
        const int nd = s_ndist[s];
        for (int r = 0; r < nd; r++) {
            const int w = dist[s * kMbMaxSent + r];
            for (int c = 0; c < CPT; c++) {
                const int k = tid + c * kMbThreads;
                if (k < D) {
                    const float cur = cache[(s * kMbMaxSent + r) * LD + k];
                    const float ini = sent_init[((uint64_t)s * kMbMaxSent + r) * D + k];
                    in_rows.add(w, k, cur - ini, mix32(key0 ^ mix32(w * 0x01000193u + k) ^ (step << 1) ^ s));
                }
            }
        }
    };
    auto flush_pool = [&]() {
        const int np = s_npool;
        for (int r = 0; r < np; r++) {
            const int w = pool_word[r];
            for (int c = 0; c < CPT; c++) {
                const int k = tid + c * kMbThreads;
                if (k < D) {
                    const float d = pool_cur[(uint64_t)r * D + k] - pool_init[(uint64_t)r * D + k];
                    out_rows.add(w, k, d, mix32(key1 ^ mix32(w * 0x01000193u + k) ^ (step << 2) ^ 0x55u));
                }
            }
        }
    };

    for (;;) {
        // ---- fill empty sentence slots (dsgl.hpp:903-1028) ----
        for (int s = 0; s < 2; s++) {
            while (true) {
                __syncthreads();
                if (s_len[s] != 0) break;
                if (next_walk >= w_end) break;
                const uint32_t walk = next_walk++;
                if (tid < 32) {
                    // vocabulary lookup + subsampling, compacted by ballot
                    uint64_t begin;
                    uint32_t len;
                    ws.range(walk, begin, len);
                    if (len > kMbMaxSent) len = kMbMaxSent;
                    const uint32_t wid = ws.ids ? ws.ids[walk] : walk + ws.id_base;
                    uint32_t n = 0;
                    for (uint32_t base = 0; base < len; base += 32) {
                        const uint32_t i = base + tid;
                        bool keep = false;
                        int32_t w = -1;
                        if (i < len) {
                            w = a.v2w[ws.verts[begin + i]];
                            if (w >= 0) {
                                const uint32_t u = philox4x32_10(make_uint4(i, wid, a.pass, kSubTag), a.seed_lo,
                                                                 a.seed_hi).x & 0xFFFFu;
                                keep = u < a.keep_thr[w];
                            }
                        }
                        const uint32_t mask = __ballot_sync(0xffffffffu, keep);
                        if (keep) sen[s * kMbMaxSent + n + __popc(mask & ((1u << tid) - 1))] = w;
                        n += __popc(mask);
                    }
                    __syncwarp();
                    // distinct words in first-occurrence order (dsgl.hpp:948-956)
                    int nd = 0;
                    for (uint32_t t = 0; t < n; t++) {
                        const int w = sen[s * kMbMaxSent + t];
                        const bool hit0 = tid < nd && dist[s * kMbMaxSent + tid] == w;
                        const bool hit1 = tid + 32 < nd && dist[s * kMbMaxSent + tid + 32] == w;
                        const uint32_t m0 = __ballot_sync(0xffffffffu, hit0), m1 = __ballot_sync(0xffffffffu, hit1);
                        int r;
                        if (m0) r = __ffs(m0) - 1;
                        else if (m1) r = 32 + __ffs(m1) - 1;
                        else {
                            r = nd;
                            if (tid == 0) dist[s * kMbMaxSent + nd] = w;
                            nd++;
                        }
                        if (tid == 0) slot[s * kMbMaxSent + t] = r;
                        __syncwarp();
                    }
                    if (tid == 0) {
                        s_words += len;
                        s_trained += n;
                        s_len[s] = n <= 1 ? 0 : (int)n;   // dsgl.hpp:941-945
                        s_pos[s] = 0;
                        s_ndist[s] = nd;
                        s_walk[s] = (int)wid;
                    }
                }
                __syncthreads();
                if (s_len[s] != 0) {
                    const int nd = s_ndist[s];
                    for (int r = 0; r < nd; r++) {
                        const int w = dist[s * kMbMaxSent + r];
                        for (int c = 0; c < CPT; c++) {
                            const int k = tid + c * kMbThreads;
                            if (k < D) {
                                const float v = in_rows.get(w, k);
                                cache[(s * kMbMaxSent + r) * LD + k] = v;
                                sent_init[((uint64_t)s * kMbMaxSent + r) * D + k] = v;
                            }
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (s_len[0] == 0 || s_len[1] == 0) break;   // slice exhausted (dsgl.hpp:1029-1049)

        // ---- shared negative pool (dsgl.hpp:1052-1083) ----
        if (change_neg) {
            if (tid == 0) {
                const int nbn = max(s_len[0], s_len[1]);
                int np = 0;
                for (int j = 0; j < nbn * negative; j++) {
                    uint4 x = philox4x32_10(make_uint4((uint32_t)j >> 2, pool_no, worker, kMbPoolTag), key0, key1);
                    const uint32_t q = j & 3;
                    const uint32_t r = q == 0 ? x.x : q == 1 ? x.y : q == 2 ? x.z : x.w;
                    int32_t smp = a.table[r % a.table_size];
                    if (!smp) smp = a.vocab_size > 1 ? (int32_t)((r >> 8) % (a.vocab_size - 1) + 1) : 0;
                    int at = -1;
                    for (int t = 0; t < np; t++)
                        if (pool_word[t] == smp) { at = t; break; }
                    if (at < 0) { at = np; pool_word[np++] = smp; }
                    pool_slot[j] = at;
                }
                s_npool = np;
                s_nbn = nbn;
            }
            __syncthreads();
            const int np = s_npool;
            for (int r = 0; r < np; r++) {
                const int w = pool_word[r];
                for (int c = 0; c < CPT; c++) {
                    const int k = tid + c * kMbThreads;
                    if (k < D) {
                        const float v = out_rows.get(w, k);
                        pool_cur[(uint64_t)r * D + k] = v;
                        pool_init[(uint64_t)r * D + k] = v;
                    }
                }
            }
            pool_no++;
            change_neg = false;
            pool_loaded = true;
        }

        // ---- step bookkeeping: inputs and outputs (dsgl.hpp:1089-1160) ----
        if (tid == 0) {
            const uint32_t b = philox4x32_10(make_uint4(step, worker, 0, kMbWinTag), key0, key1).x % (uint32_t)window;
            int ni = 0;
            for (int s = 0; s < 2; s++) {
                const int pos = s_pos[s], len = s_len[s];
                for (int i = (int)b; i < 2 * window + 1 - (int)b; i++) {
                    if (i == window) continue;
                    const int c = pos - window + i;
                    if (c < 0) continue;
                    if (c >= len) break;
                    in_row[ni++] = s * kMbMaxSent + slot[s * kMbMaxSent + c];
                }
                if (s == 0) s_first = ni;
            }
            s_I = ni;
            neg_count++;
            const int start = (int)(neg_count % (uint32_t)s_nbn);
            int off = 1;
            out_word[0] = sen[s_pos[0]];
            out_meta[0] = 1;
            out_slot[0] = -1;
            for (int k = 0; k < negative; k++) {
                const int ps = pool_slot[start * negative + k];
                const int smp = pool_word[ps];
                int at = -1;
                for (int t = 0; t < off; t++)
                    if (out_word[t] == smp) { at = t; break; }
                if (at < 0) {
                    out_word[off] = smp;
                    out_meta[off] = 1;
                    out_slot[off] = ps;
                    off++;
                } else {
                    out_meta[at]++;
                }
            }
            out_meta[0] = 1;                          // dsgl.hpp:1153-1154
            out_word[off] = sen[kMbMaxSent + s_pos[1]];
            out_meta[off] = 1;
            out_slot[off] = -1;
            s_O = off + 1;
            s_pairs += ni;
        }
        __syncthreads();
        const int O = s_O, I = s_I, first = s_first;

        // ---- stage output rows (target rows from the tables, negatives from the pool) ----
        for (int o = 0; o < O; o++) {
            const int w = out_word[o], ps = out_slot[o];
            for (int c = 0; c < CPT; c++) {
                const int k = tid + c * kMbThreads;
                if (k < D) outs[o * LD + k] = ps < 0 ? out_rows.get(w, k) : pool_cur[(uint64_t)ps * D + k];
            }
        }
        __syncthreads();

        // ---- corr = outputs . inputs^T, gradients (dsgl.hpp:1241-1274) ----
        for (int q = tid; q < O * I; q += kMbThreads) {
            const int o = q / I, i = q - o * I;
            const float *x = outs + o * LD;
            const float *y = cache + in_row[i] * LD;
            float f = 0.f;
#pragma unroll 8
            for (int k = 0; k < D; k++) f = fmaf(x[k], y[k], f);
            const int label = i < first ? (o == 0) : (o == O - 1);
            float g;
            if (f > kMaxExp) g = (label - 1) * alpha;
            else if (f < -kMaxExp) g = label * alpha;
            else g = (label - a.exp_table[(int)((f + kMaxExp) * (kExpTableSize / kMaxExp / 2))]) * alpha;
            gm[o * MI + i] = g * (float)out_meta[o];
        }
        __syncthreads();

        // ---- outputs += corr . inputs ; inputs += corr^T . outputs (dsgl.hpp:1290-1396) ----
        for (int c = 0; c < CPT; c++) {
            const int k = tid + c * kMbThreads;
            if (k >= D) continue;
            float md[24];
#pragma unroll
            for (int o = 0; o < 24; o++) {
                if (o >= O) break;
                float acc = 0.f;
                for (int i = 0; i < I; i++) acc = fmaf(gm[o * MI + i], cache[in_row[i] * LD + k], acc);
                md[o] = acc;
            }
            for (int i = 0; i < I; i++) {
                float acc = 0.f;
                for (int o = 0; o < O; o++) acc = fmaf(gm[o * MI + i], outs[o * LD + k], acc);
                cache[in_row[i] * LD + k] += acc;
            }
            const uint32_t salt = mix32(key0 + step * 0x9E3779B9u + (uint32_t)k);
            out_rows.add(out_word[0], k, md[0], mix32(salt ^ (uint32_t)out_word[0]));
            out_rows.add(out_word[O - 1], k, md[O - 1], mix32(salt ^ (uint32_t)out_word[O - 1] ^ 0xA5A5u));
#pragma unroll
            for (int o = 1; o < 23; o++) {
                if (o >= O - 1) break;
                pool_cur[(uint64_t)out_slot[o] * D + k] += md[o];
            }
        }
        __syncthreads();

        // ---- advance; write back finished sentences and spent pools (dsgl.hpp:1398-1424) ----
        step++;
        const int p0 = s_pos[0] + 1, p1 = s_pos[1] + 1;
        const bool end0 = p0 >= s_len[0], end1 = p1 >= s_len[1];
        if (end0) { flush_sentence(0); train_sen_num++; }
        if (end1) { flush_sentence(1); train_sen_num++; }
        if (train_sen_num >= 2) {
            flush_pool();
            change_neg = true;
            pool_loaded = false;
            train_sen_num = 0;
        }
        __syncthreads();
        if (tid == 0) {
            s_pos[0] = p0;
            s_pos[1] = p1;
            if (end0) s_len[0] = 0;
            if (end1) s_len[1] = 0;
        }
    }
    // Slice exhausted: keep the updates of the sentence still in flight and of
    // the pool (dsgl drops them; here they are written back).
    __syncthreads();
    for (int s = 0; s < 2; s++)
        if (s_len[s] != 0) flush_sentence(s);
    if (pool_loaded) flush_pool();
    if (tid == 0) {
        atomicAdd(&a.stats[0], s_words);
        atomicAdd(&a.stats[1], s_trained);
        atomicAdd(&a.stats[2], s_pairs);
    }
}

static size_t mb_smem_bytes(int d, int max_out, int max_in, uint32_t pool_cap) {
    const size_t ld = (size_t)d + 1;
    size_t f = 2 * kMbMaxSent * ld + (size_t)max_out * ld + (size_t)max_out * max_in;
    size_t i = 6 * kMbMaxSent + (size_t)max_in + 3 * (size_t)max_out + 2 * (size_t)pool_cap;
    return f * 4 + i * 4;
}

int launch_minibatch(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    const int d = s->p.size;
    DG_CHECK(d <= 256, DG_ERR_ARG, "minibatch mode supports size <= 256 (got %d)", d);
    DG_CHECK(a.negative <= 22, DG_ERR_ARG, "minibatch mode supports negative <= 22 (got %d)", a.negative);
    MbArgs m{};
    m.pool_cap = (uint32_t)kMbMaxSent * (uint32_t)std::max(a.negative, 1);
    m.max_out = a.negative + 2;
    m.max_in = 4 * a.window;
    const size_t smem = mb_smem_bytes(d, m.max_out, m.max_in, m.pool_cap);
    m.scratch_stride = (uint64_t)m.pool_cap * d * 2 + 2ull * kMbMaxSent * d;
    int per_sm = 1;
    auto setup = [&](auto kern) -> int {
        DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMbThreads, smem));
        return DG_OK;
    };
    int rc = DG_OK;
    switch (d) {
    case 32: rc = setup(sgns_mb_kernel<32>); break;
    case 64: rc = setup(sgns_mb_kernel<64>); break;
    case 128: rc = setup(sgns_mb_kernel<128>); break;
    case 256: rc = setup(sgns_mb_kernel<256>); break;
    default: return dg::fail(DG_ERR_ARG, "size %d not supported in minibatch mode", d);
    }
    if (rc) return rc;
    DG_CHECK(per_sm >= 1, DG_ERR_ARG, "minibatch kernel does not fit (%zu bytes of shared memory)", smem);
    uint32_t workers = a.deterministic ? 1u : (uint32_t)(dg::sm_count(s->device) * per_sm);
    if (workers > ws.n_walks / 2 + 1) workers = std::max(1u, ws.n_walks / 2);
    const uint64_t need = m.scratch_stride * workers;
    if (s->scratch.n < need) DG_CUDA(s->scratch.alloc(need));
    m.scratch = s->scratch.p;
    switch (d) {
    case 32: sgns_mb_kernel<32><<<workers, kMbThreads, smem, s->stream>>>(a, ws, m); break;
    case 64: sgns_mb_kernel<64><<<workers, kMbThreads, smem, s->stream>>>(a, ws, m); break;
    case 128: sgns_mb_kernel<128><<<workers, kMbThreads, smem, s->stream>>>(a, ws, m); break;
    case 256: sgns_mb_kernel<256><<<workers, kMbThreads, smem, s->stream>>>(a, ws, m); break;
    }
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    return DG_OK;
}

}  // namespace dgs

// ---------------------------------------------------------------------------
// Allocation-free entry point: the minibatch trainer with its per-worker
// scratch (negative pools and cache snapshots) in a fixed device array that is
// part of this library, so that a call performs no device or host allocation.
// It serves callers that must not allocate: code running inside a CUDA graph
// capture, a memory pool owned by a framework that forbids foreign cudaMalloc,
// or a real-time loop that cannot pay an allocator's latency or failure modes.
// ---------------------------------------------------------------------------
namespace dgs {
namespace {

// Scratch shared by every call on a device (held by each GPU that loads the library).
constexpr size_t kNoAllocScratchBytes = 16u << 20;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchBytes / sizeof(float)];
static __device__ __align__(256) unsigned long long g_noalloc_stats[4];

// Device address of the scratch array, looked up once per device (the host-side
// name of a __device__ array is not a device address).
struct NoAllocSetup {
    std::mutex mu;
    float *scratch[kNoAllocMaxDevices] = {};
    unsigned long long *stats[kNoAllocMaxDevices] = {};
};
NoAllocSetup &noalloc_setup() {
    static NoAllocSetup s;
    return s;
}

int noalloc_pointers(int device, float **scratch, unsigned long long **stats) {
    DG_CHECK(device >= 0 && device < kNoAllocMaxDevices, DG_ERR_ARG, "device %d beyond the %d supported", device,
             kNoAllocMaxDevices);
    NoAllocSetup &s = noalloc_setup();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.scratch[device]) {
        void *p = nullptr, *q = nullptr;
        DG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        DG_CUDA(cudaGetSymbolAddress(&q, g_noalloc_stats));
        s.scratch[device] = static_cast<float *>(p);
        s.stats[device] = static_cast<unsigned long long *>(q);
    }
    *scratch = s.scratch[device];
    *stats = s.stats[device];
    return DG_OK;
}

}  // namespace
}  // namespace dgs

extern "C" int dg_sgns_minibatch_train_noalloc(const dg_sgns_minibatch_args *x, void *stream, dg_train_info *info) {
    using namespace dgs;
    DG_CHECK(x, DG_ERR_ARG, "dg_sgns_minibatch_train_noalloc: NULL arguments");
    DG_CHECK(x->verts && x->offsets && x->v2w && x->keep_thr && x->table && x->exp_table, DG_ERR_ARG,
             "dg_sgns_minibatch_train_noalloc: walk or table pointer is NULL");
    DG_CHECK(x->in_bf16 && x->out_bf16 && (x->n_master == 0 || (x->in_master && x->out_master)), DG_ERR_ARG,
             "dg_sgns_minibatch_train_noalloc: row pointer is NULL");
    const int d = x->size;
    DG_CHECK(d == 32 || d == 64 || d == 128 || d == 256, DG_ERR_ARG, "size %d not supported (32, 64, 128, 256)", d);
    DG_CHECK(x->window >= 1 && x->window <= 64, DG_ERR_ARG, "window %d out of range [1, 64]", x->window);
    DG_CHECK(x->negative >= 0 && x->negative <= 22, DG_ERR_ARG, "negative %d out of range [0, 22]", x->negative);
    DG_CHECK(x->vocab_size > 0 && x->table_size > 0 && x->table_size < (1ull << 32), DG_ERR_ARG,
             "empty vocabulary or unigram table");
    int device = 0;
    DG_CUDA(cudaGetDevice(&device));
    float *scratch = nullptr;
    unsigned long long *stats = nullptr;
    int rc = noalloc_pointers(device, &scratch, &stats);
    if (rc) return rc;

    MbArgs m{};
    m.pool_cap = (uint32_t)kMbMaxSent * (uint32_t)std::max(x->negative, 1);
    m.max_out = x->negative + 2;
    m.max_in = 4 * x->window;
    m.scratch_stride = (uint64_t)m.pool_cap * d * 2 + 2ull * kMbMaxSent * d;
    m.scratch = scratch;
    const uint64_t per_worker = m.scratch_stride * sizeof(float);
    const uint64_t max_workers = kNoAllocScratchBytes / per_worker;
    DG_CHECK(max_workers >= 1, DG_ERR_ARG,
             "size %d with negative %d needs %llu bytes of scratch per worker, more than the %zu-byte static area",
             d, x->negative, (unsigned long long)per_worker, kNoAllocScratchBytes);
    const size_t smem = mb_smem_bytes(d, m.max_out, m.max_in, m.pool_cap);
    int per_sm = 1;
    auto setup = [&](auto kern) -> int {
        DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMbThreads, smem));
        return DG_OK;
    };
    switch (d) {
    case 32: rc = setup(sgns_mb_kernel<32>); break;
    case 64: rc = setup(sgns_mb_kernel<64>); break;
    case 128: rc = setup(sgns_mb_kernel<128>); break;
    default: rc = setup(sgns_mb_kernel<256>); break;
    }
    if (rc) return rc;
    DG_CHECK(per_sm >= 1, DG_ERR_ARG, "minibatch kernel does not fit (%zu bytes of shared memory)", smem);
    uint64_t workers = x->deterministic ? 1 : (uint64_t)dg::sm_count(device) * per_sm;
    workers = std::min<uint64_t>(workers, max_workers);
    if (workers > x->n_walks / 2 + 1) workers = std::max<uint64_t>(1, x->n_walks / 2);

    SgnsArgs a{};
    a.v2w = x->v2w;
    a.keep_thr = x->keep_thr;
    a.table = x->table;
    a.exp_table = x->exp_table;
    a.in_bf = reinterpret_cast<__nv_bfloat16 *>(x->in_bf16);
    a.out_bf = reinterpret_cast<__nv_bfloat16 *>(x->out_bf16);
    a.in_master = x->in_master;
    a.out_master = x->out_master;
    a.n_master = x->n_master;
    a.stats = stats;
    a.table_size = x->table_size;
    a.vocab_size = x->vocab_size;
    a.window = x->window;
    a.negative = x->negative;
    a.d = d;
    a.alpha = x->alpha;
    a.pass = x->pass;
    a.seed_lo = (uint32_t)x->seed;
    a.seed_hi = (uint32_t)(x->seed >> 32);
    a.deterministic = x->deterministic;
    WalkSet ws{};
    ws.verts = x->verts;
    ws.offsets = x->offsets;
    ws.n_walks = x->n_walks;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DG_CUDA(cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), s));  // counters start at zero every call
    switch (d) {
    case 32: sgns_mb_kernel<32><<<(unsigned)workers, kMbThreads, smem, s>>>(a, ws, m); break;
    case 64: sgns_mb_kernel<64><<<(unsigned)workers, kMbThreads, smem, s>>>(a, ws, m); break;
    case 128: sgns_mb_kernel<128><<<(unsigned)workers, kMbThreads, smem, s>>>(a, ws, m); break;
    default: sgns_mb_kernel<256><<<(unsigned)workers, kMbThreads, smem, s>>>(a, ws, m); break;
    }
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    if (info) {
        unsigned long long st[4];
        DG_CUDA(cudaMemcpyAsync(st, stats, sizeof(st), cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        info->words = st[0];
        info->trained = st[1];
        info->pairs = st[2];
        info->train_ms = 0.0;
    }
    return DG_OK;
}
