// The two other negative-sampling trainers of word2vec.cu, on FP32 rows over
// device-resident walks, one warp per walk (lane l owns columns
// [l*VEC, l*VEC+VEC) of every row):
//
//  * DG_SGNS_CBOW (DG_SGNS_CBOW_BF16 on BF16 rows): cbow_kernel (word2vec.cu:401-509), the reference's default
//    trainer (cbow = 1, word2vec.cu:59).  Per centre: the mean of the shrunk
//    window's context rows, one positive and `negative` sampled targets, their
//    gradient e added to every context row.
//  * DG_SGNS_SG_SHARED: __sgNegReuse (word2vec.cu:231-303), the reference's
//    skip-gram when -cbow 0 (reuseNeg = 1): one negative set per walk, the
//    full window, the centre's output row as the positive, the context row
//    updated by the pair's e.  The reference instantiates it for size 200 and
//    300 only and exits for others (word2vec.cu:914-926); here every size the
//    trainer supports runs it.  Its dot products are warp sums (the reference's
//    reduceInWarp adds a fixed lane's value at each step, not the partner's).
//
// Per-pair arithmetic is the reference's: cbow e += g*syn1 fused, syn1 +=
// rounded g*neu1; shared-negative e += rounded g*syn1, syn1 += g*l1 fused.
// deterministic = 1: one warp, walks in order, plain loads and stores (bit-
// exact against oracle/dg_oracle_w2v.c's device form).  Hogwild: many warps,
// vector atomics for row updates.
#include "dg_sgns.h"
#include "dg_sgns_dev.cuh"

#include <algorithm>

namespace dgs {

constexpr int kW2vThreads = 256;

// Negative j (0-based) drawn from (c0, walk, pass, tag + j/4), word j%4, with
// word2vec's replacement of index 0 (word2vec.cu:365-368).
__device__ __forceinline__ int32_t tagged_negative(const SgnsArgs &a, uint32_t c0, uint32_t wid, uint32_t tag, int j) {
    const uint4 blk = philox(c0, wid, a.pass, tag + (uint32_t)(j >> 2), a.seed_lo, a.seed_hi);
    const uint32_t q = j & 3;
    const uint32_t r = q == 0 ? blk.x : q == 1 ? blk.y : q == 2 ? blk.z : blk.w;
    int32_t t = a.table[r % a.table_size];
    if (t == 0) t = (int32_t)((r >> 8) % (a.vocab_size - 1) + 1);
    return t;
}

template <int VEC>
__device__ __forceinline__ void zero_row(RowVec<VEC> &r) {
#pragma unroll
    for (int i = 0; i < VEC; i++) r.v[i] = 0.f;
}

// Hierarchical softmax over the Huffman path of `word` (word2vec.cu:334-356,
// 436-455): per inner node, f = x . syn1[node]; nodes with |f| >= MAX_EXP are
// skipped, else g = (1 - code - sigmoid(f)) alpha, e += g syn1[node] (fused),
// syn1[node] += rounded g x.  Inner nodes index the same output table as the
// words, so every node row is read before and written after its own update.
template <int VEC>
__device__ __forceinline__ void hs_path(const SgnsArgs &a, int32_t word, const RowVec<VEC> &x, RowVec<VEC> &e,
                                        uint32_t lane) {
    const int d = 32 * VEC;
    const int32_t k0 = a.hs_off[word], k1 = a.hs_off[word + 1];
    for (int32_t k = k0; k < k1; k++) {
        float *rp = a.syn1 + (size_t)a.hs_point[k] * d + lane * VEC;
        RowVec<VEC> row;
        load_row<VEC>(rp, row);
        const float f = warp_dot<VEC>(x, row);
        if (f <= -kMaxExp || f >= kMaxExp) continue;
        const float g =
            ((float)(1 - a.hs_code[k]) - __ldg(a.exp_table + (int)((f + kMaxExp) * (kExpTableSize / kMaxExp / 2)))) *
            a.alpha;
        RowVec<VEC> upd;
#pragma unroll
        for (int i = 0; i < VEC; i++) {
            e.v[i] = fmaf(g, row.v[i], e.v[i]);
            upd.v[i] = __fmul_rn(g, x.v[i]);
            row.v[i] += upd.v[i];
        }
        if (a.deterministic) store_row<VEC>(rp, row);
        else add_row<VEC>(rp, upd);
    }
}

// ------------------------------------------------------------------ CBOW

// Blocks per SM the CBOW kernel's registers are capped for: the kernel waits on
// row gathers, so residency pays (size 128, YouTube-shaped vocabulary: 44.8 ms
// per pass at four 256-thread blocks and three target rows in flight, 64.8 ms
// at two blocks and six rows).
constexpr int cbow_min_blocks(int vec) { return vec <= 4 ? 4 : 1; }
// Target rows in flight per group: BF16 rows (BF) hold more registers per row
// (the decoded copy and its noise), so size 128 takes two at a time there.
constexpr int cbow_group(int vec, bool bf) { return vec == 4 ? (bf ? 2 : 3) : vec <= 2 ? 4 : 2; }

// G: target rows fetched together (their loads overlap); later groups are
// fetched after the earlier ones are written.
// BF = true: DG_SGNS_CBOW_BF16, the same rule on BF16 rows (FP32 arithmetic;
// FP32 master rows for the hottest words, updated by vector atomics; a BF16
// target row is written as the copy loaded for its dot product plus the update,
// a BF16 context row as its value re-read before the write plus e, each rounded
// stochastically with noise keyed by row, walk, centre and target or window
// slot).
template <int VEC, int G, bool BF>
__global__ void __launch_bounds__(kW2vThreads, cbow_min_blocks(VEC)) sgns_cbow_kernel(SgnsArgs a, WalkSet ws) {
    __shared__ int32_t sen_all[kW2vThreads / 32][kMaxSentence];
    const uint32_t lane = threadIdx.x & 31;
    int32_t *sen = sen_all[threadIdx.x >> 5];
    const int d = 32 * VEC;
    const uint32_t w = (uint32_t)a.window;
    const BfRows<VEC> in{a.in_bf, a.in_master, a.n_master, d};
    const BfRows<VEC> out{a.out_bf, a.out_master, a.n_master, d};
    const uint32_t key = a.seed_lo ^ bf_mix(a.pass * 0x9E3779B9u + 0x5851F42Du);
    // Row `id` of the input (context) or output table, this lane's columns.
    auto load_in = [&](int32_t id, RowVec<VEC> &r) {
        if constexpr (BF) in.load(id, lane, r);
        else load_row<VEC>(a.syn0 + (size_t)id * d + lane * VEC, r);
    };
    auto load_out = [&](int32_t id, RowVec<VEC> &r) {
        if constexpr (BF) out.load(id, lane, r);
        else load_row<VEC>(a.syn1 + (size_t)id * d + lane * VEC, r);
    };
    unsigned long long n_words = 0, n_trained = 0, n_pairs = 0;
    for (;;) {
        uint32_t walk = 0;
        if (lane == 0) walk = atomicAdd(a.queue, 1u);
        walk = __shfl_sync(0xffffffffu, walk, 0);
        if (walk >= ws.n_walks) break;
        const uint32_t wid = ws.ids ? ws.ids[walk] : walk + ws.id_base;
        uint32_t words;
        const uint32_t n = warp_sentence(ws, walk, a, sen, words);
        n_words += words;
        n_trained += n;
        for (uint32_t p = 0; p < n; p++) {
            const int32_t word = sen[p];
            const uint32_t b = philox(p, wid, a.pass, kWinTag, a.seed_lo, a.seed_hi).x % w;
            const uint32_t lo = max(b, w > p ? w - p : 0u), hi = min(2 * w + 1 - b, n + w - p);
            const uint32_t cw = hi > lo ? hi - lo - ((lo <= w && w < hi) ? 1u : 0u) : 0u;
            if (cw == 0) continue;
            n_pairs += cw;
            // neu1: context rows summed in window order (word2vec.cu:419-428), four
            // rows in flight at a time, then divided by their count.
            RowVec<VEC> neu1;
            zero_row(neu1);
            for (uint32_t s = lo; s < hi; s += 4) {
                RowVec<VEC> r[4];
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (s + k < hi && s + k != w) load_in(sen[p - w + s + k], r[k]);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (s + k < hi && s + k != w) {
#pragma unroll
                        for (int i = 0; i < VEC; i++) neu1.v[i] = neu1.v[i] + r[k].v[i];
                    }
            }
#pragma unroll
            for (int i = 0; i < VEC; i++) neu1.v[i] = __fdiv_rn(neu1.v[i], (float)cw);
            // Targets: the centre, then the negatives that differ from it
            // (word2vec.cu:453-462); lane j draws negative j.
            int32_t mine = -1;
            if (a.vocab_size > 1 && (int)lane < a.negative)
                mine = tagged_negative(a, p, wid, kCbowTag, (int)lane);
            const int nt = 1 + (a.vocab_size > 1 ? a.negative : 0);
            RowVec<VEC> e;
            zero_row(e);
            if (!BF && a.hs) hs_path<VEC>(a, word, neu1, e, lane);
            const uint32_t base = BF ? bf_mix(key ^ bf_mix(wid * 0x01000193u + p * 0x2545F491u) ^ lane * 0x85EBCA6Bu) : 0u;
            for (int g0 = 0; g0 < nt; g0 += G) {
                int32_t t[G];
                RowVec<VEC> row[G];
#pragma unroll
                for (int k = 0; k < G; k++) {
                    const int j = g0 + k;
                    t[k] = j >= nt ? -1 : j == 0 ? word : __shfl_sync(0xffffffffu, mine, (j - 1) & 31);
                    if (j > 0 && t[k] == word) t[k] = -1;
                    if (t[k] >= 0) load_out(t[k], row[k]);
                }
#pragma unroll
                for (int k = 0; k < G; k++) {
                    if (t[k] < 0) continue;
                    const float g = sg_grad(warp_dot<VEC>(neu1, row[k]), g0 + k == 0, a.exp_table, a.alpha);
                    RowVec<VEC> upd;
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g, row[k].v[i], e.v[i]);
                        upd.v[i] = __fmul_rn(g, neu1.v[i]);
                        row[k].v[i] += upd.v[i];
                    }
                    if constexpr (BF) {
                        const uint32_t salt = base + (uint32_t)t[k] * 0x27D4EB2Fu + (uint32_t)(g0 + k);
                        if (a.deterministic) out.put(t[k], lane, row[k], salt);
                        else out.update(t[k], lane, upd, row[k], salt);
                    } else {
                        float *rp = a.syn1 + (size_t)t[k] * d + lane * VEC;
                        if (a.deterministic) store_row<VEC>(rp, row[k]);
                        else add_row<VEC>(rp, upd);
                    }
                    // A repeat of this target later in the group sees this update.
#pragma unroll
                    for (int q = k + 1; q < G; q++)
                        if (t[q] == t[k]) row[q] = row[k];
                }
            }
            // e to every context row, in window order (word2vec.cu:498-505).
            for (uint32_t s = lo; s < hi; s++) {
                if (s == w) continue;
                if constexpr (BF) {
                    // The row as it is now (a repeat of a context word in the
                    // window sees the earlier slot's store), plus e.
                    const int32_t cw = sen[p - w + s];
                    RowVec<VEC> r;
                    zero_row(r);
                    if ((uint32_t)cw >= a.n_master || a.deterministic) in.load(cw, lane, r);
#pragma unroll
                    for (int i = 0; i < VEC; i++) r.v[i] = r.v[i] + e.v[i];
                    const uint32_t salt = base + (uint32_t)cw * 0x165667B1u + s * 16u + 15u;
                    if (a.deterministic) in.put(cw, lane, r, salt);
                    else in.update(cw, lane, e, r, salt);
                    continue;
                }
                float *cp = a.syn0 + (size_t)sen[p - w + s] * d + lane * VEC;
                if (a.deterministic) {
                    RowVec<VEC> r;
                    load_row<VEC>(cp, r);
#pragma unroll
                    for (int i = 0; i < VEC; i++) r.v[i] = r.v[i] + e.v[i];
                    store_row<VEC>(cp, r);
                } else {
                    add_row<VEC>(cp, e);
                }
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_words);
        atomicAdd(&a.stats[1], n_trained);
        atomicAdd(&a.stats[2], n_pairs);
    }
}

// ------------------------------------------------ shared-negative skip-gram

// Negative rows fetched together per pair (their loads overlap).
constexpr int kShareGroup = 4;

// One negative set per walk (kept in shared memory), the full window; per pair
// the negatives that differ from the centre, then the centre as the positive,
// each against the unchanged context row.  Negative rows are read and written
// at every pair, as the reference writes them (an update that a hot negative
// row receives from another warp is seen at the next pair, so no warp holds a
// stale copy for long); the centre's output row stays in registers for the
// centre, as in the plain kernels.  Hogwild: vector atomics add the rounded
// increments g*l1 (the reference adds g*l1 to the row fused, without atomics).
template <int VEC>
__global__ void __launch_bounds__(kW2vThreads) sgns_negshare_kernel(SgnsArgs a, WalkSet ws) {
    __shared__ int32_t sen_all[kW2vThreads / 32][kMaxSentence];
    __shared__ int32_t negs_all[kW2vThreads / 32][kShareMaxNeg];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t *sen = sen_all[warp];
    int32_t *negs = negs_all[warp];
    const int d = 32 * VEC;
    const int neg = a.vocab_size > 1 ? a.negative : 0;
    const uint32_t w = (uint32_t)a.window;
    unsigned long long n_words = 0, n_trained = 0, n_pairs = 0;
    for (;;) {
        uint32_t walk = 0;
        if (lane == 0) walk = atomicAdd(a.queue, 1u);
        walk = __shfl_sync(0xffffffffu, walk, 0);
        if (walk >= ws.n_walks) break;
        const uint32_t wid = ws.ids ? ws.ids[walk] : walk + ws.id_base;
        uint32_t words;
        const uint32_t n = warp_sentence(ws, walk, a, sen, words);
        n_words += words;
        n_trained += n;
        if (n < 2) continue;
        __syncwarp();
        if ((int)lane < neg) negs[lane] = tagged_negative(a, 0, wid, kShareTag, (int)lane);
        __syncwarp();
        for (uint32_t p = 0; p < n; p++) {
            const int32_t word = sen[p];
            RowVec<VEC> pos, pos0;
            load_row<VEC>(a.syn1 + (size_t)word * d + lane * VEC, pos);
            pos0 = pos;
            const uint32_t lo = w > p ? w - p : 0u, hi = min(2 * w + 1, n + w - p);
            for (uint32_t s = lo; s < hi; s++) {
                if (s == w) continue;
                n_pairs++;
                float *l1p = a.syn0 + (size_t)sen[p - w + s] * d + lane * VEC;
                RowVec<VEC> l1, e;
                load_row<VEC>(l1p, l1);
                zero_row(e);
                // Negatives in order, those equal to the centre skipped (word2vec.cu:
                // 256-297: warps y < negative, then y = negative for the positive).
                for (int j0 = 0; j0 < neg; j0 += kShareGroup) {
                    int32_t t[kShareGroup];
                    RowVec<VEC> row[kShareGroup];
#pragma unroll
                    for (int k = 0; k < kShareGroup; k++) {
                        t[k] = j0 + k < neg ? negs[j0 + k] : -1;
                        if (t[k] == word) t[k] = -1;
                        if (t[k] >= 0) load_row<VEC>(a.syn1 + (size_t)t[k] * d + lane * VEC, row[k]);
                    }
#pragma unroll
                    for (int k = 0; k < kShareGroup; k++) {
                        if (t[k] < 0) continue;
                        const float g = sg_grad(warp_dot<VEC>(l1, row[k]), 0, a.exp_table, a.alpha);
                        RowVec<VEC> upd;
#pragma unroll
                        for (int i = 0; i < VEC; i++) {
                            e.v[i] += __fmul_rn(g, row[k].v[i]);
                            upd.v[i] = __fmul_rn(g, l1.v[i]);
                            row[k].v[i] = fmaf(g, l1.v[i], row[k].v[i]);
                        }
                        float *rp = a.syn1 + (size_t)t[k] * d + lane * VEC;
                        if (a.deterministic) store_row<VEC>(rp, row[k]);
                        else add_row<VEC>(rp, upd);
                        // A repeat of this negative later in the group sees this update.
#pragma unroll
                        for (int q = k + 1; q < kShareGroup; q++)
                            if (t[q] == t[k]) row[q] = row[k];
                    }
                }
                {   // the positive: the centre's output row
                    const float g = sg_grad(warp_dot<VEC>(l1, pos), 1, a.exp_table, a.alpha);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] += __fmul_rn(g, pos.v[i]);
                        pos.v[i] = fmaf(g, l1.v[i], pos.v[i]);
                    }
                }
                if (a.deterministic) {
#pragma unroll
                    for (int i = 0; i < VEC; i++) l1.v[i] = l1.v[i] + e.v[i];
                    store_row<VEC>(l1p, l1);
                } else {
                    add_row<VEC>(l1p, e);
                }
            }
            float *dst = a.syn1 + (size_t)word * d + lane * VEC;
            if (a.deterministic) {
                store_row<VEC>(dst, pos);
            } else {
#pragma unroll
                for (int i = 0; i < VEC; i++) pos.v[i] -= pos0.v[i];
                add_row<VEC>(dst, pos);
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_words);
        atomicAdd(&a.stats[1], n_trained);
        atomicAdd(&a.stats[2], n_pairs);
    }
}

// ------------------------------------------- skip-gram with hierarchical softmax

// skip_gram_kernel with -hs 1 (word2vec.cu:330-397): per (context, centre) pair
// the centre's Huffman path, then the positive and the negatives (the plain
// kernels' draws), every target row read before and written after its own update,
// then the context row.  No row is kept in registers across pairs: an inner node
// can be the row of the centre word itself.
template <int VEC>
__global__ void __launch_bounds__(kW2vThreads) sgns_plain_hs_kernel(SgnsArgs a, WalkSet ws) {
    __shared__ int32_t sen_all[kW2vThreads / 32][kMaxSentence];
    const uint32_t lane = threadIdx.x & 31;
    int32_t *sen = sen_all[threadIdx.x >> 5];
    const int d = 32 * VEC;
    const uint32_t w = (uint32_t)a.window;
    const int neg = a.vocab_size > 1 ? a.negative : 0;
    unsigned long long n_words = 0, n_trained = 0, n_pairs = 0;
    for (;;) {
        uint32_t walk = 0;
        if (lane == 0) walk = atomicAdd(a.queue, 1u);
        walk = __shfl_sync(0xffffffffu, walk, 0);
        if (walk >= ws.n_walks) break;
        const uint32_t wid = ws.ids ? ws.ids[walk] : walk + ws.id_base;
        uint32_t words;
        const uint32_t n = warp_sentence(ws, walk, a, sen, words);
        n_words += words;
        n_trained += n;
        for (uint32_t p = 0; p < n; p++) {
            const int32_t word = sen[p];
            const uint32_t b = philox(p, wid, a.pass, kWinTag, a.seed_lo, a.seed_hi).x % w;
            const uint32_t lo = max(b, w > p ? w - p : 0u), hi = min(2 * w + 1 - b, n + w - p);
            for (uint32_t s = lo; s < hi; s++) {
                if (s == w) continue;
                n_pairs++;
                float *l1p = a.syn0 + (size_t)sen[p - w + s] * d + lane * VEC;
                RowVec<VEC> l1, e;
                load_row<VEC>(l1p, l1);
                zero_row(e);
                hs_path<VEC>(a, word, l1, e, lane);
                for (int j = 0; j <= neg; j++) {
                    int32_t t = word;
                    if (j > 0) {
                        t = tagged_negative(a, p * (2 * w + 1) + s, wid, kNegTag, j - 1);
                        if (t == word) continue;
                    }
                    float *rp = a.syn1 + (size_t)t * d + lane * VEC;
                    RowVec<VEC> row, upd;
                    load_row<VEC>(rp, row);
                    const float g = sg_grad(warp_dot<VEC>(l1, row), j == 0, a.exp_table, a.alpha);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g, row.v[i], e.v[i]);
                        upd.v[i] = __fmul_rn(g, l1.v[i]);
                        row.v[i] += upd.v[i];
                    }
                    if (a.deterministic) store_row<VEC>(rp, row);
                    else add_row<VEC>(rp, upd);
                }
                if (a.deterministic) {
#pragma unroll
                    for (int i = 0; i < VEC; i++) l1.v[i] = l1.v[i] + e.v[i];
                    store_row<VEC>(l1p, l1);
                } else {
                    add_row<VEC>(l1p, e);
                }
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_words);
        atomicAdd(&a.stats[1], n_trained);
        atomicAdd(&a.stats[2], n_pairs);
    }
}

// --------------------------------------------------------------- launchers

template <typename K>
static int resident_blocks(K kern, int threads, size_t smem, int device) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    return std::max(per_sm, 1) * dg::sm_count(device);
}

// Threads per block: one warp in deterministic mode; a worker count below a
// block's eight warps is one block of that many warps.
static int w2v_threads(const dg_sgns *s) {
    if (s->p.deterministic) return 32;
    if (s->p.workers > 0 && s->p.workers < (uint32_t)(kW2vThreads / 32)) return 32 * (int)s->p.workers;
    return kW2vThreads;
}

static int worker_blocks(const dg_sgns *s, int resident, int threads) {
    if (s->p.workers == 0) return resident;
    const int want = (int)((s->p.workers + threads / 32 - 1) / (threads / 32));
    return std::max(1, std::min(resident, want));
}

template <int V, bool BF>
static int cbow_launch(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    constexpr int G = cbow_group(V, BF);
    auto kern = sgns_cbow_kernel<V, G, BF>;
    const int threads = w2v_threads(s);
    const int blocks = s->p.deterministic ? 1 : worker_blocks(s, resident_blocks(kern, threads, 0, s->device), threads);
    kern<<<blocks, threads, 0, s->stream>>>(a, ws);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    return DG_OK;
}

template <int V>
static int negshare_launch(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    auto kern = sgns_negshare_kernel<V>;
    const int threads = w2v_threads(s);
    const int blocks = s->p.deterministic ? 1 : worker_blocks(s, resident_blocks(kern, threads, 0, s->device), threads);
    kern<<<blocks, threads, 0, s->stream>>>(a, ws);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    return DG_OK;
}

int launch_cbow(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    if (s->p.mode == DG_SGNS_CBOW_BF16) {
        switch (s->p.size / 32) {
            case 2: return cbow_launch<2, true>(s, a, ws);
            case 4: return cbow_launch<4, true>(s, a, ws);
            case 8: return cbow_launch<8, true>(s, a, ws);
            default: return dg::fail(DG_ERR_ARG, "size %d not supported on BF16 rows (64, 128, 256)", s->p.size);
        }
    }
    switch (s->p.size / 32) {
        case 1: return cbow_launch<1, false>(s, a, ws);
        case 2: return cbow_launch<2, false>(s, a, ws);
        case 4: return cbow_launch<4, false>(s, a, ws);
        case 8: return cbow_launch<8, false>(s, a, ws);
        case 16: return cbow_launch<16, false>(s, a, ws);
        default: return dg::fail(DG_ERR_ARG, "size %d not supported (32, 64, 128, 256, 512)", s->p.size);
    }
}

template <int V>
static int plain_hs_launch(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    auto kern = sgns_plain_hs_kernel<V>;
    const int threads = w2v_threads(s);
    const int blocks = s->p.deterministic ? 1 : worker_blocks(s, resident_blocks(kern, threads, 0, s->device), threads);
    kern<<<blocks, threads, 0, s->stream>>>(a, ws);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    return DG_OK;
}

int launch_plain_hs(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    switch (s->p.size / 32) {
        case 1: return plain_hs_launch<1>(s, a, ws);
        case 2: return plain_hs_launch<2>(s, a, ws);
        case 4: return plain_hs_launch<4>(s, a, ws);
        case 8: return plain_hs_launch<8>(s, a, ws);
        case 16: return plain_hs_launch<16>(s, a, ws);
        default: return dg::fail(DG_ERR_ARG, "size %d not supported (32, 64, 128, 256, 512)", s->p.size);
    }
}

int launch_negshare(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    switch (s->p.size / 32) {
        case 1: return negshare_launch<1>(s, a, ws);
        case 2: return negshare_launch<2>(s, a, ws);
        case 4: return negshare_launch<4>(s, a, ws);
        case 8: return negshare_launch<8>(s, a, ws);
        case 16: return negshare_launch<16>(s, a, ws);
        default: return dg::fail(DG_ERR_ARG, "size %d not supported (32, 64, 128, 256, 512)", s->p.size);
    }
}

}  // namespace dgs
