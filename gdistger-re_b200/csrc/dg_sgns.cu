// Skip-gram negative-sampling trainer over device-resident walks.
//
//  * plain form (DG_SGNS_PLAIN): the update rule of word2vec.cu skip_gram_kernel
//    (word2vec.cu:305-399) on FP32 rows; one warp per walk, each lane owning
//    size/32 contiguous dimensions, dot products by warp shuffles, Hogwild
//    vector atomics between warps;
//  * minibatch form (DG_SGNS_MINIBATCH): dsgl.hpp Train_SGNS_MPI semantics
//    (dsgl.hpp:783-1407), see dg_sgns_mb.cu.
#include "dg_sgns.h"
#include "dg_sgns_dev.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <thread>

namespace dgs {

// ------------------------------------------------------------------ host prep

// ReadVocabFromDegree + SortVocab (word2vec.cu:791-809, 632-659).
void build_vocab(const uint32_t *counts, uint32_t v_num, int min_count, std::vector<uint32_t> &ids,
                 std::vector<uint32_t> &cn, std::vector<int32_t> &v2w, uint64_t &train_words) {
    std::vector<uint32_t> order(v_num);
    for (uint32_t v = 0; v < v_num; v++) order[v] = v;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return counts[a] > counts[b]; });
    v2w.assign(v_num, -1);
    ids.clear();
    cn.clear();
    train_words = 0;
    for (uint32_t i = 0; i < v_num; i++) {
        const uint32_t v = order[i];
        if ((int64_t)counts[v] < min_count && i != 0) continue;
        v2w[v] = (int32_t)ids.size();
        ids.push_back(v);
        cn.push_back(counts[v]);
        train_words += counts[v];
    }
}

// InitUnigramTable (word2vec.cu:537-556), power 0.75.
void unigram_table(const std::vector<uint32_t> &cn, uint64_t table_size, std::vector<int32_t> &table) {
    const uint32_t vs = (uint32_t)cn.size();
    table.resize(table_size);
    double train_words_pow = 0;
    for (uint32_t a = 0; a < vs; a++) train_words_pow += std::pow((double)cn[a], 0.75);
    uint32_t i = 0;
    double d1 = std::pow((double)cn[0], 0.75) / train_words_pow;
    for (uint64_t a = 0; a < table_size; a++) {
        table[a] = (int32_t)i;
        if (a / (double)table_size > d1) {
            i++;
            if (i < vs) d1 += std::pow((double)cn[i], 0.75) / train_words_pow;
        }
        if (i >= vs) i = vs - 1;
    }
}

// Subsampling: a token of word w is kept iff its 16 random bits are < thr[w]
// (discard iff ran < u / 65536, word2vec.cu:1022-1026 or dsgl.hpp:931-937).
void keep_thresholds(const std::vector<uint32_t> &cn, float sample, uint64_t train_words, bool dsgl_form,
                     std::vector<uint32_t> &thr) {
    thr.resize(cn.size());
    for (size_t w = 0; w < cn.size(); w++) {
        if (!(sample > 0)) {
            thr[w] = 65536;
            continue;
        }
        const float sT = sample * (float)train_words;
        float ran;
        if (dsgl_form) {
            const float ratio = sT / (float)cn[w];
            ran = std::sqrt(ratio) + ratio;
        } else {
            ran = (std::sqrt((float)cn[w] / sT) + 1) * sT / (float)cn[w];
        }
        uint32_t k;
        if (ran != ran || ran < 0.0f) k = 0;
        else if (ran >= 1.0f) k = 65536;
        else k = std::min<uint32_t>(65536, (uint32_t)std::floor(ran * 65536.0f) + 1);
        thr[w] = k;
    }
}

// CreateBinaryTree (word2vec.cu:684-740): the two smallest of the sorted counts
// and the inner nodes made so far are merged (bit 1 for the second), then each
// word's path is read back from the root: bit k of word a is decided by inner
// node point[k] (0 .. n-2; the root is n-2).  Layout of InitVocabStructCUDA
// (word2vec.cu:511-535): off[a] .. off[a+1] index word a's bits.
bool huffman_codes(const std::vector<uint32_t> &cn, std::vector<int32_t> &off, std::vector<int32_t> &point,
                   std::vector<int8_t> &code) {
    const int64_t n = (int64_t)cn.size();
    if (n < 2) return false;
    std::vector<int64_t> count(2 * n + 1, 0), parent(2 * n + 1, 0);
    std::vector<int8_t> binary(2 * n + 1, 0);
    for (int64_t a = 0; a < n; a++) count[a] = cn[a];
    for (int64_t a = n; a < 2 * n; a++) count[a] = (int64_t)1e15;
    int64_t p1 = n - 1, p2 = n;
    for (int64_t a = 0; a + 1 < n; a++) {
        int64_t m[2];
        for (int k = 0; k < 2; k++) m[k] = (p1 >= 0 && count[p1] < count[p2]) ? p1-- : p2++;
        count[n + a] = count[m[0]] + count[m[1]];
        parent[m[0]] = parent[m[1]] = n + a;
        binary[m[1]] = 1;
    }
    off.assign(n + 1, 0);
    point.clear();
    code.clear();
    int64_t path[41];
    int8_t bits[41];
    for (int64_t a = 0; a < n; a++) {
        int len = 0;
        int64_t b = a;
        for (;;) {
            if (len == 40) return false;   // beyond the reference's MAX_CODE_LENGTH
            bits[len] = binary[b];
            path[len] = b;
            len++;
            b = parent[b];
            if (b == 2 * n - 2) break;
        }
        for (int k = 0; k < len; k++) {
            code.push_back(bits[len - 1 - k]);
            point.push_back(k == 0 ? (int32_t)(n - 2) : (int32_t)(path[len - k] - n));
        }
        off[a + 1] = (int32_t)point.size();
    }
    return true;
}

// expTable (word2vec.cu:1569-1573).
void exp_table(std::vector<float> &t) {
    t.assign(kExpTableSize + 1, 0.0f);
    for (int i = 0; i < kExpTableSize; i++) {
        t[i] = std::exp((i / (float)kExpTableSize * 2 - 1) * kMaxExp);
        t[i] = t[i] / (t[i] + 1);
    }
}

// -------------------------------------------------------------- device init

// word2vec's LCG (word2vec.cu:870-873) evaluated at element k directly: the
// state after k + 1 steps from 1, by composing the affine map x -> A x + C.
__device__ __forceinline__ unsigned long long lcg_state(unsigned long long k) {
    unsigned long long ra = 1, rc = 0;                      // identity
    unsigned long long ba = 25214903917ULL, bc = 11ULL;     // one step
    unsigned long long n = k + 1;
    while (n) {
        if (n & 1) {
            rc = ra * bc + rc;
            ra = ra * ba;
        }
        bc = ba * bc + bc;
        ba = ba * ba;
        n >>= 1;
    }
    return ra * 1ULL + rc;
}

// Row r, column c < d gets element r * d + c of word2vec's sequence (rows of d
// columns); rows are stored with stride dp >= d and the padding columns are 0.
__global__ void init_rows_f32(float *rows, uint64_t n, int d, int dp) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = k / (uint64_t)dp, c = k % (uint64_t)dp;
        if (c >= (uint64_t)d) {
            rows[k] = 0.f;
            continue;
        }
        const unsigned long long x = lcg_state(r * (uint64_t)d + c);
        rows[k] = (float)(((double)((x & 0xFFFF) / (float)65536) - 0.5) / (double)d);   // double, as word2vec.cu:872
    }
}

__global__ void init_rows_bf16(__nv_bfloat16 *rows, float *master, uint64_t n, uint64_t n_master, int d) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long x = lcg_state(k);
        const float v = (float)(((double)((x & 0xFFFF) / (float)65536) - 0.5) / (double)d);
        rows[k] = __float2bfloat16_rn(v);
        if (k < n_master) master[k] = v;
    }
}

// ------------------------------------------------------------ plain kernel

// Negative target j (1-based) of pair (centre p, window slot s) of walk wid:
// unigram table draw with word2vec's replacement of index 0 (word2vec.cu:365-368).
__device__ __forceinline__ int32_t negative_target(const SgnsArgs &a, uint32_t p, uint32_t s, uint32_t wid, int j) {
    const uint4 blk = philox((uint32_t)(p * (2 * a.window + 1) + s), wid, a.pass, kNegTag + (uint32_t)((j - 1) >> 2),
                             a.seed_lo, a.seed_hi);
    const uint32_t q = (j - 1) & 3;
    const uint32_t r = q == 0 ? blk.x : q == 1 ? blk.y : q == 2 ? blk.z : blk.w;
    int32_t t = a.table[r % a.table_size];
    if (t == 0) t = (int32_t)((r >> 8) % (a.vocab_size - 1) + 1);
    return t;
}

// Plain SGNS with the pair's targets fetched together: lane j - 1 draws negative
// j, every lane then issues the loads of all 1 + negative target rows and the
// context row before any of them is consumed, so a pair costs one table round
// trip and one row round trip instead of a chain of 1 + 2 * negative.  The
// update order is unchanged: targets are applied in order, and a negative that
// repeats an earlier one of the same pair is re-read from the updated copy.
// Handles negative <= kFastNeg; larger counts use sgns_plain_seq_kernel.
constexpr int kFastNeg = 8;
constexpr uint32_t kSlotChunk = 32;   // window slots whose negatives are drawn together

// Draws the negatives of window slots [cs, ce) of centre p into tb (kFastNeg per
// slot), all lanes at once, so that the pairs of a centre wait on the unigram
// table once instead of once per pair.  The draws are the per-pair draws
// (negative_target), so the result is unchanged.  Slot == window is skipped.
// Slot cs + k, negative j goes to tb[k * stride + j].
__device__ __forceinline__ void draw_negatives(const SgnsArgs &a, uint32_t p, uint32_t wid, uint32_t cs, uint32_t ce,
                                               int neg, int32_t *tb, int stride = kFastNeg) {
    const uint32_t lane = threadIdx.x & 31;
    __syncwarp();
    const uint32_t total = (ce - cs) * (uint32_t)neg;
    for (uint32_t q = lane; q < total; q += 32) {
        const uint32_t k = q / (uint32_t)neg, j = q % (uint32_t)neg;
        const uint32_t s = cs + k;
        if (s == (uint32_t)a.window) continue;
        tb[k * stride + j] = negative_target(a, p, s, wid, (int)j + 1);
    }
    __syncwarp();
}

// Window slots of centre p whose context lies inside the sentence:
// [max(b, w - p), min(2w + 1 - b, n + w - p)), slot w excluded by the caller.
__device__ __forceinline__ void slot_range(uint32_t p, uint32_t n, uint32_t w, uint32_t b, uint32_t &lo,
                                           uint32_t &hi) {
    lo = max(b, w > p ? w - p : 0u);
    hi = min(2 * w + 1 - b, n + w - p);
}

// Pairs ahead whose rows are prefetched into L2 while the current pair runs.
constexpr uint32_t kPrefetchPairs = 2;
// Negative count with its own compile-time instance (word2vec's and DistGER's default).
constexpr int kPlainNeg = 5;

// NEG > 0: the negative count fixed at compile time (a.negative == NEG, vocabulary
// of more than one word); NEG == 0: any count <= kFastNeg read from a.negative.
// FIT > 0: registers capped so that FIT blocks fit on an SM.
template <int VEC, int THREADS, int NEG, int FIT>
__global__ void __launch_bounds__(THREADS, FIT > 0 ? FIT : 1) sgns_plain_kernel(SgnsArgs a, WalkSet ws) {
    constexpr int NS = NEG > 0 ? NEG : kFastNeg;   // negative slots held in registers
    __shared__ int32_t sen_all[THREADS / 32][kMaxSentence];
    __shared__ int32_t tb_all[THREADS / 32][kSlotChunk * kFastNeg];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = threadIdx.x >> 5;
    int32_t *sen = sen_all[warp];
    int32_t *tb = tb_all[warp];
    const int d = 32 * VEC;
    const uint32_t w = (uint32_t)a.window;
    const float alpha = a.alpha;
    const int neg = NEG > 0 ? NEG : (a.vocab_size > 1 ? a.negative : 0);
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
        uint32_t b_next = philox(0, wid, a.pass, kWinTag, a.seed_lo, a.seed_hi).x % w;
        for (uint32_t p = 0; p < n; p++) {
            const int32_t word = sen[p];
            const uint32_t b = b_next;
            float *pos_row = a.syn1 + (size_t)word * d + lane * VEC;
            RowVec<VEC> pos, pos0;
            load_row<VEC>(pos_row, pos);
            pos0 = pos;
            uint32_t s_lo, s_hi;
            slot_range(p, n, w, b, s_lo, s_hi);
            // Slot w lies in [s_lo, s_hi) (s_lo <= w < s_hi since p < n), so the
            // centre has s_hi - s_lo - 1 pairs; likewise the next centre.
            const uint32_t n_pairs_here = s_hi - s_lo - 1;
            uint32_t q_lo = 0, q_hi = 0;
            if (p + 1 < n) {
                b_next = philox(p + 1, wid, a.pass, kWinTag, a.seed_lo, a.seed_hi).x % w;
                slot_range(p + 1, n, w, b_next, q_lo, q_hi);
                if (lane == 0) prefetch_l2(a.syn1 + (size_t)sen[p + 1] * d, (uint32_t)d * 4);
            }
            for (uint32_t cs = s_lo; cs < s_hi; cs += kSlotChunk) {
            const uint32_t ce = min(cs + kSlotChunk, s_hi);
            draw_negatives(a, p, wid, cs, ce, neg, tb);
            for (uint32_t s = cs; s < ce; s++) {
                if (s == w) continue;
                {   // L2 prefetch of the rows of the pair kPrefetchPairs ahead: its
                    // context row (lane 0) and, inside this slot chunk, its negatives'
                    // rows (lanes 1..neg); past this centre, the next centre's context row.
                    const uint32_t kp = s - s_lo - (s > w ? 1u : 0u) + kPrefetchPairs;
                    if (kp < n_pairs_here) {
                        const uint32_t sp = s_lo + kp + (s_lo + kp >= w ? 1u : 0u);
                        if (sp < ce) {
                            if (lane == 0) prefetch_l2(a.syn0 + (size_t)sen[p - w + sp] * d, (uint32_t)d * 4);
                            else if (lane <= (uint32_t)neg)
                                prefetch_l2(a.syn1 + (size_t)tb[(sp - cs) * kFastNeg + lane - 1] * d, (uint32_t)d * 4);
                        }
                    } else if (p + 1 < n && lane == 0) {
                        const uint32_t kq = kp - n_pairs_here;
                        if (kq + 1 < q_hi - q_lo) {
                            const uint32_t sq = q_lo + kq + (q_lo + kq >= w ? 1u : 0u);
                            prefetch_l2(a.syn0 + (size_t)sen[p + 1 - w + sq] * d, (uint32_t)d * 4);
                        }
                    }
                }
                const int64_t c = (int64_t)p - a.window + s;
                const int32_t last = sen[c];
                float *l1p = a.syn0 + (size_t)last * d + lane * VEC;
                int32_t t[NS];
#pragma unroll
                for (int j = 0; j < NS; j++) t[j] = j < neg ? tb[(s - cs) * kFastNeg + j] : -1;
                // Issue every row load of the pair before consuming any.
                RowVec<VEC> l1, e, l2[NS];
                load_row<VEC>(l1p, l1);
#pragma unroll
                for (int j = 0; j < NS; j++)
                    if (j < neg && t[j] != word) load_row<VEC>(a.syn1 + (size_t)t[j] * d + lane * VEC, l2[j]);
#pragma unroll
                for (int i = 0; i < VEC; i++) e.v[i] = 0.f;
                n_pairs++;
                bool repeat = false;
#pragma unroll
                for (int j = 0; j < NS; j++)
#pragma unroll
                    for (int k = j + 1; k < NS; k++) repeat |= k < neg && t[k] == t[j];
                if (!repeat) {
                    // No negative row occurs twice in the pair, so no target's dot
                    // product reads another target's update: all 1 + neg dot products
                    // (same per-lane order and tree as warp_dot) and their gradients
                    // are formed together, one gradient per lane group, then
                    // applied in the sequential order.
                    constexpr int M = pow2_at_least(NS + 1);
                    constexpr int GROUP = 32 / M;   // lanes holding one sum
                    float f[M], g[NS + 1];
                    {
                        float s0 = 0.f;
#pragma unroll
                        for (int i = 0; i < VEC; i++) s0 = fmaf(l1.v[i], pos.v[i], s0);
                        f[0] = s0;
                    }
                    uint32_t live = 0;   // bit j: negative j has a row
#pragma unroll
                    for (int j = 0; j < NS; j++) {
                        float sj = 0.f;
#pragma unroll
                        for (int i = 0; i < VEC; i++) sj = fmaf(l1.v[i], l2[j].v[i], sj);
                        f[j + 1] = sj;
                        if (j < neg && t[j] != word) live |= 1u << j;
                    }
#pragma unroll
                    for (int j = NS + 1; j < M; j++) f[j] = 0.f;
                    const float mine = warp_sums_split<M>(f, lane);
                    const uint32_t jm = lane / GROUP;
                    // Slots without a row (and padding) get no table lookup.
                    float gm = 0.f;
                    if (jm == 0) gm = sg_grad(mine, 1, a.exp_table, alpha);
                    else if (jm <= (uint32_t)NS && ((live >> (jm - 1)) & 1u)) gm = sg_grad(mine, 0, a.exp_table, alpha);
#pragma unroll
                    for (int j = 0; j <= NS; j++) g[j] = __shfl_sync(0xffffffffu, gm, j * GROUP);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g[0], pos.v[i], e.v[i]);
                        pos.v[i] += __fmul_rn(g[0], l1.v[i]);  // rounded product, as the reference's atomicAdd
                    }
#pragma unroll
                    for (int j = 0; j < NS; j++) {
                        if (!((live >> j) & 1u)) continue;
                        RowVec<VEC> upd;
#pragma unroll
                        for (int i = 0; i < VEC; i++) {
                            e.v[i] = fmaf(g[j + 1], l2[j].v[i], e.v[i]);
                            upd.v[i] = __fmul_rn(g[j + 1], l1.v[i]);  // rounded product, never fused
                        }
                        float *l2p = a.syn1 + (size_t)t[j] * d + lane * VEC;
                        if (a.deterministic) {
#pragma unroll
                            for (int i = 0; i < VEC; i++) l2[j].v[i] += upd.v[i];
                            store_row<VEC>(l2p, l2[j]);
                        } else {
                            add_row<VEC>(l2p, upd);
                        }
                    }
                } else {
                {   // positive target: the centre word (kept in registers for this centre)
                    const float g = sg_grad(warp_dot<VEC>(l1, pos), 1, a.exp_table, alpha);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g, pos.v[i], e.v[i]);
                        pos.v[i] += __fmul_rn(g, l1.v[i]);  // rounded product, as the reference's atomicAdd
                    }
                }
#pragma unroll
                for (int j = 0; j < NS; j++) {
                    if (j >= neg || t[j] == word) continue;
                    const float g = sg_grad(warp_dot<VEC>(l1, l2[j]), 0, a.exp_table, alpha);
                    RowVec<VEC> upd;
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g, l2[j].v[i], e.v[i]);
                        upd.v[i] = __fmul_rn(g, l1.v[i]);  // rounded product, never fused
                        l2[j].v[i] += upd.v[i];
                    }
                    float *l2p = a.syn1 + (size_t)t[j] * d + lane * VEC;
                    if (a.deterministic) store_row<VEC>(l2p, l2[j]);
                    else add_row<VEC>(l2p, upd);
                    // A later negative of this pair on the same row sees this update.
#pragma unroll
                    for (int k = j + 1; k < NS; k++)
                        if (t[k] == t[j]) l2[k] = l2[j];
                }
                }
                if (a.deterministic) {
#pragma unroll
                    for (int i = 0; i < VEC; i++) l1.v[i] += e.v[i];
                    store_row<VEC>(l1p, l1);
                } else {
                    add_row<VEC>(l1p, e);
                }
            }
            }
            if (a.deterministic) {
                store_row<VEC>(pos_row, pos);
            } else {
#pragma unroll
                for (int i = 0; i < VEC; i++) pos.v[i] -= pos0.v[i];
                add_row<VEC>(pos_row, pos);
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_words);
        atomicAdd(&a.stats[1], n_trained);
        atomicAdd(&a.stats[2], n_pairs);
    }
}

// ------------------------------------------ plain rule, rows staged ahead

// Hogwild form of the plain rule whose row loads overlap the previous pairs'
// arithmetic: while pair m computes, the rows of pair m + S - 1 (its context row
// and its negatives' rows) are copied into this warp's shared memory with
// cp.async, so a pair waits on a copy issued S - 1 pairs earlier instead of a
// DRAM round trip.  Each lane copies, and later reads, only its own columns.
// A copy made before this warp's last updates of the same row would miss them;
// the kernel restores them where they matter:
//  * context rows: a context word used by one of the previous S pairs is read
//    from that pair's updated row (kept in shared memory), so a context row sees
//    every update of this warp, as in sgns_plain_kernel;
//  * the centre's output row is loaded when the centre starts (after every
//    earlier update) and kept in registers, as in sgns_plain_kernel;
//  * a negative's output row copied before one of the previous S pairs (or a
//    finished centre) updated it misses that update: staleness of at most S
//    pairs, of the kind other warps' concurrent updates cause in any Hogwild run.
// Draws, pairs, sums, gradients and the update order of each pair are
// sgns_plain_kernel's.  The launcher uses it only without `deterministic`, for
// sentences of at most kPipeSentence tokens, window <= kPipeMaxWindow and
// negative <= kFastNeg.
constexpr uint32_t kPipeSentence = 64;
constexpr int kPipeMaxWindow = 15;

template <int VEC>
__device__ __forceinline__ void copy_row_async(float *dst, const float *src) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst);
    const size_t ga = __cvta_generic_to_global(src);
    if constexpr (VEC % 4 == 0) {
#pragma unroll
        for (int i = 0; i < VEC; i += 4)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa + 4 * i), "l"(ga + 4 * i) : "memory");
    } else if constexpr (VEC == 2) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(ga) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(ga) : "memory");
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// This lane's columns of a row held in shared memory.
template <int VEC>
__device__ __forceinline__ void lds_row(const float *p, RowVec<VEC> &r) {
    if constexpr (VEC % 4 == 0) {
#pragma unroll
        for (int i = 0; i < VEC; i += 4) {
            const float4 t = *reinterpret_cast<const float4 *>(p + i);
            r.v[i] = t.x; r.v[i + 1] = t.y; r.v[i + 2] = t.z; r.v[i + 3] = t.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < VEC; i++) r.v[i] = p[i];
    }
}

template <int VEC>
__device__ __forceinline__ void sts_row(float *p, const RowVec<VEC> &r) {
    if constexpr (VEC % 4 == 0) {
#pragma unroll
        for (int i = 0; i < VEC; i += 4)
            *reinterpret_cast<float4 *>(p + i) = make_float4(r.v[i], r.v[i + 1], r.v[i + 2], r.v[i + 3]);
    } else {
#pragma unroll
        for (int i = 0; i < VEC; i++) p[i] = r.v[i];
    }
}

template <int VEC, int NS, int S>
struct alignas(16) PipeWarp {
    float stage[S][1 + NS][32 * VEC];             // rows of S pairs: context, negatives 0..NS-1
    float hist[S][32 * VEC];                      // updated context rows of the last S pairs
    int32_t sen[kPipeSentence];
    int32_t tb[S][(2 * kPipeMaxWindow + 1) * NS];  // negatives of S centres, ring by centre
    // Per slot of those centres: bit j set when negative j trains (it exists and
    // is not the centre's word); bit 15 when a negative repeats within the slot.
    uint16_t fl[S][2 * kPipeMaxWindow + 1];
    uint16_t lohi[kPipeSentence];                 // slot range of each centre: lo | hi << 8
};

// BF16 rows in a staging slot: this lane's VEC values at 2 bytes (the slot's
// first 2 * VEC bytes).
template <int VEC>
__device__ __forceinline__ void copy_half_row_async(float *dst, const __nv_bfloat16 *src) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst);
    const size_t ga = __cvta_generic_to_global(src);
    if constexpr (VEC == 8) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(ga) : "memory");
    } else if constexpr (VEC == 4) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(ga) : "memory");
    } else {
        static_assert(VEC == 2, "BF16 staging supports 2, 4 or 8 values per lane");
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(ga) : "memory");
    }
}

template <int VEC>
__device__ __forceinline__ void lds_half_row(const float *p, RowVec<VEC> &r) {
    const uint32_t *q = reinterpret_cast<const uint32_t *>(p);
#pragma unroll
    for (int i = 0; i < VEC / 2; i++) {
        const uint32_t t = q[i];
        r.v[2 * i] = __uint_as_float(t << 16);
        r.v[2 * i + 1] = __uint_as_float(t & 0xFFFF0000u);
    }
}

// BF = false: FP32 rows (syn0, syn1), updates by vector atomics (DG_SGNS_PLAIN).
// BF = true: the BF16 plain mode's rows and writes (BfRows: FP32 masters by
// atomics, BF16 rows stored as the warp's updated copy with stochastic
// rounding, the same noise keys as sgns_plain_bf16_kernel).  A BF16 row is
// written back as (staged copy + update), so a concurrent update made since
// the copy is lost; the launcher stages BF16 rows only where such collisions
// are rare (dg_sgns::bf_staged).
template <int VEC, int THREADS, int NEG, int S, int FIT, bool BF>
__global__ void __launch_bounds__(THREADS, FIT > 0 ? FIT : 1) sgns_plain_pipe_kernel(SgnsArgs a, WalkSet ws) {
    constexpr int NS = NEG > 0 ? NEG : kFastNeg;
    constexpr int D = 32 * VEC;
    constexpr int M = pow2_at_least(NS + 1);
    constexpr int GROUP = 32 / M;
    __shared__ PipeWarp<VEC, NS, S> sm_all[THREADS / 32];
    PipeWarp<VEC, NS, S> &sm = sm_all[threadIdx.x >> 5];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t w = (uint32_t)a.window;
    const float alpha = a.alpha;
    const int neg = NEG > 0 ? NEG : (a.vocab_size > 1 ? a.negative : 0);
    const BfRows<VEC> in{a.in_bf, a.in_master, a.n_master, D};
    const BfRows<VEC> out{a.out_bf, a.out_master, a.n_master, D};
    const uint32_t key = a.seed_lo ^ bf_mix(a.pass * 0x9E3779B9u + 0x2F6B3A91u);
    unsigned long long n_words = 0, n_trained = 0, n_pairs = 0;
    int32_t hw[S];   // context words of this warp's last S pairs, newest first
#pragma unroll
    for (int k = 0; k < S; k++) hw[k] = -1;
    uint32_t mm = 0;  // pairs trained by this warp (ring position of hist)
    // Copy of row `id` of the input (context) or output table into a staging slot.
    auto copy_in = [&](float *dst, int32_t id, bool input) {
        if constexpr (!BF) {
            copy_row_async<VEC>(dst, (input ? a.syn0 : a.syn1) + (size_t)id * D + lane * VEC);
        } else {
            if ((uint32_t)id < a.n_master)
                copy_row_async<VEC>(dst, (input ? a.in_master : a.out_master) + (size_t)id * D + lane * VEC);
            else
                copy_half_row_async<VEC>(dst, (input ? a.in_bf : a.out_bf) + (size_t)id * D + lane * VEC);
        }
    };
    // A staged row of `id`; f32 = the slot holds FP32 values whatever the row's storage.
    auto read_slot = [&](const float *src, int32_t id, bool f32, RowVec<VEC> &r) {
        if (!BF || f32 || (uint32_t)id < a.n_master) lds_row<VEC>(src, r);
        else lds_half_row<VEC>(src, r);
    };
    for (;;) {
        uint32_t walk = 0;
        if (lane == 0) walk = atomicAdd(a.queue, 1u);
        walk = __shfl_sync(0xffffffffu, walk, 0);
        if (walk >= ws.n_walks) break;
        const uint32_t wid = ws.ids ? ws.ids[walk] : walk + ws.id_base;
        uint32_t words;
        const uint32_t n = warp_sentence<kPipeSentence>(ws, walk, a, sm.sen, words);
        n_words += words;
        n_trained += n;
        if (n < 2) continue;   // a one-token sentence has no pairs
        for (uint32_t q = lane; q < n; q += 32) {
            const uint32_t b = philox(q, wid, a.pass, kWinTag, a.seed_lo, a.seed_hi).x % w;
            uint32_t lo, hi;
            slot_range(q, n, w, b, lo, hi);
            sm.lohi[q] = (uint16_t)(lo | (hi << 8));
        }
        __syncwarp();
        // With n >= 2 every centre has a pair, and slot w lies inside its range.
        auto first_slot = [&](uint32_t q) {
            const uint32_t s0 = sm.lohi[q] & 0xFFu;
            return s0 == w ? s0 + 1 : s0;
        };
        auto advance = [&](uint32_t &q, uint32_t &s) {   // next pair; true when centre q ended
            s++;
            if (s == w) s++;
            if (s < (uint32_t)(sm.lohi[q] >> 8)) return false;
            q++;
            if (q < n) s = first_slot(q);
            return true;
        };
        auto enter = [&](uint32_t q) {   // the copies reach centre q: draw its negatives
            const uint32_t lo = sm.lohi[q] & 0xFFu, hi = sm.lohi[q] >> 8;
            draw_negatives(a, q, wid, lo, hi, neg, sm.tb[q % S], NS);
            {   // each slot's flags, once per centre instead of at every pair
                const int32_t cw = sm.sen[q];
                for (uint32_t k = lane; k < hi - lo; k += 32) {
                    const int32_t *tk = sm.tb[q % S] + k * NS;
                    uint32_t f = 0;
#pragma unroll
                    for (int j = 0; j < NS; j++) {
                        if (j >= neg) break;
                        const int32_t tj = tk[j];
                        if (tj != cw) f |= 1u << j;
#pragma unroll
                        for (int i = 0; i < j; i++)
                            if (tk[i] == tj) f |= 0x8000u;
                    }
                    sm.fl[q % S][k] = (uint16_t)f;   // slot w (no pair) gets an unused value
                }
                __syncwarp();
            }
            if (lane == 0) {
                const int32_t cw = sm.sen[q];
                if (!BF) prefetch_l2(a.syn1 + (size_t)cw * D, (uint32_t)D * 4);
                else if ((uint32_t)cw < a.n_master) prefetch_l2(a.out_master + (size_t)cw * D, (uint32_t)D * 4);
                else prefetch_l2(a.out_bf + (size_t)cw * D, (uint32_t)D * 2);
            }
        };
        auto issue = [&](uint32_t q, uint32_t s, uint32_t st) {
            copy_in(&sm.stage[st][0][lane * VEC], sm.sen[q - w + s], true);
            const int32_t *tq = sm.tb[q % S] + (s - (sm.lohi[q] & 0xFFu)) * NS;
#pragma unroll
            for (int j = 0; j < NS; j++)
                if (j < neg) copy_in(&sm.stage[st][1 + j][lane * VEC], tq[j], false);
        };
        // The centre's output row, kept in registers while the centre trains.
        auto load_pos = [&](int32_t cw, RowVec<VEC> &r) {
            if constexpr (BF) out.load(cw, lane, r);
            else load_row<VEC>(a.syn1 + (size_t)cw * D + lane * VEC, r);
        };
        auto centre_noise = [&](uint32_t q) {   // sgns_plain_bf16_kernel's per-centre noise base
            return bf_mix(key ^ bf_mix(wid * 0x01000193u + q * 0x2545F491u) ^ lane * 0x85EBCA6Bu);
        };
        uint32_t pp = 0, sp = first_slot(0);   // next pair to copy
        enter(0);
#pragma unroll
        for (int i = 0; i < S - 1; i++) {
            if (pp < n) {
                issue(pp, sp, (uint32_t)i);
                if (advance(pp, sp) && pp < n) enter(pp);
            }
            cp_async_commit();
        }
        uint32_t p = 0, s = first_slot(0);     // pair to train
        int32_t word = sm.sen[0];
        uint32_t base = BF ? centre_noise(0) : 0u;
        RowVec<VEC> pos, pos0;
        load_pos(word, pos);
        pos0 = pos;
        for (uint32_t m = 0; p < n; m++) {
            if (pp < n) {
                issue(pp, sp, (m + S - 1) % S);
                if (advance(pp, sp) && pp < n) enter(pp);
            }
            cp_async_commit();
            cp_async_wait<S - 1>();   // this lane's copies of pair m have landed
            const uint32_t st = m % S;
            const int32_t last = sm.sen[p - w + s];
            RowVec<VEC> l1, e;
            read_slot(&sm.stage[st][0][lane * VEC], last, false, l1);
#pragma unroll
            for (int k = S - 1; k >= 0; k--)   // newest match last: it wins
                if (hw[k] == last) lds_row<VEC>(&sm.hist[(mm + S - 1 - k) % S][lane * VEC], l1);
            const uint32_t ks = s - (sm.lohi[p] & 0xFFu);
            const int32_t *tq = sm.tb[p % S] + ks * NS;
            int32_t t[NS];
#pragma unroll
            for (int j = 0; j < NS; j++) t[j] = j < neg ? tq[j] : -1;
#pragma unroll
            for (int i = 0; i < VEC; i++) e.v[i] = 0.f;
            n_pairs++;
            const uint32_t flags = sm.fl[p % S][ks];
            const bool repeat = (flags & 0x8000u) != 0;
            // Writes negative j's row: an atomic delta (FP32 rows, masters) or the
            // warp's updated copy (BF16 rows).
            auto write_neg = [&](int j, const RowVec<VEC> &upd, const RowVec<VEC> &value) {
                if constexpr (BF) out.update(t[j], lane, upd, value, base + (uint32_t)t[j] * 0x27D4EB2Fu + s * 16u + (uint32_t)j);
                else add_row<VEC>(a.syn1 + (size_t)t[j] * D + lane * VEC, upd);
            };
            if (!repeat) {   // as in sgns_plain_kernel: all sums and gradients at once
                float f[M], g[NS + 1];
                {
                    float s0 = 0.f;
#pragma unroll
                    for (int i = 0; i < VEC; i++) s0 = fmaf(l1.v[i], pos.v[i], s0);
                    f[0] = s0;
                }
                const uint32_t live = flags & 0xFFu;
                // BF16 rows: decoded once and kept for the update phase (FP32 rows
                // are read from shared memory again instead, to save registers).
                RowVec<VEC> kept[BF ? NS : 1];
#pragma unroll
                for (int j = 0; j < NS; j++) {
                    float sj = 0.f;
                    if (j < neg) {
                        RowVec<VEC> r;
                        read_slot(&sm.stage[st][1 + j][lane * VEC], t[j], false, r);
#pragma unroll
                        for (int i = 0; i < VEC; i++) sj = fmaf(l1.v[i], r.v[i], sj);
                        if constexpr (BF) kept[j] = r;
                    }
                    f[j + 1] = sj;
                }
#pragma unroll
                for (int j = NS + 1; j < M; j++) f[j] = 0.f;
                const float mine = warp_sums_split<M>(f, lane);
                const uint32_t jm = lane / GROUP;
                float gm = 0.f;
                if (jm == 0) gm = sg_grad(mine, 1, a.exp_table, alpha);
                else if (jm <= (uint32_t)NS && ((live >> (jm - 1)) & 1u)) gm = sg_grad(mine, 0, a.exp_table, alpha);
#pragma unroll
                for (int j = 0; j <= NS; j++) g[j] = __shfl_sync(0xffffffffu, gm, j * GROUP);
#pragma unroll
                for (int i = 0; i < VEC; i++) {
                    e.v[i] = fmaf(g[0], pos.v[i], e.v[i]);
                    pos.v[i] += __fmul_rn(g[0], l1.v[i]);  // rounded product, as the reference's atomicAdd
                }
#pragma unroll
                for (int j = 0; j < NS; j++) {
                    if (!((live >> j) & 1u)) continue;
                    RowVec<VEC> r, upd;
                    if constexpr (BF) r = kept[j];
                    else read_slot(&sm.stage[st][1 + j][lane * VEC], t[j], false, r);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g[j + 1], r.v[i], e.v[i]);
                        upd.v[i] = __fmul_rn(g[j + 1], l1.v[i]);  // rounded product, never fused
                        if (BF) r.v[i] += upd.v[i];
                    }
                    write_neg(j, upd, r);
                }
            } else {   // a negative repeats: one target after the other
                {
                    const float g = sg_grad(warp_dot<VEC>(l1, pos), 1, a.exp_table, alpha);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g, pos.v[i], e.v[i]);
                        pos.v[i] += __fmul_rn(g, l1.v[i]);  // rounded product, as the reference's atomicAdd
                    }
                }
                uint32_t f32 = 0;   // bit k: slot k was rewritten with FP32 values
#pragma unroll
                for (int j = 0; j < NS; j++) {
                    if (j >= neg || t[j] == word) continue;
                    RowVec<VEC> r, upd;
                    read_slot(&sm.stage[st][1 + j][lane * VEC], t[j], (f32 >> j) & 1u, r);
                    const float g = sg_grad(warp_dot<VEC>(l1, r), 0, a.exp_table, alpha);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g, r.v[i], e.v[i]);
                        upd.v[i] = __fmul_rn(g, l1.v[i]);
                        r.v[i] += upd.v[i];
                    }
                    write_neg(j, upd, r);
                    // A later negative of this pair on the same row sees this update.
#pragma unroll
                    for (int k = j + 1; k < NS; k++)
                        if (t[k] == t[j]) {
                            sts_row<VEC>(&sm.stage[st][1 + k][lane * VEC], r);
                            f32 |= 1u << k;
                        }
                }
            }
            if constexpr (BF) {
                RowVec<VEC> v1;
#pragma unroll
                for (int i = 0; i < VEC; i++) v1.v[i] = l1.v[i] + e.v[i];
                in.update(last, lane, e, v1, base + (uint32_t)last * 0x165667B1u + s * 16u + 15u);
            } else {
                add_row<VEC>(a.syn0 + (size_t)last * D + lane * VEC, e);
            }
#pragma unroll
            for (int i = 0; i < VEC; i++) l1.v[i] += e.v[i];
            sts_row<VEC>(&sm.hist[mm % S][lane * VEC], l1);
#pragma unroll
            for (int k = S - 1; k > 0; k--) hw[k] = hw[k - 1];
            hw[0] = last;
            mm++;
            if (advance(p, s)) {   // centre done: its output row's update, then the next centre's row
                RowVec<VEC> delta;
#pragma unroll
                for (int i = 0; i < VEC; i++) delta.v[i] = pos.v[i] - pos0.v[i];
                if constexpr (BF) out.update(word, lane, delta, pos, base + (uint32_t)word * 0xD3A2646Cu + 0x5BD1E995u);
                else add_row<VEC>(a.syn1 + (size_t)word * D + lane * VEC, delta);
                if (p < n) {
                    word = sm.sen[p];
                    if (BF) base = centre_noise(p);
                    load_pos(word, pos);
                    pos0 = pos;
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

// The plain kernel's schedule and update rule (word2vec.cu:305-399) on BF16
// rows: the same pairs, draws and update order as sgns_plain_kernel, arithmetic
// in FP32; each row write rounds stochastically with noise keyed by
// (row, walk, centre, slot), so a deterministic run is reproducible.
// NEG as in sgns_plain_kernel.
template <int VEC, int THREADS, int NEG, int FIT>
__global__ void __launch_bounds__(THREADS, FIT > 0 ? FIT : 1) sgns_plain_bf16_kernel(SgnsArgs a, WalkSet ws) {
    constexpr int NS = NEG > 0 ? NEG : kFastNeg;
    __shared__ int32_t sen_all[THREADS / 32][kMaxSentence];
    __shared__ int32_t tb_all[THREADS / 32][kSlotChunk * kFastNeg];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = threadIdx.x >> 5;
    int32_t *sen = sen_all[warp];
    int32_t *tb = tb_all[warp];
    const int d = 32 * VEC;
    const float alpha = a.alpha;
    const int neg = NEG > 0 ? NEG : (a.vocab_size > 1 ? a.negative : 0);
    const BfRows<VEC> in{a.in_bf, a.in_master, a.n_master, d};
    const BfRows<VEC> out{a.out_bf, a.out_master, a.n_master, d};
    const uint32_t key = a.seed_lo ^ bf_mix(a.pass * 0x9E3779B9u + 0x2F6B3A91u);
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
            const uint32_t b = philox(p, wid, a.pass, kWinTag, a.seed_lo, a.seed_hi).x % (uint32_t)a.window;
            // Row noise: distinct per (walk, centre, slot, row, lane).
            const uint32_t base = bf_mix(key ^ bf_mix(wid * 0x01000193u + p * 0x2545F491u) ^ lane * 0x85EBCA6Bu);
            RowVec<VEC> pos, pos0;
            out.load(word, lane, pos);
            pos0 = pos;
            uint32_t s_lo, s_hi;
            slot_range(p, n, (uint32_t)a.window, b, s_lo, s_hi);
            for (uint32_t cs = s_lo; cs < s_hi; cs += kSlotChunk) {
            const uint32_t ce = min(cs + kSlotChunk, s_hi);
            draw_negatives(a, p, wid, cs, ce, neg, tb);
            for (uint32_t s = cs; s < ce; s++) {
                if (s == (uint32_t)a.window) continue;
                const int64_t c = (int64_t)p - a.window + s;
                const int32_t last = sen[c];
                int32_t t[NS];
#pragma unroll
                for (int j = 0; j < NS; j++) t[j] = j < neg ? tb[(s - cs) * kFastNeg + j] : -1;
                RowVec<VEC> l1, e, l2[NS];
                in.load(last, lane, l1);
#pragma unroll
                for (int j = 0; j < NS; j++)
                    if (j < neg && t[j] != word) out.load(t[j], lane, l2[j]);
#pragma unroll
                for (int i = 0; i < VEC; i++) e.v[i] = 0.f;
                n_pairs++;
                bool repeat = false;
#pragma unroll
                for (int j = 0; j < NS; j++)
#pragma unroll
                    for (int k = j + 1; k < NS; k++) repeat |= k < neg && t[k] == t[j];
                if (!repeat) {   // all sums and gradients at once, as in sgns_plain_kernel
                    constexpr int M = pow2_at_least(NS + 1);
                    constexpr int GROUP = 32 / M;
                    float f[M], g[NS + 1];
                    {
                        float s0 = 0.f;
#pragma unroll
                        for (int i = 0; i < VEC; i++) s0 = fmaf(l1.v[i], pos.v[i], s0);
                        f[0] = s0;
                    }
                    uint32_t live = 0;
#pragma unroll
                    for (int j = 0; j < NS; j++) {
                        float sj = 0.f;
#pragma unroll
                        for (int i = 0; i < VEC; i++) sj = fmaf(l1.v[i], l2[j].v[i], sj);
                        f[j + 1] = sj;
                        if (j < neg && t[j] != word) live |= 1u << j;
                    }
#pragma unroll
                    for (int j = NS + 1; j < M; j++) f[j] = 0.f;
                    const float mine = warp_sums_split<M>(f, lane);
                    const uint32_t jm = lane / GROUP;
                    float gm = 0.f;
                    if (jm == 0) gm = sg_grad(mine, 1, a.exp_table, alpha);
                    else if (jm <= (uint32_t)NS && ((live >> (jm - 1)) & 1u)) gm = sg_grad(mine, 0, a.exp_table, alpha);
#pragma unroll
                    for (int j = 0; j <= NS; j++) g[j] = __shfl_sync(0xffffffffu, gm, j * GROUP);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g[0], pos.v[i], e.v[i]);
                        pos.v[i] += __fmul_rn(g[0], l1.v[i]);  // rounded product, as the reference's atomicAdd
                    }
#pragma unroll
                    for (int j = 0; j < NS; j++) {
                        if (!((live >> j) & 1u)) continue;
                        RowVec<VEC> upd;
#pragma unroll
                        for (int i = 0; i < VEC; i++) {
                            e.v[i] = fmaf(g[j + 1], l2[j].v[i], e.v[i]);
                            upd.v[i] = __fmul_rn(g[j + 1], l1.v[i]);
                            l2[j].v[i] += upd.v[i];
                        }
                        const uint32_t salt = base + (uint32_t)t[j] * 0x27D4EB2Fu + s * 16u + (uint32_t)j;
                        if (a.deterministic) out.put(t[j], lane, l2[j], salt);
                        else out.update(t[j], lane, upd, l2[j], salt);
                    }
                } else {
                {
                    const float g = sg_grad(warp_dot<VEC>(l1, pos), 1, a.exp_table, alpha);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g, pos.v[i], e.v[i]);
                        pos.v[i] += __fmul_rn(g, l1.v[i]);  // rounded product, as the reference's atomicAdd
                    }
                }
#pragma unroll
                for (int j = 0; j < NS; j++) {
                    if (j >= neg || t[j] == word) continue;
                    const float g = sg_grad(warp_dot<VEC>(l1, l2[j]), 0, a.exp_table, alpha);
                    RowVec<VEC> upd;
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g, l2[j].v[i], e.v[i]);
                        upd.v[i] = __fmul_rn(g, l1.v[i]);
                        l2[j].v[i] += upd.v[i];
                    }
                    const uint32_t salt = base + (uint32_t)t[j] * 0x27D4EB2Fu + s * 16u + (uint32_t)j;
                    if (a.deterministic) out.put(t[j], lane, l2[j], salt);
                    else out.update(t[j], lane, upd, l2[j], salt);
#pragma unroll
                    for (int k = j + 1; k < NS; k++)
                        if (t[k] == t[j]) l2[k] = l2[j];
                }
                }
                const uint32_t salt1 = base + (uint32_t)last * 0x165667B1u + s * 16u + 15u;
#pragma unroll
                for (int i = 0; i < VEC; i++) l1.v[i] += e.v[i];
                if (a.deterministic) in.put(last, lane, l1, salt1);
                else in.update(last, lane, e, l1, salt1);
            }
            }
            const uint32_t salt0 = base + (uint32_t)word * 0xD3A2646Cu + 0x5BD1E995u;
            if (a.deterministic) {
                out.put(word, lane, pos, salt0);
            } else {
                RowVec<VEC> delta;
#pragma unroll
                for (int i = 0; i < VEC; i++) delta.v[i] = pos.v[i] - pos0.v[i];
                out.update(word, lane, delta, pos, salt0);
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_words);
        atomicAdd(&a.stats[1], n_trained);
        atomicAdd(&a.stats[2], n_pairs);
    }
}

// One target at a time (any negative count up to 64).
template <int VEC>
__global__ void __launch_bounds__(kPlainThreads) sgns_plain_seq_kernel(SgnsArgs a, WalkSet ws) {
    __shared__ int32_t sen_all[kPlainThreads / 32][kMaxSentence];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = threadIdx.x >> 5;
    int32_t *sen = sen_all[warp];
    const int d = 32 * VEC;
    const float alpha = a.alpha;
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
            const uint32_t b = philox(p, wid, a.pass, kWinTag, a.seed_lo, a.seed_hi).x % (uint32_t)a.window;
            float *pos_row = a.syn1 + (size_t)word * d + lane * VEC;
            RowVec<VEC> pos, pos0;
            load_row<VEC>(pos_row, pos);
            pos0 = pos;
            for (uint32_t s = b; s < (uint32_t)(2 * a.window + 1) - b; s++) {
                if (s == (uint32_t)a.window) continue;
                const int64_t c = (int64_t)p - a.window + s;
                if (c < 0 || c >= (int64_t)n) continue;
                const int32_t last = sen[c];
                float *l1p = a.syn0 + (size_t)last * d + lane * VEC;
                RowVec<VEC> l1, e;
                load_row<VEC>(l1p, l1);
#pragma unroll
                for (int i = 0; i < VEC; i++) e.v[i] = 0.f;
                n_pairs++;
                // Positive target: the centre word (row kept in registers for this centre).
                {
                    const float g = sg_grad(warp_dot<VEC>(l1, pos), 1, a.exp_table, alpha);
#pragma unroll
                    for (int i = 0; i < VEC; i++) {
                        e.v[i] = fmaf(g, pos.v[i], e.v[i]);
                        pos.v[i] += __fmul_rn(g, l1.v[i]);  // rounded product, as the reference's atomicAdd
                    }
                }
                if (a.vocab_size > 1) {
                    uint4 blk = make_uint4(0, 0, 0, 0);
                    for (int j = 1; j <= a.negative; j++) {
                        if (((j - 1) & 3) == 0)
                            blk = philox(p * (2 * a.window + 1) + s, wid, a.pass, kNegTag + (uint32_t)((j - 1) >> 2),
                                         a.seed_lo, a.seed_hi);
                        const uint32_t q = (j - 1) & 3;
                        const uint32_t r = q == 0 ? blk.x : q == 1 ? blk.y : q == 2 ? blk.z : blk.w;
                        int32_t target = a.table[r % a.table_size];
                        if (target == 0) target = (int32_t)((r >> 8) % (a.vocab_size - 1) + 1);  // word2vec.cu:367
                        if (target == word) continue;
                        float *l2p = a.syn1 + (size_t)target * d + lane * VEC;
                        RowVec<VEC> l2, upd;
                        load_row<VEC>(l2p, l2);
                        const float g = sg_grad(warp_dot<VEC>(l1, l2), 0, a.exp_table, alpha);
#pragma unroll
                        for (int i = 0; i < VEC; i++) {
                            e.v[i] = fmaf(g, l2.v[i], e.v[i]);
                            upd.v[i] = __fmul_rn(g, l1.v[i]);  // rounded product, never fused
                        }
                        if (a.deterministic) {
#pragma unroll
                            for (int i = 0; i < VEC; i++) l2.v[i] += upd.v[i];
                            store_row<VEC>(l2p, l2);
                        } else {
                            add_row<VEC>(l2p, upd);
                        }
                    }
                }
                if (a.deterministic) {
#pragma unroll
                    for (int i = 0; i < VEC; i++) l1.v[i] += e.v[i];
                    store_row<VEC>(l1p, l1);
                } else {
                    add_row<VEC>(l1p, e);
                }
            }
            if (a.deterministic) {
                store_row<VEC>(pos_row, pos);
            } else {
#pragma unroll
                for (int i = 0; i < VEC; i++) pos.v[i] -= pos0.v[i];
                add_row<VEC>(pos_row, pos);
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_words);
        atomicAdd(&a.stats[1], n_trained);
        atomicAdd(&a.stats[2], n_pairs);
    }
}

// ------------------------------------------------------- adjoint-mode pairs
// The (context, centre) pairs the plain trainer forms in the same pass -- same
// sentence (vocabulary lookup + subsampling draw), same window shrink b, contexts
// at distance 1 .. window - b (word2vec.cu:328-340) -- laid out in walk order,
// centre order, then left-to-right context order.  Counted first, written at
// the scanned offsets second.
constexpr int kPairThreads = 256;

__device__ __forceinline__ uint32_t pair_span(uint32_t p, uint32_t wid, const SgnsArgs &a) {
    return (uint32_t)a.window - philox(p, wid, a.pass, kWinTag, a.seed_lo, a.seed_hi).x % (uint32_t)a.window;
}

__global__ void __launch_bounds__(kPairThreads) adj_pair_count(SgnsArgs a, WalkSet ws, uint32_t *count) {
    __shared__ int32_t sen_all[kPairThreads / 32][kMaxSentence];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t *sen = sen_all[warp];
    unsigned long long n_words = 0, n_trained = 0;
    for (uint32_t walk = blockIdx.x * (kPairThreads / 32) + warp; walk < ws.n_walks;
         walk += gridDim.x * (kPairThreads / 32)) {
        const uint32_t wid = ws.ids ? ws.ids[walk] : walk + ws.id_base;
        uint32_t words;
        const uint32_t n = warp_sentence(ws, walk, a, sen, words);
        n_words += words;
        n_trained += n;
        uint32_t c = 0;
        for (uint32_t p = lane; p < n; p += 32) {
            const uint32_t span = pair_span(p, wid, a);
            c += min(p, span) + min(n - 1 - p, span);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) count[walk] = c;
        __syncwarp();
    }
    if (lane == 0) {
        atomicAdd(&a.stats[0], n_words);
        atomicAdd(&a.stats[1], n_trained);
    }
}

__global__ void __launch_bounds__(kPairThreads) adj_pair_fill(SgnsArgs a, WalkSet ws, const uint64_t *offs,
                                                              uint32_t *inputs, uint32_t *outputs) {
    __shared__ int32_t sen_all[kPairThreads / 32][kMaxSentence];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t *sen = sen_all[warp];
    for (uint32_t walk = blockIdx.x * (kPairThreads / 32) + warp; walk < ws.n_walks;
         walk += gridDim.x * (kPairThreads / 32)) {
        const uint32_t wid = ws.ids ? ws.ids[walk] : walk + ws.id_base;
        uint32_t words;
        const uint32_t n = warp_sentence(ws, walk, a, sen, words);
        uint64_t base = offs[walk];
        for (uint32_t p0 = 0; p0 < n; p0 += 32) {
            const uint32_t p = p0 + lane;
            uint32_t lo = 0, hi = 0, cnt = 0;
            if (p < n) {
                const uint32_t span = pair_span(p, wid, a);
                lo = p - min(p, span);
                hi = p + min(n - 1 - p, span);
                cnt = hi - lo;
            }
            uint32_t incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if ((int)lane >= o) incl += t;
            }
            if (p < n) {
                uint64_t q = base + incl - cnt;
                for (uint32_t c = lo; c <= hi; c++) {
                    if (c == p) continue;
                    inputs[q] = (uint32_t)sen[c];
                    outputs[q] = (uint32_t)sen[p];
                    q++;
                }
            }
            base += __shfl_sync(0xffffffffu, incl, 31);
        }
        __syncwarp();
    }
}

int adjoint_pairs(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws, uint64_t &n_pairs) {
    n_pairs = 0;
    if (ws.n_walks == 0) return DG_OK;
    const unsigned blocks = (unsigned)std::min<uint64_t>((ws.n_walks + kPairThreads / 32 - 1) / (kPairThreads / 32),
                                                         (uint64_t)dg::sm_count(s->device) * 8);
    dg::DevArray<uint32_t> count;
    DG_CUDA(count.alloc(ws.n_walks));
    if (s->adj_offs.n < (size_t)ws.n_walks + 1) DG_CUDA(s->adj_offs.alloc((size_t)ws.n_walks + 1));
    adj_pair_count<<<blocks, kPairThreads, 0, s->stream>>>(a, ws, count.p); dg::note_launch();
    DG_CUDA(cudaGetLastError());
    int rc = dg::exclusive_scan_u32_to_u64(count.p, s->adj_offs.p, ws.n_walks, s->stream);
    if (rc) return rc;
    DG_CUDA(cudaMemcpyAsync(&n_pairs, s->adj_offs.p + ws.n_walks, 8, cudaMemcpyDeviceToHost, s->stream));
    DG_CUDA(cudaStreamSynchronize(s->stream));
    if (s->adj_pin.n < n_pairs) {
        DG_CUDA(s->adj_pin.alloc(n_pairs + n_pairs / 8));
        DG_CUDA(s->adj_pout.alloc(n_pairs + n_pairs / 8));
    }
    if (n_pairs) {
        adj_pair_fill<<<blocks, kPairThreads, 0, s->stream>>>(a, ws, s->adj_offs.p, s->adj_pin.p, s->adj_pout.p);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
    }
    return DG_OK;
}

// Staged BF16 rows (sgns_plain_pipe_kernel<..., true>) are written back as the
// warp's (copy + update), so an update another warp made to the row since the
// copy is lost.  They are used only when the hottest BF16 row (vocabulary id
// n_master; the vocabulary is sorted by count) is expected to be held by at
// most kBfStagedHolders pairs in flight at once: 24 resident warps per SM, 2
// pairs each, holding it as one of `negative` draws (unigram^0.75 share) or as
// a context or centre token (twice its token share).  The YouTube-shaped
// vocabulary gives 0.10; a 10,000-word table with 1,000 FP32 masters gives 8.
constexpr double kBfStagedHolders = 0.5;

bool bf_staging_safe(const std::vector<uint32_t> &cn, uint32_t n_master, int negative, int sms) {
    if (n_master >= cn.size()) return true;   // every row an FP32 master (atomic updates)
    double pow_sum = 0.0, tok_sum = 0.0;
    for (uint32_t c : cn) {
        pow_sum += std::pow((double)c, 0.75);
        tok_sum += c;
    }
    if (!(pow_sum > 0) || !(tok_sum > 0)) return false;
    const double c = cn[n_master];
    const double holders = (double)sms * 24.0 * 2.0 * (negative * std::pow(c, 0.75) / pow_sum + 2.0 * c / tok_sum);
    return holders <= kBfStagedHolders;
}

// An explicit worker count (warps) lowers the resident grid, never raises it.
static int plain_blocks(const dg_sgns *s, int resident, int threads) {
    if (s->p.workers == 0) return resident;
    const int want = (int)((s->p.workers + threads / 32 - 1) / (threads / 32));
    return std::max(1, std::min(resident, want));
}

// One launch of the fast plain kernel in launch shape I (threads per block,
// blocks per SM, register cap); dg_sgns_autotune picks the shape.
// The staged-rows kernel's conditions (see sgns_plain_pipe_kernel).
static bool pipe_applies(const dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    return !s->p.deterministic && ws.max_len > 0 && ws.max_len <= kPipeSentence && a.window <= kPipeMaxWindow &&
           a.negative <= kFastNeg;
}

template <int V, int I, bool BF>
static void plain_fast_launch(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    constexpr int T = kPlainShapes[I].threads;
    constexpr int FIT = V >= 8 ? 0 : kPlainShapes[I].fit;
    constexpr int STG = kPlainShapes[I].stages;
    int blocks = 1, threads = 32;
    void (*kern)(SgnsArgs, WalkSet);
    bool staged = false;
    const bool neg_fixed = a.negative == kPlainNeg && a.vocab_size > 1;
    if constexpr (BF) {
        kern = neg_fixed ? sgns_plain_bf16_kernel<V, T, kPlainNeg, FIT> : sgns_plain_bf16_kernel<V, T, 0, FIT>;
        if constexpr (STG >= 2 && V == 4) {
            if (s->bf_staged && pipe_applies(s, a, ws)) {
                kern = neg_fixed ? sgns_plain_pipe_kernel<V, T, kPlainNeg, STG, FIT, true>
                                 : sgns_plain_pipe_kernel<V, T, 0, STG, FIT, true>;
                staged = true;
            }
        }
    } else {
        kern = neg_fixed ? sgns_plain_kernel<V, T, kPlainNeg, FIT> : sgns_plain_kernel<V, T, 0, FIT>;
        if constexpr (STG >= 2 && (V == 2 || V == 4)) {
            if (pipe_applies(s, a, ws)) {
                kern = neg_fixed ? sgns_plain_pipe_kernel<V, T, kPlainNeg, STG, FIT, false>
                                 : sgns_plain_pipe_kernel<V, T, 0, STG, FIT, false>;
                staged = true;
            }
        }
    }
    if (!s->p.deterministic) {
        // Register-capped shapes and the staged-rows kernel hold more blocks than
        // the default shared-memory carveout leaves room for.
        if (FIT || staged)
            cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T, 0);
        per_sm = std::max(per_sm, 1);
        if (kPlainShapes[I].per_sm > 0) per_sm = std::min(per_sm, kPlainShapes[I].per_sm);
        blocks = plain_blocks(s, dg::sm_count(s->device) * per_sm, T);
        threads = T;
    }
    kern<<<blocks, threads, 0, s->stream>>>(a, ws);
}

template <int V, bool BF>
static int plain_fast_shape(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    static_assert(kPlainShapeCount == 13, "dispatch below lists every shape");
    switch (s->plain_shape) {
    case 0: plain_fast_launch<V, 0, BF>(s, a, ws); break;
    case 1: plain_fast_launch<V, 1, BF>(s, a, ws); break;
    case 2: plain_fast_launch<V, 2, BF>(s, a, ws); break;
    case 3: plain_fast_launch<V, 3, BF>(s, a, ws); break;
    case 4: plain_fast_launch<V, 4, BF>(s, a, ws); break;
    case 5: plain_fast_launch<V, 5, BF>(s, a, ws); break;
    case 6: plain_fast_launch<V, 6, BF>(s, a, ws); break;
    case 7: plain_fast_launch<V, 7, BF>(s, a, ws); break;
    case 8: plain_fast_launch<V, 8, BF>(s, a, ws); break;
    case 9: plain_fast_launch<V, 9, BF>(s, a, ws); break;
    case 10: plain_fast_launch<V, 10, BF>(s, a, ws); break;
    case 11: plain_fast_launch<V, 11, BF>(s, a, ws); break;
    case 12: plain_fast_launch<V, 12, BF>(s, a, ws); break;
    default: return dg::fail(DG_ERR_ARG, "plain launch shape %d out of range", s->plain_shape);
    }
    return DG_OK;
}

// The plain rule on BF16 rows (DG_SGNS_PLAIN_BF16): size 64, 128 or 256, negative <= kFastNeg.
static int launch_plain_bf16(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    DG_CHECK(a.negative <= kFastNeg, DG_ERR_ARG, "the BF16 plain trainer supports negative <= %d", kFastNeg);
    int rc;
    switch (s->p.size) {
    case 64: rc = plain_fast_shape<2, true>(s, a, ws); break;
    case 128: rc = plain_fast_shape<4, true>(s, a, ws); break;
    case 256: rc = plain_fast_shape<8, true>(s, a, ws); break;
    default: return dg::fail(DG_ERR_ARG, "the BF16 plain trainer supports size 64, 128 or 256 (got %d)", s->p.size);
    }
    if (rc) return rc;
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    return DG_OK;
}

int launch_plain(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    if (s->p.mode == DG_SGNS_PLAIN_BF16) return launch_plain_bf16(s, a, ws);
    if (a.hs) return launch_plain_hs(s, a, ws);
    const int vec = s->p.size / 32;
    int blocks = 1, threads = 32;
    auto occ = [&](auto kern) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPlainThreads, 0);
        return std::max(per_sm, 1);
    };
    if (!s->p.deterministic) threads = kPlainThreads;
    const bool fast = a.negative <= kFastNeg;
    switch (vec) {
#define DG_PLAIN_CASE(V)                                                                             \
    case V:                                                                                          \
        if (fast) {                                                                                  \
            int rc_ = plain_fast_shape<V, false>(s, a, ws);                                          \
            if (rc_) return rc_;                                                                     \
        } else {                                                                                     \
            if (!s->p.deterministic)                                                                 \
                blocks = plain_blocks(s, dg::sm_count(s->device) * occ(sgns_plain_seq_kernel<V>), kPlainThreads); \
            sgns_plain_seq_kernel<V><<<blocks, threads, 0, s->stream>>>(a, ws);                      \
        }                                                                                            \
        dg::note_launch();                                                                           \
        break;
        DG_PLAIN_CASE(1)
        DG_PLAIN_CASE(2)
        DG_PLAIN_CASE(4)
        DG_PLAIN_CASE(8)
        DG_PLAIN_CASE(16)
#undef DG_PLAIN_CASE
    default:
        return dg::fail(DG_ERR_ARG, "size %d not supported (32, 64, 128, 256, 512)", s->p.size);
    }
    DG_CUDA(cudaGetLastError());
    return DG_OK;
}

// ----------------------------------------------------------------- output

__global__ void rows_to_f32(const __nv_bfloat16 *rows, const float *master, uint64_t n, uint64_t n_master, float *out) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        out[k] = k < n_master ? master[k] : __bfloat162float(rows[k]);
}

// Largest vertex id of a host-supplied walk set, checked on the device after the
// copy instead of element by element on the host.
__global__ void max_vertex_kernel(const uint32_t *v, uint64_t n, unsigned int *out) {
    uint32_t m = 0;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, __ldg(v + k));
#pragma unroll
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void rows_from_f32(const float *in, uint64_t n, uint64_t n_master, __nv_bfloat16 *rows, float *master) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        rows[k] = __float2bfloat16_rn(in[k]);
        if (k < n_master) master[k] = in[k];
    }
}

bool fp32_rows(const dg_sgns *s) {
    return s->p.mode == DG_SGNS_PLAIN || s->p.mode == DG_SGNS_CBOW || s->p.mode == DG_SGNS_SG_SHARED;
}

int copy_rows(const dg_sgns *s, bool input, float *host) {
    const uint64_t n = (uint64_t)s->vocab_size * s->p.size;
    if (fp32_rows(s)) {
        // Rows of out_size columns from rows stored with stride p.size.
        DG_CUDA(cudaMemcpy2DAsync(host, (size_t)s->out_size * 4, input ? s->syn0.p : s->syn1.p, (size_t)s->p.size * 4,
                                  (size_t)s->out_size * 4, s->vocab_size, cudaMemcpyDeviceToHost, s->stream));
        DG_CUDA(cudaStreamSynchronize(s->stream));
        return DG_OK;
    }
    dg::DevArray<float> tmp;
    DG_CUDA(tmp.alloc(n));
    rows_to_f32<<<dg::sm_count(s->device) * 4, 256, 0, s->stream>>>(input ? s->in_bf.p : s->out_bf.p,
                                                                     input ? s->in_master.p : s->out_master.p, n,
                                                                     (uint64_t)s->n_master * s->p.size, tmp.p); dg::note_launch();
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaMemcpyAsync(host, tmp.p, n * 4, cudaMemcpyDeviceToHost, s->stream));
    DG_CUDA(cudaStreamSynchronize(s->stream));
    return DG_OK;
}

}  // namespace dgs

dg_sgns::~dg_sgns() {
    if (stream) {
        dg::DeviceGuard guard(device);
        cudaStreamSynchronize(stream);
        v2w.release(); keep_thr.release(); table.release(); exp_table.release();
        hs_off.release(); hs_point.release(); hs_code.release();
        syn0.release(); syn1.release(); in_bf.release(); out_bf.release(); in_master.release(); out_master.release();
        scratch.release(); queue.release(); stats.release(); adj_in.release(); adj_out.release(); adj_flag.release();
        adj_offs.release(); adj_pin.release(); adj_pout.release(); adj_neg.release(); adj_step.release();
        if (adj_exec) cudaGraphExecDestroy(adj_exec);
        cudaStreamDestroy(stream);
    }
}

extern "C" int dg_sgns_create(const dg_sgns_params *p, uint32_t v_num, const uint32_t *vertex_counts, int device,
                              dg_sgns **out) {
    using namespace dgs;
    DG_CHECK(p && vertex_counts && out, DG_ERR_ARG, "dg_sgns_create: NULL argument");
    *out = nullptr;
    DG_CHECK(v_num > 0, DG_ERR_ARG, "dg_sgns_create: v_num must be positive");
    const bool fp32_mode = p->mode == DG_SGNS_PLAIN || p->mode == DG_SGNS_CBOW || p->mode == DG_SGNS_SG_SHARED;
    const bool pow2_size =
        p->size >= 32 && p->size <= 512 && p->size % 32 == 0 && ((p->size / 32) & (p->size / 32 - 1)) == 0;
    DG_CHECK(pow2_size || (fp32_mode && p->deterministic != 2 && p->size >= 1 && p->size <= 512), DG_ERR_ARG,
             "size %d not supported (32, 64, 128, 256 or 512; the FP32 word2vec rules also take any size up to 512, "
             "except in adjoint mode)", p->size);
    DG_CHECK(p->window >= 1 && p->window <= 64, DG_ERR_ARG, "window %d out of range [1, 64]", p->window);
    DG_CHECK(p->negative >= 0 && p->negative <= 64, DG_ERR_ARG, "negative %d out of range [0, 64]", p->negative);
    DG_CHECK(p->mode == DG_SGNS_PLAIN || p->mode == DG_SGNS_MINIBATCH || p->mode == DG_SGNS_PLAIN_BF16 ||
                 p->mode == DG_SGNS_CBOW || p->mode == DG_SGNS_SG_SHARED || p->mode == DG_SGNS_CBOW_BF16,
             DG_ERR_ARG, "unknown mode %d", p->mode);
    DG_CHECK((p->mode != DG_SGNS_CBOW && p->mode != DG_SGNS_CBOW_BF16) || p->negative <= kCbowMaxNeg, DG_ERR_ARG,
             "the CBOW trainer supports negative <= %d", kCbowMaxNeg);
    DG_CHECK(p->mode != DG_SGNS_CBOW_BF16 || p->size == 64 || p->size == 128 || p->size == 256, DG_ERR_ARG,
             "the BF16 CBOW trainer supports size 64, 128 or 256");
    DG_CHECK(p->mode != DG_SGNS_SG_SHARED || p->negative <= kShareMaxNeg, DG_ERR_ARG,
             "the shared-negative trainer supports negative <= %d", kShareMaxNeg);
    DG_CHECK(p->deterministic != 2 || p->mode == DG_SGNS_PLAIN || p->mode == DG_SGNS_MINIBATCH ||
                 p->mode == DG_SGNS_PLAIN_BF16,
             DG_ERR_ARG, "adjoint mode trains the skip-gram rules only");
    DG_CHECK(!p->hs || (p->deterministic != 2 && (p->mode == DG_SGNS_PLAIN || p->mode == DG_SGNS_CBOW ||
                                                  p->mode == DG_SGNS_SG_SHARED)),
             DG_ERR_ARG, "hierarchical softmax (hs) is available in the FP32 word2vec rules, not in adjoint mode");
    DG_CHECK(p->mode != DG_SGNS_PLAIN_BF16 || ((p->size == 64 || p->size == 128 || p->size == 256) && p->negative <= 8),
             DG_ERR_ARG, "the BF16 plain trainer supports size 64, 128 or 256 and negative <= 8");
    DG_CHECK(p->iter >= 1, DG_ERR_ARG, "iter must be >= 1");
    DG_CHECK(p->deterministic >= 0 && p->deterministic <= 2, DG_ERR_ARG, "deterministic must be 0, 1 or 2");
    DG_CHECK(p->deterministic != 2 || p->negative <= 16, DG_ERR_ARG, "adjoint mode supports negative <= 16");
    int n_dev = 0;
    DG_CUDA(cudaGetDeviceCount(&n_dev));
    DG_CHECK(device >= 0 && device < n_dev, DG_ERR_ARG, "device %d out of range (%d)", device, n_dev);

    std::unique_ptr<dg_sgns> s(new dg_sgns());
    s->device = device;
    s->p = *p;
    // FP32 rules: rows of any size are stored padded to the next of 32 .. 512
    // columns (zeros that no update changes: every update of a padding column
    // adds g * 0), so the kernels see one of their sizes.
    s->out_size = p->size;
    if (fp32_mode) {
        int dp = 32;
        while (dp < p->size) dp *= 2;
        s->p.size = dp;
    }
    if (s->p.table_size == 0) s->p.table_size = kDefaultTableSize;
    DG_CHECK(s->p.table_size < (1ull << 32), DG_ERR_ARG, "table_size must be < 2^32");
    s->v_num = v_num;
    build_vocab(vertex_counts, v_num, p->min_count, s->vocab_ids, s->vocab_cn, s->h_v2w, s->train_words);
    s->vocab_size = (uint32_t)s->vocab_ids.size();
    std::vector<uint32_t> thr;
    keep_thresholds(s->vocab_cn, p->sample, s->train_words, p->mode == DG_SGNS_MINIBATCH, thr);
    if (p->mode == DG_SGNS_MINIBATCH) s->mb_workers = dgs::mb_worker_bound(s->vocab_cn, thr, p->negative);
    if (p->deterministic == 2)
        s->adj_step_batches = dgs::adjoint_step_bound(
            s->vocab_cn, thr, p->batch_size > 0 ? p->batch_size : 2 * p->window + 1, p->negative);
    std::vector<int32_t> hs_off, hs_point;
    std::vector<int8_t> hs_code;
    const bool use_hs = p->hs && p->mode != DG_SGNS_SG_SHARED;   // __sgNegReuse has no HS branch
    if (use_hs)
        DG_CHECK(huffman_codes(s->vocab_cn, hs_off, hs_point, hs_code), DG_ERR_ARG,
                 "hierarchical softmax needs at least 2 words and codes of at most 40 bits (word2vec.cu:33)");
    s->p.hs = use_hs ? 1 : 0;
    std::vector<int32_t> table;
    unigram_table(s->vocab_cn, s->p.table_size, table);
    std::vector<float> et;
    exp_table(et);

    dg::DeviceGuard guard(device);
    DG_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    DG_CUDA(s->v2w.alloc(v_num));
    DG_CUDA(s->keep_thr.alloc(s->vocab_size));
    DG_CUDA(s->table.alloc(s->p.table_size));
    DG_CUDA(s->exp_table.alloc(et.size()));
    DG_CUDA(s->queue.alloc(1));
    DG_CUDA(s->stats.alloc(4));
    DG_CUDA(cudaMemcpyAsync(s->v2w.p, s->h_v2w.data(), (size_t)v_num * 4, cudaMemcpyHostToDevice, s->stream));
    DG_CUDA(cudaMemcpyAsync(s->keep_thr.p, thr.data(), thr.size() * 4, cudaMemcpyHostToDevice, s->stream));
    DG_CUDA(cudaMemcpyAsync(s->table.p, table.data(), table.size() * 4, cudaMemcpyHostToDevice, s->stream));
    DG_CUDA(cudaMemcpyAsync(s->exp_table.p, et.data(), et.size() * 4, cudaMemcpyHostToDevice, s->stream));
    if (use_hs) {
        DG_CUDA(s->hs_off.alloc(hs_off.size()));
        DG_CUDA(s->hs_point.alloc(hs_point.size()));
        DG_CUDA(s->hs_code.alloc(hs_code.size()));
        DG_CUDA(cudaMemcpyAsync(s->hs_off.p, hs_off.data(), hs_off.size() * 4, cudaMemcpyHostToDevice, s->stream));
        DG_CUDA(cudaMemcpyAsync(s->hs_point.p, hs_point.data(), hs_point.size() * 4, cudaMemcpyHostToDevice,
                                s->stream));
        DG_CUDA(cudaMemcpyAsync(s->hs_code.p, hs_code.data(), hs_code.size(), cudaMemcpyHostToDevice, s->stream));
        // The host vectors are freed on return: the copies must have read them.
        DG_CUDA(cudaStreamSynchronize(s->stream));
    }
    const uint64_t n = (uint64_t)s->vocab_size * s->p.size;
    const int blocks = dg::sm_count(device) * 8;
    if (p->mode == DG_SGNS_PLAIN || p->mode == DG_SGNS_CBOW || p->mode == DG_SGNS_SG_SHARED) {
        DG_CUDA(s->syn0.alloc(n));
        DG_CUDA(s->syn1.alloc(n));
        init_rows_f32<<<blocks, 256, 0, s->stream>>>(s->syn0.p, n, s->out_size, s->p.size); dg::note_launch();
        DG_CUDA(cudaGetLastError());
        DG_CUDA(cudaMemsetAsync(s->syn1.p, 0, n * 4, s->stream));
    } else {
        s->n_master = std::min<uint32_t>(s->vocab_size, p->master_rows ? p->master_rows : kMasterRows);
        if (p->mode == DG_SGNS_PLAIN_BF16) s->bf_staged = bf_staging_safe(s->vocab_cn, s->n_master, p->negative,
                                                                            dg::sm_count(device));
        const uint64_t nm = (uint64_t)s->n_master * p->size;
        DG_CUDA(s->in_bf.alloc(n));
        DG_CUDA(s->out_bf.alloc(n));
        DG_CUDA(s->in_master.alloc(nm));
        DG_CUDA(s->out_master.alloc(nm));
        init_rows_bf16<<<blocks, 256, 0, s->stream>>>(s->in_bf.p, s->in_master.p, n, nm, p->size); dg::note_launch();
        DG_CUDA(cudaGetLastError());
        DG_CUDA(cudaMemsetAsync(s->out_bf.p, 0, n * 2, s->stream));
        DG_CUDA(cudaMemsetAsync(s->out_master.p, 0, nm * 4, s->stream));
    }
    DG_CUDA(cudaStreamSynchronize(s->stream));
    *out = s.release();
    return DG_OK;
}

extern "C" void dg_sgns_free(dg_sgns *s) { delete s; }

static int train_walks(dg_sgns *s, const dgs::WalkSet &ws, float alpha, dg_train_info *info) {
    using namespace dgs;
    dg::DeviceGuard guard(s->device);
    SgnsArgs a{};
    a.v2w = s->v2w.p;
    a.keep_thr = s->keep_thr.p;
    a.table = s->table.p;
    a.exp_table = s->exp_table.p;
    a.syn0 = s->syn0.p;
    a.syn1 = s->syn1.p;
    a.in_bf = s->in_bf.p;
    a.out_bf = s->out_bf.p;
    a.in_master = s->in_master.p;
    a.out_master = s->out_master.p;
    a.n_master = s->n_master;
    a.queue = s->queue.p;
    a.stats = s->stats.p;
    a.table_size = s->p.table_size;
    a.vocab_size = s->vocab_size;
    a.window = s->p.window;
    a.negative = s->p.negative;
    a.d = s->p.size;
    a.alpha = alpha > 0 ? alpha : s->p.alpha;
    a.seed_lo = (uint32_t)s->p.seed;
    a.seed_hi = (uint32_t)(s->p.seed >> 32);
    a.deterministic = s->p.deterministic;
    a.train_words = s->train_words;
    a.hs = s->p.hs;
    a.hs_off = s->hs_off.p;
    a.hs_point = s->hs_point.p;
    a.hs_code = s->hs_code.p;
    DG_CUDA(cudaMemsetAsync(s->stats.p, 0, 4 * sizeof(unsigned long long), s->stream));
    dg::EventTimer t;
    t.start(s->stream);
    uint64_t adj_pairs = 0;
    for (int it = 0; it < s->p.iter; it++) {
        a.pass = s->pass++;
        DG_CUDA(cudaMemsetAsync(s->queue.p, 0, sizeof(uint32_t), s->stream));
        int rc;
        if (s->p.deterministic == 2) {
            uint64_t np = 0;
            rc = adjoint_train(s, a, ws, np);
            adj_pairs += np;
        } else {
            rc = s->p.mode == DG_SGNS_MINIBATCH   ? launch_minibatch(s, a, ws)
                 : s->p.mode == DG_SGNS_CBOW || s->p.mode == DG_SGNS_CBOW_BF16 ? launch_cbow(s, a, ws)
                 : s->p.mode == DG_SGNS_SG_SHARED ? launch_negshare(s, a, ws)
                                                  : launch_plain(s, a, ws);
        }
        if (rc) return rc;
    }
    t.stop(s->stream);
    if (s->p.deterministic == 2)
        DG_CUDA(cudaMemcpyAsync(s->stats.p + 2, &adj_pairs, 8, cudaMemcpyHostToDevice, s->stream));
    unsigned long long st[4];
    DG_CUDA(cudaMemcpyAsync(st, s->stats.p, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
    DG_CUDA(cudaStreamSynchronize(s->stream));
    if (info) {
        info->words = st[0];
        info->trained = st[1];
        info->pairs = st[2];
        info->train_ms = t.ms();
        info->rows = st[3];
    }
    return DG_OK;
}

extern "C" int dg_sgns_train_paths(dg_sgns *s, const dg_paths *paths, float alpha, dg_train_info *info);

// Times every launch shape of the plain kernel on these walks and keeps the
// fastest.  Rows and the pass counter are restored after each trial, so tuning
// leaves the trainer as it found it (apart from the launch shape).  Only the
// plain form's Hogwild kernel has shapes to choose from; other configurations
// report one candidate.
extern "C" int dg_sgns_autotune(dg_sgns *s, const dg_paths *paths, dg_tune_info *info) {
    DG_CHECK(s && paths, DG_ERR_ARG, "dg_sgns_autotune: NULL argument");
    dg_tune_info r{};
    if (s->p.mode == DG_SGNS_MINIBATCH || s->p.mode == DG_SGNS_CBOW || s->p.mode == DG_SGNS_CBOW_BF16 ||
        s->p.mode == DG_SGNS_SG_SHARED || s->p.deterministic || s->p.negative > dgs::kFastNeg || s->p.hs) {
        r.n_candidates = 1;
        r.chosen = 0;
        if (info) *info = r;
        return DG_OK;
    }
    dg::DeviceGuard guard(s->device);
    // Snapshots of every row buffer the trainer holds (FP32 rows, or BF16 rows + masters).
    struct Snap {
        void *dev;
        size_t bytes;
        dg::DevArray<uint8_t> copy;
    };
    Snap snaps[6] = {{s->syn0.p, s->syn0.bytes(), {}},       {s->syn1.p, s->syn1.bytes(), {}},
                     {s->in_bf.p, s->in_bf.bytes(), {}},     {s->out_bf.p, s->out_bf.bytes(), {}},
                     {s->in_master.p, s->in_master.bytes(), {}}, {s->out_master.p, s->out_master.bytes(), {}}};
    for (Snap &sn : snaps) {
        if (!sn.dev || !sn.bytes) continue;
        DG_CUDA(sn.copy.alloc(sn.bytes));
        DG_CUDA(cudaMemcpyAsync(sn.copy.p, sn.dev, sn.bytes, cudaMemcpyDeviceToDevice, s->stream));
    }
    const uint32_t pass0 = s->pass;
    const int shape0 = s->plain_shape;
    auto restore = [&]() -> int {
        for (Snap &sn : snaps)
            if (sn.dev && sn.bytes)
                DG_CUDA(cudaMemcpyAsync(sn.dev, sn.copy.p, sn.bytes, cudaMemcpyDeviceToDevice, s->stream));
        DG_CUDA(cudaStreamSynchronize(s->stream));
        s->pass = pass0;
        return DG_OK;
    };
    r.n_candidates = dgs::kPlainTunedShapes;
    double best = 1e300;
    for (int k = 0; k < dgs::kPlainTunedShapes; k++) {
        s->plain_shape = k;
        double ms = 0.0;
        for (int rep = 0; rep < 2; rep++) {   // the first run warms caches
            int rc = restore();
            if (!rc) {
                dg_train_info ti{};
                rc = dg_sgns_train_paths(s, paths, 0.0f, &ti);
                ms = ti.train_ms;
            }
            if (rc) {
                s->plain_shape = shape0;
                restore();
                return rc;
            }
        }
        if (k < DG_TUNE_MAX) {
            r.ms[k] = ms;
            r.shape[k][0] = dgs::kPlainShapes[k].threads;
            r.shape[k][1] = dgs::kPlainShapes[k].per_sm ? dgs::kPlainShapes[k].per_sm : dgs::kPlainShapes[k].fit;
            r.shape[k][2] = dgs::kPlainShapes[k].stages;
        }
        if (ms < best) {
            best = ms;
            r.chosen = k;
        }
    }
    int rc = restore();
    if (rc) return rc;
    s->plain_shape = r.chosen;
    if (info) *info = r;
    return DG_OK;
}

extern "C" int dg_sgns_set_shape(dg_sgns *s, int shape) {
    DG_CHECK(s, DG_ERR_ARG, "dg_sgns_set_shape: NULL trainer");
    DG_CHECK(shape >= 0 && shape < dgs::kPlainShapeCount, DG_ERR_ARG, "plain launch shape %d out of range [0, %d)",
             shape, dgs::kPlainShapeCount);
    s->plain_shape = shape;
    return DG_OK;
}

extern "C" int dg_sgns_train_paths(dg_sgns *s, const dg_paths *paths, float alpha, dg_train_info *info) {
    DG_CHECK(s && paths, DG_ERR_ARG, "dg_sgns_train_paths: NULL argument");
    DG_CHECK(paths->device == s->device, DG_ERR_ARG, "paths and trainer live on different devices");
    DG_CHECK(paths->g->v_num <= s->v_num, DG_ERR_ARG, "walks reference vertices beyond the vocabulary's v_num");
    dgs::WalkSet ws{};
    ws.verts = paths->verts.p;
    ws.lens = paths->lens.p;
    ws.stride = paths->stride;
    ws.n_walks = paths->n_walks;
    ws.max_len = paths->info.max_len;
    ws.id_base = 0;
    // The walk stream and the trainer stream are ordered by synchronising here.
    dg::DeviceGuard guard(s->device);
    DG_CUDA(cudaStreamSynchronize(paths->g->stream));
    return train_walks(s, ws, alpha, info);
}

extern "C" int dg_pipeline_round(dg_graph *g, dg_sgns *s, const dg_walk_params *p, uint32_t round, uint32_t n_walkers,
                                 float alpha, dg_pipeline_info *info, dg_paths **keep) {
    DG_CHECK(g && s && p, DG_ERR_ARG, "dg_pipeline_round: NULL argument");
    DG_CHECK(g->device == s->device, DG_ERR_ARG, "graph and trainer live on different devices");
    if (keep) *keep = nullptr;
    dg::DeviceGuard guard(g->device);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    DG_CUDA(cudaEventCreate(&t0));
    DG_CUDA(cudaEventCreate(&t1));
    struct Ev {
        cudaEvent_t &a, &b;
        ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } ev{t0, t1};
    DG_CUDA(cudaEventRecord(t0, g->stream));
    dg_paths *paths = nullptr;
    int rc = dg_walk_run_round(g, p, round, n_walkers, &paths);
    if (rc) return rc;
    dg_train_info tinfo{};
    rc = dg_sgns_train_paths(s, paths, alpha, &tinfo);
    if (rc) {
        dg_paths_free(paths);
        return rc;
    }
    DG_CUDA(cudaEventRecord(t1, s->stream));
    DG_CUDA(cudaEventSynchronize(t1));
    float ms = 0.f;
    DG_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    if (info) {
        info->walk = paths->info;
        info->train = tinfo;
        info->total_ms = ms;
    }
    if (keep) *keep = paths;
    else dg_paths_free(paths);
    return DG_OK;
}

extern "C" int dg_sgns_train_host(dg_sgns *s, const uint64_t *offsets, uint32_t n_walks, const uint32_t *vertices,
                                  float alpha, dg_train_info *info) {
    DG_CHECK(s && offsets && (vertices || offsets[n_walks] == 0), DG_ERR_ARG, "dg_sgns_train_host: NULL argument");
    const uint64_t total = offsets[n_walks];
    uint64_t longest = 0;   // one pass over the offsets: order check and the longest walk
    for (uint32_t i = 0; i < n_walks; i++) {
        DG_CHECK(offsets[i + 1] >= offsets[i], DG_ERR_ARG, "walk offsets decrease at walk %u", i);
        longest = std::max<uint64_t>(longest, offsets[i + 1] - offsets[i]);
    }
    dg::DeviceGuard guard(s->device);
    dg::DevArray<uint64_t> &d_off = s->host_off;
    dg::DevArray<uint32_t> &d_verts = s->host_verts;
    if (d_off.n < (size_t)n_walks + 1) DG_CUDA(d_off.alloc((size_t)n_walks + 1 + n_walks / 8));
    if (d_verts.n < (total ? total : 1)) DG_CUDA(d_verts.alloc((total ? total : 1) + total / 8));
    DG_CUDA(cudaMemcpyAsync(d_off.p, offsets, ((size_t)n_walks + 1) * 8, cudaMemcpyHostToDevice, s->stream));
    if (total) {
        DG_CUDA(cudaMemcpyAsync(d_verts.p, vertices, total * 4, cudaMemcpyHostToDevice, s->stream));
        if (!s->vmax.p) DG_CUDA(s->vmax.alloc(1));
        DG_CUDA(cudaMemsetAsync(s->vmax.p, 0, sizeof(unsigned int), s->stream));
        dgs::max_vertex_kernel<<<dg::sm_count(s->device) * 4, 256, 0, s->stream>>>(d_verts.p, total, s->vmax.p);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
        unsigned int vmax = 0;
        DG_CUDA(cudaMemcpyAsync(&vmax, s->vmax.p, sizeof(vmax), cudaMemcpyDeviceToHost, s->stream));
        DG_CUDA(cudaStreamSynchronize(s->stream));
        DG_CHECK(vmax < s->v_num, DG_ERR_ARG, "vertex %u >= v_num %u", vmax, s->v_num);
    }
    dgs::WalkSet ws{};
    ws.verts = d_verts.p;
    ws.offsets = d_off.p;
    ws.n_walks = n_walks;
    ws.max_len = (uint32_t)std::min<uint64_t>(longest, UINT32_MAX);
    ws.id_base = 0;
    return train_walks(s, ws, alpha, info);
}

extern "C" int dg_sgns_copy_embedding(const dg_sgns *s, float *rows, uint32_t *vocab_ids, uint32_t *n_rows) {
    DG_CHECK(s, DG_ERR_ARG, "dg_sgns_copy_embedding: NULL trainer");
    if (n_rows) *n_rows = s->vocab_size;
    if (vocab_ids) memcpy(vocab_ids, s->vocab_ids.data(), s->vocab_ids.size() * 4);
    if (!rows) return DG_OK;
    dg::DeviceGuard guard(s->device);
    return dgs::copy_rows(s, true, rows);
}

extern "C" int dg_sgns_copy_output(const dg_sgns *s, float *rows) {
    DG_CHECK(s && rows, DG_ERR_ARG, "dg_sgns_copy_output: NULL argument");
    dg::DeviceGuard guard(s->device);
    return dgs::copy_rows(s, false, rows);
}

extern "C" int dg_sgns_copy_tables(const dg_sgns *s, int32_t *table, uint32_t *keep_thr, int32_t *v2w,
                                   float *exp_table) {
    DG_CHECK(s, DG_ERR_ARG, "dg_sgns_copy_tables: NULL trainer");
    dg::DeviceGuard guard(s->device);
    DG_CUDA(cudaStreamSynchronize(s->stream));
    if (table) DG_CUDA(cudaMemcpy(table, s->table.p, s->table.bytes(), cudaMemcpyDeviceToHost));
    if (keep_thr) DG_CUDA(cudaMemcpy(keep_thr, s->keep_thr.p, s->keep_thr.bytes(), cudaMemcpyDeviceToHost));
    if (v2w) DG_CUDA(cudaMemcpy(v2w, s->v2w.p, s->v2w.bytes(), cudaMemcpyDeviceToHost));
    if (exp_table) DG_CUDA(cudaMemcpy(exp_table, s->exp_table.p, s->exp_table.bytes(), cudaMemcpyDeviceToHost));
    return DG_OK;
}

extern "C" int dg_sgns_get_info(const dg_sgns *s, dg_sgns_info *info) {
    DG_CHECK(s && info, DG_ERR_ARG, "dg_sgns_get_info: NULL argument");
    info->vocab_size = s->vocab_size;
    info->master_rows = s->n_master;
    info->bf_staged = s->bf_staged ? 1 : 0;
    info->workers = s->p.workers ? s->p.workers : s->p.deterministic == 2 ? s->adj_step_batches : s->mb_workers;
    info->train_words = s->train_words;
    info->table_size = s->p.table_size;
    info->device_bytes = s->v2w.bytes() + s->keep_thr.bytes() + s->table.bytes() + s->exp_table.bytes() +
                         s->syn0.bytes() + s->syn1.bytes() + s->in_bf.bytes() + s->out_bf.bytes() +
                         s->in_master.bytes() + s->out_master.bytes() + s->scratch.bytes();
    return DG_OK;
}

extern "C" int dg_sgns_set_rows(dg_sgns *s, const float *input_rows, const float *output_rows) {
    DG_CHECK(s, DG_ERR_ARG, "dg_sgns_set_rows: NULL trainer");
    dg::DeviceGuard guard(s->device);
    const uint64_t n = (uint64_t)s->vocab_size * s->p.size;
    for (int k = 0; k < 2; k++) {
        const float *src = k == 0 ? input_rows : output_rows;
        if (!src) continue;
        if (dgs::fp32_rows(s)) {
            DG_CUDA(cudaMemcpy2DAsync(k == 0 ? s->syn0.p : s->syn1.p, (size_t)s->p.size * 4, src,
                                      (size_t)s->out_size * 4, (size_t)s->out_size * 4, s->vocab_size,
                                      cudaMemcpyHostToDevice, s->stream));
        } else {
            dg::DevArray<float> tmp;
            DG_CUDA(tmp.alloc(n));
            DG_CUDA(cudaMemcpyAsync(tmp.p, src, n * 4, cudaMemcpyHostToDevice, s->stream));
            dgs::rows_from_f32<<<dg::sm_count(s->device) * 4, 256, 0, s->stream>>>(
                tmp.p, n, (uint64_t)s->n_master * s->p.size, k == 0 ? s->in_bf.p : s->out_bf.p,
                k == 0 ? s->in_master.p : s->out_master.p); dg::note_launch();
            DG_CUDA(cudaGetLastError());
            DG_CUDA(cudaStreamSynchronize(s->stream));
        }
    }
    DG_CUDA(cudaStreamSynchronize(s->stream));
    return DG_OK;
}

// Embedding text (word2vec.cu:1353-1362): "%lld %lld\n", then per row the word
// (the vertex id in decimal), a space, size x "%lf ", "\n".  Rows are formatted
// by host threads in blocks and written in order.
extern "C" int dg_sgns_write_embedding(const dg_sgns *s, const char *file_path) {
    DG_CHECK(s && file_path, DG_ERR_ARG, "dg_sgns_write_embedding: NULL argument");
    const uint32_t rows = s->vocab_size;
    const int d = s->out_size;
    std::vector<float> emb((size_t)rows * d);
    dg::DeviceGuard guard(s->device);
    int rc = dgs::copy_rows(s, true, emb.data());
    if (rc) return rc;
    FILE *f = fopen(file_path, "wb");
    DG_CHECK(f != nullptr, DG_ERR_IO, "cannot open %s for writing", file_path);
    fprintf(f, "%lld %lld\n", (long long)rows, (long long)d);
    const uint32_t block = 4096;
    unsigned n_threads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    bool ok = true;
    for (uint32_t base = 0; base < rows && ok; base += block * n_threads) {
        std::vector<std::string> parts(n_threads);
        std::vector<std::thread> th;
        for (unsigned t = 0; t < n_threads; t++) {
            th.emplace_back([&, t] {
                const uint32_t lo = base + t * block, hi = std::min<uint32_t>(rows, lo + block);
                std::string &out = parts[t];
                char buf[64];
                for (uint32_t r = lo; r < hi; r++) {
                    int k = snprintf(buf, sizeof(buf), "%u ", s->vocab_ids[r]);
                    out.append(buf, k);
                    for (int j = 0; j < d; j++) {
                        k = snprintf(buf, sizeof(buf), "%lf ", (double)emb[(size_t)r * d + j]);
                        out.append(buf, k);
                    }
                    out.push_back('\n');
                }
            });
        }
        for (auto &x : th) x.join();
        for (auto &p : parts)
            if (!p.empty() && fwrite(p.data(), 1, p.size(), f) != p.size()) ok = false;
    }
    const int cl = fclose(f);
    DG_CHECK(ok && cl == 0, DG_ERR_IO, "short write to %s", file_path);
    return DG_OK;
}
