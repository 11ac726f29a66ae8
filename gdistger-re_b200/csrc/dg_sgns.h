// Internal declarations of the SGNS trainer (not part of the C ABI).
#pragma once

#include "dg_internal.h"
#include "dg_philox.cuh"

#include <cuda_bf16.h>

#include <string>
#include <vector>

namespace dgs {

constexpr int kExpTableSize = 1000;               // word2vec.cu:29
constexpr int kMaxExp = 6;                        // word2vec.cu:30
constexpr uint64_t kDefaultTableSize = 100000000; // word2vec.cu:66
constexpr uint32_t kMaxSentence = 1024;           // tokens of one walk used for training
constexpr int kPlainThreads = 256;
// Launch shapes of the fast plain kernel: threads per block (one walk per warp),
// blocks per SM (0: as many as fit), for register-capped instances the number
// of resident blocks per SM the kernel is compiled to fit (its __launch_bounds__
// minimum; 0: no cap; ignored for rows of 256 floats and more, where the cap
// would spill), and the pairs whose rows are staged ahead in shared memory
// (0: sgns_plain_kernel; S >= 2: sgns_plain_pipe_kernel where it applies, else
// sgns_plain_kernel with the same threads and cap).  Shape 0 is the default.
// The autotuner times the first kPlainTunedShapes; the last shape, one warp per
// block, exists so that a run with one worker is one warp of the staged kernel
// (its exact replay test).
struct PlainShape {
    int threads, per_sm, fit, stages;
};
constexpr PlainShape kPlainShapes[] = {{64, 0, 12, 2}, {256, 0, 0, 0}, {128, 0, 0, 0}, {64, 0, 0, 0},
                                       {64, 0, 12, 0}, {64, 0, 16, 0}, {256, 2, 0, 0}, {128, 4, 0, 0},
                                       {64, 0, 0, 2},  {64, 0, 16, 2}, {64, 0, 12, 3}, {64, 0, 0, 3},
                                       {32, 0, 0, 2}};
constexpr int kPlainShapeCount = (int)(sizeof(kPlainShapes) / sizeof(kPlainShapes[0]));
constexpr int kPlainTunedShapes = 12;
constexpr uint32_t kMasterRows = 1u << 16;        // hottest rows kept in FP32 in the minibatch form

// Philox counter word 3 of each random choice (counter words 0-2: index, walk, pass).
constexpr uint32_t kSubTag = 0x53554253u;  // subsampling of token i
constexpr uint32_t kWinTag = 0x57494E44u;  // window shrink of centre p
constexpr uint32_t kNegTag = 0x4E454730u;  // negatives of pair (p, slot), + j / 4
constexpr uint32_t kCbowTag = 0x43424F57u;   // CBOW negatives of centre p, + j / 4
constexpr uint32_t kShareTag = 0x53484E47u;  // shared negatives of a walk (counter word 0 = 0), + j / 4

// Walks to train on: slot layout (verts + w * stride, lens[w]) or compact
// (verts + offsets[w] .. offsets[w + 1]).
struct WalkSet {
    const uint32_t *verts = nullptr;
    const uint32_t *lens = nullptr;
    const uint64_t *offsets = nullptr;
    const uint32_t *ids = nullptr;  // walk id for the random counters (default: index + id_base)
    uint32_t stride = 0;
    uint32_t n_walks = 0;
    uint32_t max_len = 0;            // longest walk in footprints (0: not known)
    uint32_t id_base = 0;
    __device__ __forceinline__ void range(uint32_t w, uint64_t &begin, uint32_t &len) const {
        if (offsets) {
            begin = offsets[w];
            len = (uint32_t)(offsets[w + 1] - begin);
        } else {
            begin = (uint64_t)w * stride;
            len = lens[w];
        }
    }
};

struct SgnsArgs {
    const int32_t *v2w;
    const uint32_t *keep_thr;
    const int32_t *table;
    const float *exp_table;
    float *syn0, *syn1;                 // plain form, FP32 rows
    __nv_bfloat16 *in_bf, *out_bf;      // minibatch form, BF16 rows
    float *in_master, *out_master;      // minibatch form, FP32 rows of the hottest words
    uint32_t n_master;
    uint32_t *queue;
    unsigned long long *stats;          // words, trained, pairs
    uint64_t table_size;
    uint64_t train_words;
    uint32_t vocab_size;
    int window, negative, d;
    float alpha;
    uint32_t pass, seed_lo, seed_hi;
    int deterministic;
    int hs;                             // hierarchical softmax: Huffman paths below
    const int32_t *hs_off, *hs_point;   // [vocab + 1] code-length prefix; inner node per bit
    const int8_t *hs_code;              // bit per path entry
};

// Warp sums of M per-lane partials v[0..M) (M a power of two <= 32) for the cost
// of about one: each halving stage sends half of the values still held to the
// partner lane and keeps the other half, so after log2(M) stages lane l holds
// one value, index l >> (5 - log2 M), summed over its lane group; plain
// butterfly stages finish it.  Every addition is the one the plain butterfly
// (s += shfl_xor(s, o), o = 16 .. 1) makes for that value (own partial +
// partner's, then the same tree), so each sum is bit-identical to the plain
// butterfly's.  Returns the held sum; v is clobbered.
template <int M>
__device__ __forceinline__ float warp_sums_split(float (&v)[M], uint32_t lane) {
    static_assert(M >= 1 && M <= 32 && (M & (M - 1)) == 0, "M must be a power of two <= 32");
#pragma unroll
    for (int m = M, o = 16; m > 1; m >>= 1, o >>= 1) {
        const bool up = (lane & (uint32_t)o) != 0;
#pragma unroll
        for (int k = 0; k < m / 2; k++) {
            const float send = up ? v[k] : v[k + m / 2];
            const float keep = up ? v[k + m / 2] : v[k];
            v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    float s = v[0];
#pragma unroll
    for (int o = 16 / M; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

constexpr int pow2_at_least(int x) { return x <= 1 ? 1 : 2 * pow2_at_least((x + 1) / 2); }

int launch_plain(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws);
bool bf_staging_safe(const std::vector<uint32_t> &cn, uint32_t n_master, int negative, int sms);
int launch_minibatch(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws);
// cbow_kernel and __sgNegReuse semantics (dg_sgns_w2v.cu).
int launch_cbow(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws);
int launch_plain_hs(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws);
// word2vec's Huffman coding (CreateBinaryTree, word2vec.cu:684-740) of counts in
// vocabulary order, laid out as off[n + 1] / point / code.  false if a code
// would exceed the reference's 40 bits.
bool huffman_codes(const std::vector<uint32_t> &cn, std::vector<int32_t> &off, std::vector<int32_t> &point,
                   std::vector<int8_t> &code);
int launch_negshare(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws);
constexpr int kCbowMaxNeg = 32;   // one negative per lane
constexpr int kShareMaxNeg = 16;  // shared negatives held in shared memory per warp

// Concurrency bound of the minibatch form from the vocabulary (counts in
// vocabulary order, subsampling keep thresholds out of 65536).
uint32_t mb_worker_bound(const std::vector<uint32_t> &cn, const std::vector<uint32_t> &keep_thr, int negative);

// Shares of the hottest row: among negative draws (unigram^0.75) and among
// tokens kept by subsampling.
void hot_row_shares(const std::vector<uint32_t> &cn, const std::vector<uint32_t> &keep_thr, double &p_neg,
                    double &p_tok);

// Adjoint mode (deterministic = 2): gradient steps of the hand-written backward
// kernel over the pass's pairs in shared-negative minibatches.
int adjoint_pairs(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws, uint64_t &n_pairs);
int adjoint_train(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws, uint64_t &n_pairs);
uint32_t adjoint_step_bound(const std::vector<uint32_t> &cn, const std::vector<uint32_t> &keep_thr, int batch,
                            int negative);

// Device-resident parameters of the adjoint mode's gradient steps.  The kernels
// of a captured CUDA graph read the step index here (adj_advance moves it on),
// so one instantiated graph of several steps serves every round.
struct AdjStep {
    uint64_t n_pairs, n_batches, k;  // k: minibatches per step
    float alpha;
    uint64_t step;
};

}  // namespace dgs

struct dg_sgns;
namespace dgs {
// Whether the trainer keeps its rows in FP32 (syn0 / syn1): the word2vec.cu
// rules; the minibatch and BF16 forms keep BF16 rows + FP32 masters.
bool fp32_rows(const dg_sgns *s);
}  // namespace dgs

struct dg_sgns {
    int device = 0;
    cudaStream_t stream = nullptr;
    dg_sgns_params p{};                // p.size: the row stride the kernels use (padded for the FP32 rules)
    int out_size = 0;                  // the caller's -size: columns of the embedding
    uint32_t v_num = 0;
    uint32_t vocab_size = 0;
    uint32_t n_master = 0;
    uint32_t mb_workers = 0;           // minibatch form: staleness bound on concurrent workers
    int plain_shape = 0;               // plain form: launch shape (dg_sgns_autotune)
    bool bf_staged = false;            // BF16 plain mode: rows may be staged (dgs::bf_staging_safe)
    uint64_t train_words = 0;
    uint32_t pass = 0;
    std::vector<uint32_t> vocab_ids, vocab_cn;
    std::vector<int32_t> h_v2w;
    dg::DevArray<int32_t> v2w;
    dg::DevArray<uint32_t> keep_thr;
    dg::DevArray<int32_t> table;
    dg::DevArray<float> exp_table;
    dg::DevArray<float> syn0, syn1;
    dg::DevArray<__nv_bfloat16> in_bf, out_bf;
    dg::DevArray<float> in_master, out_master;
    dg::DevArray<float> scratch;       // minibatch form: per-worker negative pools and cache snapshots
    dg::DevArray<unsigned long long> adj_in, adj_out;  // adjoint: fixed-point gradient sums (vocab x size)
    dg::DevArray<unsigned int> adj_flag;
    dg::DevArray<uint64_t> adj_offs;                    // adjoint mode: pair offsets per walk
    dg::DevArray<uint32_t> adj_pin, adj_pout, adj_neg;  // adjoint mode: pairs and shared negatives
    bool adj_dirty = false;                             // accumulators hold a finished gradient
    uint32_t adj_step_batches = 1;                      // adjoint mode: minibatches per gradient step
    dg::DevArray<dgs::AdjStep> adj_step;                // adjoint mode: step parameters read by the graph
    cudaGraphExec_t adj_exec = nullptr;                 // adjoint mode: kAdjGraphSteps steps, captured once
    const void *adj_exec_key[3] = {nullptr, nullptr, nullptr};  // buffers the captured graph points at
    uint64_t adj_exec_k = 0;
    dg::DevArray<int32_t> hs_off, hs_point;   // hierarchical softmax: Huffman paths (dgs::huffman_codes)
    dg::DevArray<int8_t> hs_code;
    dg::DevArray<uint32_t> queue;
    dg::DevArray<unsigned long long> stats;
    dg::DevArray<uint64_t> host_off;     // dg_sgns_train_host: device copies of the caller's walks,
    dg::DevArray<uint32_t> host_verts;   // kept (and grown) between calls
    dg::DevArray<unsigned int> vmax;     // dg_sgns_train_host: largest vertex id of the call
    ~dg_sgns();
};
