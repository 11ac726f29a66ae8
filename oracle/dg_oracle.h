/*
 * CPU restatement of the reference's walk hot path and SGNS updates.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that the CUDA library is compared
 * against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it; the shipped library never links or calls it.
 *
 * Walk parity is pinned against the reference itself: with the stream random
 * source (dgo_stream_*), dgo_walk_rounds() reproduces, byte for byte, the walk
 * files of the unmodified reference engine built by `make -C oracle ref`
 * (oracle/_ref/ref_walk, one worker thread, pinned mt19937 seed).
 */
#ifndef DG_ORACLE_H
#define DG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Directed CSR built exactly as include/graph.hpp:642-824 + 509-540 build it
 * for one partition: optional undirected doubling in record order
 * (graph.hpp:671-686), out/in degrees (694-717), neighbours bucketed by source in
 * edge order (build_edge_container, 509-540). */
typedef struct {
    uint32_t v_num;
    uint64_t m;
    uint64_t *offsets;  /* v_num + 1 */
    uint32_t *nbr;      /* m */
    float *data;        /* m */
    uint32_t *out_deg;  /* v_num */
    uint32_t *in_deg;   /* v_num */
} dgo_csr;

typedef struct {
    uint32_t src, dst;
    float data;
} dgo_edge;

int dgo_csr_build(const dgo_edge *edges, uint64_t n_edges, uint32_t v_num, int undirected, dgo_csr *out);
void dgo_csr_free(dgo_csr *g);

/* Random source for the walk. */
enum { DGO_RNG_PHILOX = 0, DGO_RNG_CALLBACK = 1 };
typedef uint32_t (*dgo_cand_fn)(void *ctx, uint32_t degree);
typedef uint32_t (*dgo_acc_fn)(void *ctx);

typedef struct {
    uint32_t min_len;    /* --min_L, walk.hpp:404 */
    uint32_t init_round; /* --min_R, walk.hpp:405 */
    uint32_t walker_num; /* -w */
    uint32_t rounds;     /* last round index; the reference stops after 30 (walk.hpp:740) */
    uint64_t seed;       /* Philox key */
    int rng_mode;
    dgo_cand_fn cand_cb; /* DGO_RNG_CALLBACK only */
    dgo_acc_fn acc_cb;
    void *cb_ctx;
} dgo_walk_params;

typedef struct {
    uint64_t footprints;  /* all footprints, start vertices included */
    uint64_t steps;       /* footprints with step >= 1: the reference's p_step (walk.hpp:864,962,988) */
    uint64_t draws;       /* candidate draws (transition attempts) */
    uint64_t traces;      /* rejected candidates: walk.hpp:938-942 trace_num */
    uint64_t pow_sq_mismatch; /* R values where pow(R,2) != R*R (expected 0) */
    uint64_t near_ties;   /* draws with |tanh(p_accept) - p| < 1e-12 */
    uint32_t max_len;     /* longest walk, in footprints */
} dgo_walk_stats;

/* Walks of one round: walker w starts at w % v_num (walk.hpp:501-509). */
typedef struct {
    uint32_t n_walks;
    uint64_t total;
    uint64_t *offsets; /* n_walks + 1 */
    uint32_t *verts;   /* total */
} dgo_paths;

/* Advances walkers [0, n_walkers) of `round` to completion, in ascending id order
 * (the order a one-worker reference run uses), following walk.hpp:845-1024. */
int dgo_walk_round(const dgo_csr *g, const dgo_walk_params *p, uint32_t round, uint32_t n_walkers,
                   dgo_paths *out, dgo_walk_stats *stats);
void dgo_paths_free(dgo_paths *p);

/* Walks of the listed walker ids of `round` (Philox mode only). */
int dgo_walk_ids(const dgo_csr *g, const dgo_walk_params *p, uint32_t round, const uint32_t *ids, uint32_t n_ids,
                 dgo_paths *out, dgo_walk_stats *stats);

/* Writes one walk per line as " %u" per vertex then "\n" (path.hpp:67-119). */
int dgo_write_walks(const char *path, const dgo_paths *p);

/* Relative entropy of cumulative visit frequency vs out-degree share
 * (walk.hpp:694-725), natural log, summed in vertex order. */
double dgo_relative_entropy(const uint32_t *out_deg, const uint32_t *freq, uint32_t v_num);

/* Per-CSR-entry acceptance threshold: the smallest k in [0, 2^31-1] with
 * tanh(p_accept) <= k / 2147483647.0 (glibc tanh), or 2^31 when none exists. */
void dgo_thresholds(const dgo_csr *g, uint32_t *thr);

/* t(Sn, fi) = log2(A(Sn) * B(fi)) as Correlation::iterateHn computes it
 * (walk.hpp:284-303), tabulated for 1 <= Sn <= max_sn, 0 <= fi <= Sn at index
 * Sn*(Sn+1)/2 + fi - 1. */
void dgo_entropy_table(uint32_t max_sn, double *out);
uint64_t dgo_entropy_table_size(uint32_t max_sn);

/* Philox4x32-10 block (known-answer tests). */
void dgo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* The reference's candidate / acceptance streams for the pin test:
 * std::mt19937(seed) + std::uniform_int_distribution<uint32_t>(0, degree-1)
 * (util.hpp:37-41) and glibc rand() from its default state (walk.hpp:928). */
void *dgo_stream_new(uint32_t seed);
void dgo_stream_free(void *s);
uint32_t dgo_stream_cand(void *s, uint32_t degree);
uint32_t dgo_stream_acc(void *s);

/* ------------------------------------------------------------------ SGNS -- */

/* Philox counter word 3 of the trainer's random choices. */
#define DGO_SUB_TAG 0x53554253u /* subsampling: counter (token index, walk, pass, tag) */
#define DGO_WIN_TAG 0x57494E44u /* window shrink: (centre position, walk, pass, tag) */
#define DGO_NEG_TAG 0x4E454730u /* negatives: (pair index, walk, pass, tag + j/4), word j%4 */
#define DGO_CBOW_TAG 0x43424F57u  /* CBOW negatives: (centre position, walk, pass, tag + j/4), word j%4 */
#define DGO_SHARE_TAG 0x53484E47u /* shared negatives of a walk: (0, walk, pass, tag + j/4), word j%4 */

typedef struct {
    int d, window, negative;
    double alpha;
    uint64_t seed;
    uint32_t pass;
    uint32_t vocab_size;
    uint64_t table_size;
    const int32_t *table;
    const uint32_t *keep_thr;
    const int32_t *v2w;
    const float *exp_table;
    int hs;                 /* hierarchical softmax (word2vec -hs 1) with the codes below */
    const int32_t *hs_off;  /* [vocab_size + 1] prefix of the code lengths (dgo_huffman) */
    const int32_t *hs_point;
    const int8_t *hs_code;
} dgo_sgns_cfg;

typedef struct {
    uint64_t words, trained, pairs;
} dgo_sgns_stats;

int dgo_vocab_build(const uint32_t *counts, uint32_t v_num, int min_count, uint32_t *vocab_ids, uint32_t *vocab_cn,
                    int32_t *v2w, uint32_t *vocab_size, uint64_t *train_words);
void dgo_unigram_table(const uint32_t *cn, uint32_t vocab_size, uint64_t table_size, int32_t *table);
void dgo_keep_thresholds(const uint32_t *cn, uint32_t vocab_size, float sample, uint64_t train_words, int dsgl_form,
                         uint32_t *thr);
void dgo_init_rows(uint32_t vocab_size, int d, float *syn0);
void dgo_exp_table(float *t);
int dgo_sgns_plain(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                   const uint32_t *walk_ids, double *syn0, double *syn1, dgo_sgns_stats *st);
/* dsgl.hpp Train_SGNS_MPI semantics, one worker over all walks (walk id = index). */
int dgo_sgns_minibatch(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                       double *syn0, double *syn1, dgo_sgns_stats *st);
/* The same two rules in FP32 in the device kernels' exact operation order
 * (dg_oracle_sgns32.c): bit-exact against the deterministic device mode. */
int dgo_sgns_plain_f32(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                       float *syn0, float *syn1, dgo_sgns_stats *st);
int dgo_sgns_minibatch_f32(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                           float *syn0, float *syn1, dgo_sgns_stats *st);

/* word2vec.cu's trainers (dg_oracle_w2v.c).  Order of a dot product: the
 * reference kernels' (a shared-memory tree for skip_gram_kernel / cbow_kernel,
 * per-lane strided sums for __sgNegReuse) or the device kernels' warp order. */
enum { DGO_ORDER_DEVICE = 0, DGO_ORDER_REF = 1 };
enum { DGO_W2V_SG = 0, DGO_W2V_CBOW = 1, DGO_W2V_NEGREUSE = 2 };

typedef struct {
    int kind, d, window, negative;
    float alpha;
    uint32_t vocab_size;
    uint64_t table_size;
    const int32_t *table;
    const float *exp_table;
    int exact_sum; /* __sgNegReuse: 0 = reduceInWarp as the reference writes it, 1 = the warp sum */
    int hs;        /* hierarchical softmax with the codes below (skip_gram_kernel, cbow_kernel) */
    const int32_t *hs_off, *hs_point;
    const int8_t *hs_code;
} dgo_w2v_cfg;

/* The reference kernels on host-built sentences (token -1 = none), sentence k
 * trained by "block" k with its LCG seeded k, sentences one after another;
 * neg_samples[k * negative + y] = __sgNegReuse's shared negatives of sentence k. */
int dgo_w2v_sentences(const dgo_w2v_cfg *c, const int32_t *sen, const int32_t *sent_off, uint32_t n_sent,
                      const int32_t *neg_samples, float *syn0, float *syn1);
/* The shared per-pair / per-centre updates (both forms); hs_point / hs_code /
 * n_hs: the centre's hierarchical-softmax path (n_hs = 0 without -hs). */
void dgo_w2v_sg_pair(int order, int d, float alpha, const float *exp_table, float *l1, const int32_t *hs_point,
                     const int8_t *hs_code, int n_hs, const int32_t *tg, int nt, float *syn1, float *e);
void dgo_w2v_cbow_centre(int order, int d, float alpha, const float *exp_table, const int32_t *ctx, int cw,
                         const int32_t *hs_point, const int8_t *hs_code, int n_hs, const int32_t *tg, int nt,
                         float *syn0, float *syn1, float *neu1, float *e);
/* word2vec's Huffman coding (CreateBinaryTree, word2vec.cu:684-740) in the
 * kernels' prefix layout; see dg_oracle_w2v.c. */
int64_t dgo_huffman(const uint64_t *cn, uint32_t n, int32_t *off, int32_t *point, int8_t *code);
void dgo_w2v_reuse_pair(int order, int exact_sum, int d, float alpha, const float *exp_table, float *l1,
                        int32_t word, const int32_t *negs, int n, float *syn1, float *e);
/* Device forms of CBOW and of shared-negative skip-gram over walks. */
int dgo_sgns_cbow_f32(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                      float *syn0, float *syn1, dgo_sgns_stats *st);
int dgo_sgns_negshare_f32(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                          float *syn0, float *syn1, dgo_sgns_stats *st);

/* The staged-rows plain kernel (sgns_plain_pipe_kernel) run by one warp,
 * modelled bit for bit (dg_oracle_pipe.c): rows of pair m copied after the
 * updates of pairs < m - stages + 1, FP32 rows / masters updated by additions,
 * BF16 rows (ids >= n_master when bf16) overwritten with stochastically rounded
 * copies.  rows_in / rows_out: FP32 values (BF16 rows hold BF16-exact values). */
typedef struct {
    int d, window, negative, stages, bf16;
    float alpha;
    uint64_t seed;        /* Philox key of the trainer's draws */
    uint32_t seed_lo;     /* low word of the seed (BF16 noise key) */
    uint32_t pass;
    uint32_t vocab_size, n_master;
    uint64_t table_size;
    const int32_t *table;
    const uint32_t *keep_thr;
    const int32_t *v2w;
    const float *exp_table;
} dgo_pipe_cfg;
int dgo_sgns_pipe(const dgo_pipe_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                  float *rows_in, float *rows_out, dgo_sgns_stats *st);

/* dsgl's Train_SGNS_MPI compute thread in the reference's own random stream and
 * arithmetic order (dg_oracle_sgns32.c): reproduces, bit for bit, the rows of the
 * unmodified dsgl trainer built by `make -C oracle ref` (oracle/_ref/ref_dsgl,
 * one compute thread).  Its minibatch step is the one dgo_sgns_minibatch_f32
 * uses. */
typedef struct {
    int d, window, negative, iter;
    float sample, alpha;        /* -sample; starting -alpha */
    uint64_t train_words;       /* sum of the vertex counts */
    uint32_t vocab_size;
    uint64_t table_size;
    const int32_t *table;       /* dsgl's unigram table (dgo_unigram_table_dsgl) */
    const float *ran;           /* per vocabulary index: sqrtf(r) + r, r = sample * train_words / count */
    const int32_t *v2w;         /* vertex id -> vocabulary index (dsgl's hash2v_vocab) */
    const float *exp_table;
    int device_order;           /* 0: the reference's GEMM order; 1: the device kernel's (split dot, fused chains) */
} dgo_dsgl_cfg;

int dgo_dsgl_ref(const dgo_dsgl_cfg *c, const int32_t *corpus, uint64_t n_tokens, float *wih, float *woh,
                 float *alpha_out, dgo_sgns_stats *st);
void dgo_unigram_table_dsgl(const uint32_t *cn, uint32_t vocab_size, uint64_t table_size, int threads,
                            int32_t *table);

/* FP64 SGNS loss and gradient over explicit minibatches (dg_oracle_adjoint.c). */
int dgo_sgns_loss_grad(const double *in, const double *out, int d, uint32_t vocab_size, const uint32_t *inputs,
                       const uint32_t *outputs, const uint32_t *negatives, uint64_t n_pairs, uint32_t batch,
                       int negative, int only_table, int64_t only_row, double *loss, double *grad_in,
                       double *grad_out);

/* Device graph generator and link-prediction split, restated (dg_oracle_gen.c). */
uint64_t dgo_chung_lu(uint32_t n, uint64_t m, double beta, double cap, uint64_t seed, uint64_t *keys);
float dgo_edge_data(uint64_t key, uint64_t seed, int weighted);
uint64_t dgo_lp_split(uint64_t *keys, uint64_t n, uint32_t v_num, double frac, uint64_t seed, uint32_t *pos_u,
                      uint32_t *pos_v, uint32_t *neg_u, uint32_t *neg_v, uint64_t *n_pos);

#ifdef __cplusplus
}
#endif
#endif
