/*
 * distger: B200 (sm_100a) implementation of DistGER's embedding hot path --
 * the information-oriented random walk and the skip-gram negative-sampling
 * (SGNS) trainer -- behind a plain C ABI.
 *
 * Conventions: every entry point returns 0 (DG_OK) or a negative DG_ERR_* code
 * and never exits the process; dg_last_error() gives the message of the calling
 * thread's last failure.  Handles own their device memory and one CUDA stream;
 * a handle is not thread-safe.  Host buffers are plain pointers with sizes.
 *
 * Reference interfaces replaced (paths within the reference project):
 *  - graph load + CSR:  GraphEngine::load_graph, include/graph.hpp:642-824,
 *                       read_graph, include/storage.hpp:15-37
 *  - walk rounds:       WalkEngine::random_walk / internal_random_walk,
 *                       include/walk.hpp:512, 609-782; internal_walk_epoch 790-1043
 *  - walk output:       PathCollector::assemble_path + PathSet::dump,
 *                       include/path.hpp:175-551, 67-119
 *  - SGNS trainer:      train_corpus_cuda / TrainModel / TrainModelThread,
 *                       src/word2vec.cu:1429, 1246, 952; dsgl(), include/dsgl.hpp:1464
 *  - LR schedule:       include/lr_scheduler.hpp:5-74
 */
#ifndef DISTGER_H
#define DISTGER_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define DG_API __attribute__((visibility("default")))
#else
#define DG_API
#endif

#define DG_OK 0
#define DG_ERR_ARG -1        /* invalid argument or size */
#define DG_ERR_IO -2         /* file missing, unreadable or malformed */
#define DG_ERR_CUDA -3       /* CUDA runtime error (message has the CUDA string) */
#define DG_ERR_NOMEM -4      /* host or device allocation failed */
#define DG_ERR_OVERFLOW -5   /* a walk outgrew its arena slot; rerun with larger max_len */
#define DG_ERR_STATE -6      /* call out of order (e.g. no paths yet) */

typedef struct dg_graph dg_graph;
typedef struct dg_paths dg_paths;
typedef struct dg_sgns dg_sgns;

/* Message of the calling thread's last failed call ("" if none). */
DG_API const char *dg_last_error(void);

/* Library build identity: "distger <version> sm_100a". */
DG_API const char *dg_version(void);

/* ------------------------------------------------------------------ graph */

/* Loads packed 12-byte {u32 src, u32 dst, f32 data} records (storage.hpp:15-37,
 * type.hpp:67-91), optionally makes them undirected by emitting each record and
 * its transpose (graph.hpp:671-686), and builds the device CSR: int64 row
 * offsets, 8-byte entries {u32 neighbour, u32 acceptance threshold}.  Vertex ids
 * >= v_num and edge data that is NaN or outside int range are DG_ERR_ARG;
 * a file whose size is not a multiple of 12 is DG_ERR_IO. */
DG_API int dg_graph_create(const char *edge_path, uint32_t v_num, int undirected, int device, dg_graph **out);

/* Same from host records already in memory (n_edges records of 12 bytes). */
DG_API int dg_graph_create_from_edges(const void *edges, uint64_t n_edges, uint32_t v_num, int undirected,
                               int device, dg_graph **out);

DG_API void dg_graph_free(dg_graph *g);

typedef struct {
    uint32_t v_num;
    uint64_t m;               /* directed CSR entries */
    uint64_t device_bytes;    /* device memory held by the graph */
    double threshold_ms;      /* acceptance-threshold kernel time */
} dg_graph_info;
DG_API int dg_graph_get_info(const dg_graph *g, dg_graph_info *info);

/* Copies the CSR to host buffers (each may be NULL): offsets[v_num+1],
 * neighbours[m], thresholds[m], out_degree[v_num], in_degree[v_num]. */
DG_API int dg_graph_copy_csr(const dg_graph *g, uint64_t *offsets, uint32_t *neighbours, uint32_t *thresholds,
                      uint32_t *out_degree, uint32_t *in_degree);

/* ------------------------------------------------------------------ walks */

typedef struct {
    uint32_t min_len;     /* --min_L: no termination test until step > min_len (walk.hpp:404, 868) */
    uint32_t init_round;  /* --min_R: round 1 runs walker_num * init_round walkers (walk.hpp:614) */
    uint32_t walker_num;  /* -w */
    uint32_t max_len;     /* arena slot, in footprints; 0 = 64.  Longer walks are DG_ERR_OVERFLOW */
    uint64_t seed;        /* Philox key for seeded replay */
} dg_walk_params;

typedef struct {
    uint32_t n_walks;
    uint64_t footprints;  /* all footprints, start vertices included */
    uint64_t steps;       /* footprints with step >= 1 (the reference's p_step counter) */
    uint64_t draws;       /* candidate draws */
    uint64_t traces;      /* rejected candidates (walk.hpp trace_num) */
    uint32_t max_len;     /* longest walk, footprints */
    double walk_ms;       /* walk kernel time (CUDA events) */
    double relative_entropy; /* after this round's visits are counted (walk.hpp:694-725) */
    double delta_h;          /* change vs the previous round (walk.hpp:727-728) */
} dg_round_info;

/* Runs one round: walkers 0..n-1 start at id % v_num (walk.hpp:501-509) with
 * n = walker_num * init_round for round 1, walker_num otherwise (n_walkers != 0
 * overrides).  The walks stay on the device in *out; the graph's cumulative
 * visit frequencies (context_map_freq, walk.hpp:645, 688) are updated.
 * Seeded replay: identical (seed, round, walker) give identical walks. */
DG_API int dg_walk_run_round(dg_graph *g, const dg_walk_params *p, uint32_t round, uint32_t n_walkers,
                      dg_paths **out);

DG_API int dg_paths_get_info(const dg_paths *paths, dg_round_info *info);

/* Copies walks in walker order: offsets[n_walks+1] (footprint offsets) and
 * vertices[footprints] (either may be NULL).  The walks are compacted on the
 * device into buffers the graph keeps for later calls. */
DG_API int dg_paths_copy(const dg_paths *paths, uint64_t *offsets, uint32_t *vertices);

/* Writes the walk file: per walk " %u" per vertex then "\n" (path.hpp:92,108).
 * The text is formatted on the device. */
DG_API int dg_paths_write_text(const dg_paths *paths, const char *file_path);

/* Frees the walks; call it before dg_graph_free of their graph.  The graph keeps
 * the largest freed walk arena and reuses it for its next round. */
DG_API void dg_paths_free(dg_paths *paths);

/* Cumulative visit frequency per vertex over all rounds run on g. */
DG_API int dg_graph_copy_visits(const dg_graph *g, uint32_t *freq);

/* ------------------------------------------------------------------- SGNS */

enum {
    DG_SGNS_PLAIN = 0,      /* word2vec.cu skip_gram_kernel semantics: FP32 rows, per-pair negatives, Hogwild */
    DG_SGNS_MINIBATCH = 1,  /* dsgl.hpp Train_SGNS_MPI semantics: shared negatives, BF16 rows, FP32 accumulation */
    DG_SGNS_PLAIN_BF16 = 2, /* the plain (word2vec.cu) rule on BF16 rows: FP32 arithmetic, FP32 master rows for
                               the hottest words (atomics), stochastic rounding for the rest; negative <= 8,
                               size 64, 128 or 256 */
    DG_SGNS_CBOW = 3,       /* word2vec.cu cbow_kernel semantics (the reference's default, -cbow 1): FP32 rows,
                               the mean of the window's context rows against the centre and per-centre
                               negatives; negative <= 32 */
    DG_SGNS_SG_SHARED = 4,  /* word2vec.cu __sgNegReuse semantics (-cbow 0 -reuse-neg 1): FP32 rows, one negative
                               set per walk, the full window; negative <= 16.  Every supported size (the
                               reference builds only 200 and 300) */
    DG_SGNS_CBOW_BF16 = 5,  /* DG_SGNS_CBOW's rule on BF16 rows: FP32 arithmetic, FP32 master rows for the
                               master_rows most frequent words, stochastic rounding of every BF16 row write;
                               size 64, 128 or 256, negative <= 32, no hierarchical softmax */
};

typedef struct {
    int size;          /* -size: embedding dimension: 32, 64, 128, 256 or 512; the FP32 word2vec rules
                          (DG_SGNS_PLAIN, _CBOW, _SG_SHARED, not in adjoint mode) take any size up to 512
                          (e.g. the reference's run.sh uses 100), stored padded to the next of those */
    int window;        /* -window */
    int negative;      /* -negative */
    int batch_size;    /* -batch-size (minibatch mode; dsgl overrides it with 2*window+1, dsgl.hpp:832) */
    float sample;      /* -sample */
    float alpha;       /* -alpha */
    int iter;          /* -iter: passes over each round's walks */
    int min_count;     /* -min-count */
    int mode;          /* DG_SGNS_* */
    int deterministic; /* 0: Hogwild (fused updates, many workers);
                          1: one warp / one worker trains everything in order (tests, replay);
                          2: adjoint mode -- the plain trainer's pairs of each pass, in minibatches of
                             batch_size pairs (0: 2*window+1) sharing `negative` (<= 16) negatives,
                             trained by gradient steps of the hand-written backward kernel
                             (dg_sgns_adjoint_step's rule); identical results at any GPU occupancy */
    uint64_t seed;
    uint64_t table_size; /* unigram table slots; 0 = 1e8 (word2vec.cu:66) */
    uint32_t master_rows; /* minibatch mode: hottest rows kept in FP32; 0 = 65536, >= vocabulary = all */
    uint32_t workers;     /* concurrent trainer workers (warps in plain mode, CTAs in minibatch mode);
                             0 = automatic; capped at what the GPU holds resident.  Adjoint mode:
                             minibatches per gradient step (0 = automatic bound) */
    int hs;               /* -hs 1: hierarchical softmax over word2vec's Huffman coding of the vocabulary
                             (CreateBinaryTree, word2vec.cu:684-740) before the negative-sampling
                             targets, in DG_SGNS_PLAIN and DG_SGNS_CBOW (word2vec.cu:334-356, 436-455;
                             inner nodes share the output rows with the words, as in the reference);
                             no effect on DG_SGNS_SG_SHARED, as __sgNegReuse has no HS branch;
                             not available in the BF16, minibatch or adjoint forms */
} dg_sgns_params;

/* Vocabulary from per-vertex counts (word2vec.cu:791-809 uses in+out degree,
 * dsgl.hpp:307-352 uses walk visit counts): sorted by count, descending, ties by
 * vertex id; counts < min_count dropped except the first (word2vec.cu:632-659).
 * Input rows initialised with word2vec's LCG (word2vec.cu:870-873), output rows
 * zero; unigram^0.75 table (word2vec.cu:537-556). */
DG_API int dg_sgns_create(const dg_sgns_params *p, uint32_t v_num, const uint32_t *vertex_counts, int device,
                   dg_sgns **out);
DG_API void dg_sgns_free(dg_sgns *s);

typedef struct {
    uint64_t words;      /* tokens consumed, subsampled ones included (word2vec.cu word_count) */
    uint64_t trained;    /* tokens kept after subsampling */
    uint64_t pairs;      /* (centre, context) pairs */
    double train_ms;     /* SGNS kernel time */
    uint64_t rows;       /* minibatch form: input + output rows of every minibatch step, summed
                            (dsgl.hpp:1089-1160); 0 for the other forms */
} dg_train_info;

/* One pass (x iter) over a round's walks with learning rate alpha (alpha <= 0:
 * the params' alpha). */
DG_API int dg_sgns_train_paths(dg_sgns *s, const dg_paths *paths, float alpha, dg_train_info *info);

/* Same over host walks in walker order (offsets[n_walks+1], vertices[...]). */
DG_API int dg_sgns_train_host(dg_sgns *s, const uint64_t *offsets, uint32_t n_walks, const uint32_t *vertices,
                       float alpha, dg_train_info *info);

/* Input rows (the embedding) as FP32, in vocabulary order; vocab_ids[rows]
 * gives the vertex of each row.  Either pointer may be NULL. */
DG_API int dg_sgns_copy_embedding(const dg_sgns *s, float *rows, uint32_t *vocab_ids, uint32_t *n_rows);
DG_API int dg_sgns_copy_output(const dg_sgns *s, float *rows);

/* The trainer's lookup tables (each may be NULL): unigram table[table_size],
 * subsampling keep thresholds[vocabulary] (a token is kept iff 16 random bits
 * are below it), vertex -> vocabulary row map[v_num] (-1 = not in vocabulary),
 * expTable[1001]. */
DG_API int dg_sgns_copy_tables(const dg_sgns *s, int32_t *table, uint32_t *keep_thr, int32_t *v2w,
                               float *exp_table);

typedef struct {
    uint32_t vocab_size;
    uint32_t master_rows;  /* rows held in FP32 (minibatch form) */
    uint32_t workers;      /* worker bound: the params' workers, else (minibatch form) the automatic
                              staleness bound; 0 = as many as the GPU holds */
    uint64_t train_words;  /* sum of the vocabulary counts */
    uint64_t table_size;
    uint64_t device_bytes;
    int32_t bf_staged;     /* BF16 plain mode: 1 if the default launch shape stages BF16 rows in shared
                              memory (only when concurrent writers of one BF16 row are rare) */
} dg_sgns_info;
DG_API int dg_sgns_get_info(const dg_sgns *s, dg_sgns_info *info);
DG_API int dg_sgns_set_rows(dg_sgns *s, const float *input_rows, const float *output_rows);

/* Embedding text: "%lld %lld\n" header then per row "%u " + size x "%lf " + "\n"
 * (word2vec.cu:1353-1362). */
DG_API int dg_sgns_write_embedding(const dg_sgns *s, const char *file_path);

/* ------------------------------------------------------ common neighbours */

/* Common-neighbour count of every edge, the edge data the HuGE transition reads
 * (walk.hpp:920): replaces the reference's gcn tool (src/tools/gcn.cpp:249-373),
 * computed on the device.  Rows are the CSR of the edges (both directions when
 * undirected) sorted by neighbour, duplicates kept; for edge (s, d) the count is
 * taken over the elements of the shorter row (N(s) on a tie) found in the other
 * row, less one if the first is s or d and, when more than one remains, less one
 * per later element that repeats its predecessor or is s or d (gcn.cpp:327-343);
 * repeated pairs report the value of their first occurrence's orientation.  An
 * empty row gives 0 (the tool reads past an empty row, directed inputs only).
 * cn[n_edges] receives the counts in input order. */
DG_API int dg_common_neighbours(const uint32_t *src, const uint32_t *dst, uint64_t n_edges, uint32_t v_num,
                                int undirected, int device, int32_t *cn);

/* ------------------------- synthetic graphs and link prediction on device */

/* The reference reads graphs from 12-byte edge files (storage.hpp:15-37) and
 * splits them for link prediction on the host (src/tools/gtrain.cpp:226-386).
 * These entry points generate, split, build and score on the device, for graphs
 * too large for host tools (the Twitter-shaped workload: 41.6M vertices, 1.47B
 * edges). */
typedef struct {
    uint32_t n;          /* vertices */
    uint64_t m;          /* edge draws; self-loops and repeated pairs are dropped, isolated vertices get one edge */
    double beta;         /* expected degrees proportional to (i + 1)^(-1/(beta - 1)) */
    double max_degree;   /* cap on the expected degree (0: none) */
    uint64_t seed;
    int weighted;        /* 1: edge data uniform (0, 1]; 0: 1.0 */
} dg_chung_lu_params;

typedef struct dg_edges dg_edges;       /* undirected edge list on the device (unique pairs) */
typedef struct dg_lp_pairs dg_lp_pairs; /* link-prediction test pairs on the device */

/* Chung-Lu edge-sampling graph (deterministic in the seed). */
DG_API int dg_edges_chung_lu(const dg_chung_lu_params *p, int device, dg_edges **out);
DG_API int dg_edges_get_info(const dg_edges *e, uint32_t *v_num, uint64_t *n_edges);
/* Host copy, pairs in ascending (src, dst) order with src < dst (each may be NULL). */
DG_API int dg_edges_copy(const dg_edges *e, uint32_t *src, uint32_t *dst, float *data);
DG_API void dg_edges_free(dg_edges *e);

/* Holds out about frac of the edges (gtrain's rule in a parallel form: a
 * hash-selected candidate stays in the graph when removing it would leave one of
 * its endpoints without an edge) plus as many uniform non-edges of the full
 * graph; the held-out edges leave `e`.  Test pairs: positives, then negatives. */
DG_API int dg_edges_split(dg_edges *e, double frac, uint64_t seed, dg_lp_pairs **test);
DG_API int dg_lp_pairs_get_info(const dg_lp_pairs *t, uint64_t *n_pos, uint64_t *n_neg);
DG_API int dg_lp_pairs_copy(const dg_lp_pairs *t, uint32_t *u, uint32_t *v, uint8_t *label);
DG_API void dg_lp_pairs_free(dg_lp_pairs *t);

/* Undirected CSR of a device edge list, built on the device (both directions of
 * every pair, rows sorted by neighbour, thresholds as for dg_graph_create). */
DG_API int dg_graph_create_from_device_edges(const dg_edges *e, dg_graph **out);

/* Link-prediction AUC of the trainer's input embedding on the test pairs: score
 * sigmoid(v_u . v_v) (and cosine), Mann-Whitney AUC with ties averaged. */
DG_API int dg_lp_auc(const dg_sgns *s, const dg_lp_pairs *t, double *auc, double *auc_cosine);

/* -------------------------------------------------------------- autotuner */

/* No counterpart in the reference (its kernels have fixed launches).  Each
 * kernel with a choice of launch shapes is timed on live data, every shape
 * twice (the second run is kept), and the fastest shape is kept by the handle
 * for later calls.  Results never depend on the shape: walks are keyed by
 * walker id, and the plain trainer's Hogwild updates depend on scheduling
 * under every shape alike. */
#define DG_TUNE_MAX 16
typedef struct {
    int n_candidates;
    int chosen;                /* index of the shape kept */
    int shape[DG_TUNE_MAX][3]; /* walks: {walks per block, footprints cached in shared memory per walk, 0};
                                  plain SGNS: {threads per block, blocks per SM: 0 = as many as fit,
                                  else that many (a cap, or the count the kernel's registers
                                  are limited to fit), pairs whose rows are staged in shared
                                  memory (0: rows loaded when the pair starts)} */
    double ms[DG_TUNE_MAX];    /* kernel time of each candidate (CUDA events) */
} dg_tune_info;

/* Times walk_kernel's launch shapes on n_walkers (0: walker_num) walkers of
 * `round`; the trial rounds' visit counts are rolled back and no round is
 * recorded. */
DG_API int dg_walk_autotune(dg_graph *g, const dg_walk_params *p, uint32_t round, uint32_t n_walkers,
                            dg_tune_info *info);
DG_API int dg_walk_set_shape(dg_graph *g, int shape);

/* Times the plain trainer's launch shapes on these walks; rows and the pass
 * counter are restored after every trial. */
DG_API int dg_sgns_autotune(dg_sgns *s, const dg_paths *paths, dg_tune_info *info);
DG_API int dg_sgns_set_shape(dg_sgns *s, int shape);

/* ------------------------------------------------- SGNS loss and adjoint */

/* Explicit minibatches for the loss / gradient entry points: n_pairs (input,
 * output) pairs in minibatches of `batch` consecutive pairs (the last one may be
 * shorter), each minibatch sharing `negative` negative output rows -- dsgl's
 * shared-negative minibatch (dsgl.hpp:1055-1156; batch 2*window+1 = 21).  Ids
 * are vocabulary rows (0 .. vocab_size-1).  Host pointers. */
typedef struct {
    const uint32_t *inputs;     /* [n_pairs] input rows (the context word of a pair) */
    const uint32_t *outputs;    /* [n_pairs] positive output rows (the centre word) */
    const uint32_t *negatives;  /* [ceil(n_pairs / batch) * negative] */
    uint64_t n_pairs;
    uint32_t batch;             /* >= 1 */
    int negative;               /* 0 .. 16 */
} dg_sgns_pairs;

/* The SGNS loss that word2vec.cu's skip_gram_kernel (word2vec.cu:305-399) and
 * dsgl's minibatch update (dsgl.hpp:1241-1311) descend with fused Hogwild
 * updates, evaluated at the trainer's current rows (FP32 rows in plain mode,
 * BF16 rows + FP32 masters in minibatch mode):
 *   L = sum_pairs softplus(-v_in . u_out) + sum_{minibatch negatives k} softplus(v_in . u_k)
 * with the exact logistic sigmoid, and its gradient by a hand-written backward
 * kernel.  loss: FP64 sum; grad_in / grad_out: vocab_size x size FP32 in
 * vocabulary order (each may be NULL).  Deterministic: contributions are summed
 * in 64-bit fixed point (2^-40 resolution), so equal inputs give bit-identical
 * gradients whatever the thread schedule.  A contribution that is not finite or
 * reaches 2^20 in magnitude is DG_ERR_ARG. */
DG_API int dg_sgns_loss_grad(dg_sgns *s, const dg_sgns_pairs *pairs, double *loss, float *grad_in, float *grad_out);

/* The deterministic training step that replaces the fused update: the gradient
 * above at the current rows, then rows -= alpha * gradient for both tables,
 * rounded to nearest in the rows' storage.  loss (may be NULL) is the loss
 * before the step. */
DG_API int dg_sgns_adjoint_step(dg_sgns *s, const dg_sgns_pairs *pairs, float alpha, double *loss);

/* --------------------------------------------------------------- pipeline */

typedef struct {
    dg_round_info walk;
    dg_train_info train;
    double total_ms;   /* device time from the walk launch to the end of training (CUDA events) */
} dg_pipeline_info;

/* One round streamed straight into the trainer: dg_walk_run_round followed by
 * dg_sgns_train_paths on the device-resident walks, ordered on the device (no
 * host copy of the walks).  The walks are freed unless keep is non-NULL, in
 * which case *keep receives them. */
DG_API int dg_pipeline_round(dg_graph *g, dg_sgns *s, const dg_walk_params *p, uint32_t round, uint32_t n_walkers,
                             float alpha, dg_pipeline_info *info, dg_paths **keep);

/* Number of kernels this library has launched in the process so far. */
DG_API uint64_t dg_launch_count(void);

/* ------------------------------------------------ allocation-free trainer */

/* Arguments of dg_sgns_minibatch_train_noalloc: every pointer is device memory
 * owned by the caller.  Tables and rows have the layouts dg_sgns_copy_tables
 * and dg_sgns_copy_embedding describe; rows are updated in place. */
typedef struct {
    const uint32_t *verts;     /* walk vertices */
    const uint64_t *offsets;   /* n_walks + 1 offsets into verts */
    uint32_t n_walks;
    const int32_t *v2w;        /* vertex -> vocabulary row, -1 = skipped */
    const uint32_t *keep_thr;  /* subsampling keep thresholds per vocabulary row */
    const int32_t *table;      /* unigram table */
    uint64_t table_size;
    const float *exp_table;    /* 1001 sigmoid entries */
    uint32_t vocab_size;
    uint16_t *in_bf16;         /* vocab_size x size input rows, BF16 bits */
    uint16_t *out_bf16;        /* vocab_size x size output rows, BF16 bits */
    float *in_master;          /* n_master x size FP32 input rows (rows 0..n_master-1) */
    float *out_master;         /* n_master x size FP32 output rows */
    uint32_t n_master;
    int size;                  /* 32, 64, 128 or 256 */
    int window, negative;      /* window <= 64, negative <= 14 */
    float alpha;
    uint64_t seed;
    uint32_t pass;             /* pass counter: one value per call, as dg_sgns_train_* count them */
    int deterministic;         /* 1: one worker, walks in order */
    uint32_t workers;          /* concurrent workers (Hogwild); 0 = 128 (see below).  dg_sgns_get_info
                                  reports the staleness bound the handle path applies to a vocabulary */
} dg_sgns_minibatch_args;

/* No counterpart in the reference.  The minibatch trainer (DG_SGNS_MINIBATCH)
 * with no allocation at all, for callers that cannot call cudaMalloc: a host
 * framework whose memory pool owns the device memory and forbids foreign
 * allocations, or a latency-bound loop that cannot pay cudaMalloc / cudaFree
 * (which can synchronise the device) or handle an allocation failure mid-run.
 * Its per-worker scratch (negative pools, cache snapshots) lives in a 16 MiB
 * device array that is part of this library and is held by every GPU that loads
 * it until the process exits; sizes whose per-worker scratch exceeds it are
 * DG_ERR_ARG, and the number of parallel workers is capped by it.  The first call
 * on a device looks up the array's device address, so make that first call
 * before any stream capture.  Every call shares the array: calls whose work
 * overlaps on the GPU (other streams, other threads) race and must not be
 * issued.  stream is a cudaStream_t (NULL = legacy default stream) of the
 * current device (another device's stream is DG_ERR_ARG).  Hogwild workers: the
 * args' workers, capped by the array; 0 = 128, a staleness bound that holds for
 * any vocabulary (the handle path's own bound, larger for most vocabularies, is
 * dg_sgns_info.workers).  With info non-NULL the call waits for the stream to
 * finish (cudaStreamSynchronize) and reports the counters (train_ms = 0); with
 * info NULL it only enqueues work. */
DG_API int dg_sgns_minibatch_train_noalloc(const dg_sgns_minibatch_args *args, void *stream, dg_train_info *info);

#ifdef __cplusplus
}
#endif
#endif
