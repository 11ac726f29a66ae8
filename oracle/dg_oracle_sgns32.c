/*
 * FP32 restatement of both SGNS update rules in the device kernels' operation
 * order, for bit-exact parity of their deterministic mode (one warp / one
 * worker, walks in order).  TEST INFRASTRUCTURE ONLY (see dg_oracle.h).
 *
 * The arithmetic follows word2vec.cu:305-399 (plain) and dsgl.hpp:1084-1407
 * (minibatch) as the FP64 checker in dg_oracle_sgns.c does; what this file adds
 * is the exact FP32 evaluation order of the kernels:
 *  - plain: lane l of a warp holds dimensions [l*v, l*v+v) (v = size/32); a dot
 *    product is a per-lane fused multiply-add chain followed by an xor butterfly
 *    over 16, 8, 4, 2, 1 lanes, lane 0's value used by all; neu1e and the
 *    positive row use fused multiply-adds, negative rows add a rounded g*x;
 *  - minibatch: the row is split into d / 64 contiguous column blocks (one
 *    block for d = 32), each reduced like a plain-rule dot over its block,
 *    block sums added in block order;
 *    output gradients chain over inputs, input gradients over outputs; cache
 *    write-back adds (current - loaded).
 * Compiled with -ffp-contract=off, so only the explicit fmaf calls fuse.
 */
#include "dg_oracle.h"
#include "philox.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define EXP_TABLE_SIZE 1000
#define MAX_EXP 6
#define MB_MAX_SENT 32
#define MB_WIN_TAG 0x4D425749u
#define MB_POOL_TAG 0x4D42504Fu

static uint32_t pword(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed, int word) {
    dgo_u32x4 ctr = {{c0, c1, c2, c3}};
    dgo_u32x4 x = dgo_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    return x.v[word];
}

static uint32_t mix32(uint32_t h) {
    h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
    return h;
}

static float grad32(float f, int label, const float *t, float alpha) {
    if (f > MAX_EXP) return (label - 1) * alpha;
    if (f < -MAX_EXP) return label * alpha;
    return (label - t[(int)((f + MAX_EXP) * (EXP_TABLE_SIZE / MAX_EXP / 2))]) * alpha;
}

static float warp_dot(const float *a, const float *b, int d) {
    const int v = d / 32;
    float p[32], q[32];
    for (int l = 0; l < 32; l++) {
        float s = 0.f;
        for (int i = 0; i < v; i++) s = fmaf(a[l * v + i], b[l * v + i], s);
        p[l] = s;
    }
    for (int o = 16; o; o >>= 1) {
        for (int l = 0; l < 32; l++) q[l] = p[l] + p[l ^ o];
        memcpy(p, q, sizeof(p));
    }
    return p[0];
}

/* Minibatch corr dot: the row's columns are split into nw contiguous blocks of
 * 64 (nw = d / 64; one block for d = 32), one warp each; every block is reduced
 * as warp_dot reduces a row, and the block sums are added in block order. */
static float split_dot(const float *a, const float *b, int d) {
    const int nw = d >= 64 ? d / 64 : 1;
    const int blk = d / nw;
    float f = warp_dot(a, b, blk);
    for (int w = 1; w < nw; w++) f += warp_dot(a + w * blk, b + w * blk, blk);
    return f;
}

int dgo_sgns_plain_f32(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                       float *syn0, float *syn1, dgo_sgns_stats *st) {
    const int d = c->d;
    const float alpha = (float)c->alpha;
    int32_t *sen = (int32_t *)malloc(1024 * sizeof(int32_t));
    float *e = (float *)malloc(d * sizeof(float));
    int32_t tg[65];
    if (!sen || !e || c->negative > 64) { free(sen); free(e); return -2; }
    for (uint32_t w = 0; w < n_walks; w++) {
        uint32_t len = (uint32_t)(offsets[w + 1] - offsets[w]);
        if (len > 1024) len = 1024;
        uint32_t n = 0;
        for (uint32_t i = 0; i < len; i++) {
            int32_t word = c->v2w[verts[offsets[w] + i]];
            if (word < 0) continue;
            if ((pword(i, w, c->pass, DGO_SUB_TAG, c->seed, 0) & 0xFFFFu) >= c->keep_thr[word]) continue;
            sen[n++] = word;
        }
        if (st) { st->words += len; st->trained += n; }
        for (uint32_t p = 0; p < n; p++) {
            const int32_t word = sen[p];
            const uint32_t b = pword(p, w, c->pass, DGO_WIN_TAG, c->seed, 0) % (uint32_t)c->window;
            for (uint32_t a = b; a < (uint32_t)(2 * c->window + 1) - b; a++) {
                if (a == (uint32_t)c->window) continue;
                int64_t cp = (int64_t)p - c->window + a;
                if (cp < 0 || cp >= n) continue;
                if (st) st->pairs++;
                int nt = 0;
                tg[nt++] = word;
                if (c->vocab_size > 1)
                    for (int j = 1; j <= c->negative; j++) {
                        uint32_t r = pword(p * (2 * c->window + 1) + a, w, c->pass,
                                           DGO_NEG_TAG + (uint32_t)((j - 1) >> 2), c->seed, (j - 1) & 3);
                        int32_t t = c->table[r % c->table_size];
                        if (t == 0) t = (int32_t)((r >> 8) % (c->vocab_size - 1) + 1);
                        if (t != word) tg[nt++] = t;
                    }
                /* The pair's arithmetic is word2vec.cu's (dgo_w2v_sg_pair); only the dot
                 * products' order is the warp's. */
                const int n_hs = c->hs ? c->hs_off[word + 1] - c->hs_off[word] : 0;
                dgo_w2v_sg_pair(DGO_ORDER_DEVICE, d, alpha, c->exp_table, syn0 + (size_t)sen[cp] * d,
                                c->hs ? c->hs_point + c->hs_off[word] : NULL,
                                c->hs ? c->hs_code + c->hs_off[word] : NULL, n_hs, tg, nt, syn1, e);
            }
        }
    }
    free(sen); free(e);
    return 0;
}

/* ------------------------------------------------------------ minibatch -- */

/* One sentence of a minibatch worker: its tokens, each token's slot among the
 * sentence's distinct words (first-occurrence order, dsgl.hpp:906-915's
 * sen_words), and the cached input rows of those words (dsgl's inputBuffer)
 * with the values they were loaded with. */
typedef struct {
    int len, pos, ndist, cap;
    int32_t *sen;
    int *slot;
    int32_t *dist;
    float *cache;
    float *init;
} mb32_sentence;

static int mb32_alloc(mb32_sentence *s, int cap, int d) {
    memset(s, 0, sizeof(*s));
    s->cap = cap;
    s->sen = (int32_t *)malloc(cap * sizeof(int32_t));
    s->slot = (int *)malloc(cap * sizeof(int));
    s->dist = (int32_t *)malloc(cap * sizeof(int32_t));
    s->cache = (float *)malloc((size_t)cap * d * sizeof(float));
    s->init = (float *)malloc((size_t)cap * d * sizeof(float));
    return s->sen && s->slot && s->dist && s->cache && s->init ? 0 : -2;
}

static void mb32_release(mb32_sentence *s) {
    free(s->sen); free(s->slot); free(s->dist); free(s->cache); free(s->init);
}

/* Distinct words and their cached input rows (dsgl.hpp:906-925). */
static void mb32_load(mb32_sentence *s, int n, const float *syn0, int d) {
    int nd = 0;
    for (int t = 0; t < n; t++) {
        int r = -1;
        for (int q = 0; q < nd; q++) if (s->dist[q] == s->sen[t]) { r = q; break; }
        if (r < 0) { r = nd; s->dist[nd++] = s->sen[t]; }
        s->slot[t] = r;
    }
    s->len = n <= 1 ? 0 : n;
    s->pos = 0;
    s->ndist = nd;
    if (s->len)
        for (int r = 0; r < nd; r++)
            for (int k = 0; k < d; k++)
                s->cache[r * d + k] = s->init[r * d + k] = syn0[(size_t)s->dist[r] * d + k];
}

/* Write-back of a finished sentence's cached rows: dsgl copies them over the
 * rows (dsgl.hpp:1374-1379, copy != 0); the device kernels add what the sentence
 * changed (copy == 0), so that concurrent workers' updates are kept. */
static void mb32_flush(mb32_sentence *s, float *syn0, int d, int copy) {
    for (int r = 0; r < s->ndist; r++)
        for (int k = 0; k < d; k++) {
            float *x = syn0 + (size_t)s->dist[r] * d + k;
            *x = copy ? s->cache[r * d + k] : *x + (s->cache[r * d + k] - s->init[r * d + k]);
        }
}

/* The shared negatives of one pool and the rows they were loaded with
 * (dsgl.hpp:1049-1080: neg_words, neg_buffer, negativeBuffer). */
typedef struct {
    int np, nbn;
    int32_t *word;  /* distinct words, first-occurrence order */
    int *slot;      /* draw j -> index into word */
    float *cur, *init;
} mb32_pool;

static void mb32_pool_flush(mb32_pool *p, float *syn1, int d, int copy) {
    for (int r = 0; r < p->np; r++)
        for (int k = 0; k < d; k++) {
            float *x = syn1 + (size_t)p->word[r] * d + k;
            *x = copy ? p->cur[(size_t)r * d + k] : *x + (p->cur[(size_t)r * d + k] - p->init[(size_t)r * d + k]);
        }
}

static void mb32_pool_load(mb32_pool *p, const float *syn1, int d) {
    for (int r = 0; r < p->np; r++)
        for (int k = 0; k < d; k++)
            p->cur[(size_t)r * d + k] = p->init[(size_t)r * d + k] = syn1[(size_t)p->word[r] * d + k];
}

/* Adds draw `smp` to the pool (dsgl.hpp:1064-1066). */
static void mb32_pool_add(mb32_pool *p, int j, int32_t smp) {
    int at = -1;
    for (int t = 0; t < p->np; t++) if (p->word[t] == smp) { at = t; break; }
    if (at < 0) { at = p->np; p->word[p->np++] = smp; }
    p->slot[j] = at;
}

/* Arithmetic order of a step.  MB_ORDER_KERNEL: the device kernel's (corr dot by
 * split_dot; dOut and dIn as fused multiply-add chains).  MB_ORDER_GEMM: the
 * reference's three cblas_sgemm calls as the project's naive GEMM stand-in
 * evaluates them (oracle/ref_shim/mkl.h: each element a sum over k in order of
 * rounded products, then alpha = 1 and beta = 0). */
enum { MB_ORDER_KERNEL = 0, MB_ORDER_GEMM = 1 };

static float seq_dot(const float *a, const float *b, int d) {
    float s = 0.f;
    for (int k = 0; k < d; k++) s += a[k] * b[k];
    return s;
}

/* One minibatch step (dsgl.hpp:1084-1359): the inputs are the shrunk-window
 * contexts of both sentences' current positions, the outputs the first centre,
 * the pool's negatives of slot `start` (repeats merged into a multiplicity, a
 * repeat of the first centre dropped), and the second centre; corr = OutM InM^T
 * -> g = (label - sigmoid) * alpha * multiplicity (MKL branch labels:
 * dsgl.hpp:1207-1236), dOut = corr InM, dIn = corr^T OutM; dIn is added to the
 * cached inputs, dOut to both centres' rows directly and to the pool's rows.
 * Returns the number of inputs. */
static int mb32_step(int order, int d, int win, int neg, float alpha, const float *exp_table, uint32_t b,
                     int start, mb32_sentence *S, mb32_pool *P, float *syn1, float *outs, float *gm, float *md) {
    const int MI = 4 * win;
    int in_row[256], out_word[64], out_meta[64], out_slot[64];
    int ni = 0, first = 0;
    for (int s = 0; s < 2; s++) {
        for (int i = (int)b; i < 2 * win + 1 - (int)b; i++) {
            if (i == win) continue;
            int cp = S[s].pos - win + i;
            if (cp < 0) continue;
            if (cp >= S[s].len) break;
            in_row[ni++] = s * 65536 + S[s].slot[cp];
        }
        if (s == 0) first = ni;
    }
    int off = 1;
    out_word[0] = S[0].sen[S[0].pos]; out_meta[0] = 1; out_slot[0] = -1;
    for (int k = 0; k < neg; k++) {
        int ps = P->slot[start * neg + k], smp = P->word[ps], at = -1;
        for (int t = 0; t < off; t++) if (out_word[t] == smp) { at = t; break; }
        if (at < 0) { out_word[off] = smp; out_meta[off] = 1; out_slot[off] = ps; off++; }
        else out_meta[at]++;
    }
    out_meta[0] = 1;
    out_word[off] = S[1].sen[S[1].pos]; out_meta[off] = 1; out_slot[off] = -1;
    const int O = off + 1, I = ni;
    for (int o = 0; o < O; o++)
        for (int k = 0; k < d; k++)
            outs[(size_t)o * d + k] = out_slot[o] < 0 ? syn1[(size_t)out_word[o] * d + k]
                                                      : P->cur[(size_t)out_slot[o] * d + k];
#define ROW(i) (in_row[i] < 65536 ? S[0].cache + (size_t)in_row[i] * d \
                                  : S[1].cache + (size_t)(in_row[i] - 65536) * d)
    for (int o = 0; o < O; o++)
        for (int i = 0; i < I; i++) {
            const float *x = outs + (size_t)o * d, *y = ROW(i);
            const float f = order == MB_ORDER_GEMM ? seq_dot(x, y, d) : split_dot(x, y, d);
            int label = i < first ? (o == 0) : (o == O - 1);
            gm[o * MI + i] = grad32(f, label, exp_table, alpha) * (float)out_meta[o];
        }
    /* Column by column: dOut from the inputs before this step's update, then
     * dIn added to the cached inputs, then dOut added to the outputs.  Columns
     * are independent, so this is the reference's matrix-at-once order. */
    for (int k = 0; k < d; k++) {
        for (int o = 0; o < O; o++) {
            float acc = 0.f;
            if (order == MB_ORDER_GEMM)
                for (int i = 0; i < I; i++) acc += gm[o * MI + i] * ROW(i)[k];
            else
                for (int i = 0; i < I; i++) acc = fmaf(gm[o * MI + i], ROW(i)[k], acc);
            md[o] = acc;
        }
        for (int i = 0; i < I; i++) {
            float acc = 0.f;
            if (order == MB_ORDER_GEMM)
                for (int o = 0; o < O; o++) acc += gm[o * MI + i] * outs[(size_t)o * d + k];
            else
                for (int o = 0; o < O; o++) acc = fmaf(gm[o * MI + i], outs[(size_t)o * d + k], acc);
            ROW(i)[k] = ROW(i)[k] + acc;
        }
        float *t1 = syn1 + (size_t)out_word[0] * d + k, *t2 = syn1 + (size_t)out_word[O - 1] * d + k;
        *t1 = *t1 + md[0];
        *t2 = *t2 + md[O - 1];
        for (int o = 1; o < O - 1; o++) {
            float *x = P->cur + (size_t)out_slot[o] * d + k;
            *x = *x + md[o];
        }
    }
#undef ROW
    return I;
}

typedef struct {
    mb32_sentence S[2];
    mb32_pool P;
    float *outs, *gm, *md;
} mb32_work;

static int mb32_work_alloc(mb32_work *w, int sent_cap, int pool_cap, int d, int neg, int win) {
    memset(w, 0, sizeof(*w));
    int rc = mb32_alloc(&w->S[0], sent_cap, d) | mb32_alloc(&w->S[1], sent_cap, d);
    w->P.word = (int32_t *)malloc(pool_cap * sizeof(int32_t));
    w->P.slot = (int *)malloc(pool_cap * sizeof(int));
    w->P.cur = (float *)malloc((size_t)pool_cap * d * sizeof(float));
    w->P.init = (float *)malloc((size_t)pool_cap * d * sizeof(float));
    w->outs = (float *)malloc((size_t)(neg + 2) * d * sizeof(float));
    w->gm = (float *)malloc((size_t)(neg + 2) * 4 * win * sizeof(float));
    w->md = (float *)malloc((size_t)(neg + 2) * sizeof(float));
    return rc || !w->P.word || !w->P.slot || !w->P.cur || !w->P.init || !w->outs || !w->gm || !w->md ? -2 : 0;
}

static void mb32_work_free(mb32_work *w) {
    mb32_release(&w->S[0]);
    mb32_release(&w->S[1]);
    free(w->P.word); free(w->P.slot); free(w->P.cur); free(w->P.init); free(w->outs); free(w->gm); free(w->md);
}

/* Fills s from the next walks until one has >= 2 kept tokens (dsgl.hpp:903-1028
 * over walks, with the device kernel's Philox subsampling draw). */
static int mb32_fill(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                     uint32_t *next, mb32_sentence *s, const float *syn0, dgo_sgns_stats *st) {
    while (s->len == 0) {
        if (*next >= n_walks) return 0;
        uint32_t w = (*next)++;
        uint32_t len = (uint32_t)(offsets[w + 1] - offsets[w]);
        if (len > MB_MAX_SENT) len = MB_MAX_SENT;
        int n = 0;
        for (uint32_t i = 0; i < len; i++) {
            int32_t word = c->v2w[verts[offsets[w] + i]];
            if (word < 0) continue;
            if ((pword(i, w, c->pass, DGO_SUB_TAG, c->seed, 0) & 0xFFFFu) >= c->keep_thr[word]) continue;
            s->sen[n++] = word;
        }
        if (st) { st->words += len; st->trained += n; }
        mb32_load(s, n, syn0, c->d);
    }
    return 1;
}

/* The device kernel's form of Train_SGNS_MPI (one worker, walks in order):
 * Philox draws, walks as sentences (at most 32 tokens), kernel arithmetic
 * order, write-back of what a sentence / pool changed, and sentences still in
 * flight when the walks run out written back too. */
int dgo_sgns_minibatch_f32(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                           float *syn0, float *syn1, dgo_sgns_stats *st) {
    const int d = c->d, neg = c->negative, win = c->window;
    const float alpha = (float)c->alpha;
    if (d > 512) return -1;
    const uint32_t key0 = (uint32_t)c->seed ^ mix32(c->pass * 0x9E3779B9u + 0x632BE5ABu);
    const uint64_t mbseed = ((uint64_t)(uint32_t)(c->seed >> 32) << 32) | key0;
    mb32_work W;
    if (mb32_work_alloc(&W, MB_MAX_SENT, MB_MAX_SENT * (neg > 0 ? neg : 1), d, neg, win)) {
        mb32_work_free(&W);
        return -2;
    }
    mb32_sentence *S = W.S;
    mb32_pool *P = &W.P;
    uint32_t next = 0, step = 0, pool_no = 0, neg_count = 0;
    int train_sen_num = 0, change_neg = 1, pool_loaded = 0;
    P->np = 0;
    P->nbn = 1;
    for (;;) {
        int ok0 = mb32_fill(c, offsets, verts, n_walks, &next, &S[0], syn0, st);
        int ok1 = ok0 ? mb32_fill(c, offsets, verts, n_walks, &next, &S[1], syn0, st) : 0;
        if (!ok0 || !ok1) break;
        if (change_neg) {
            P->nbn = S[0].len > S[1].len ? S[0].len : S[1].len;
            P->np = 0;
            for (int j = 0; j < P->nbn * neg; j++) {
                uint32_t r = pword((uint32_t)j >> 2, pool_no, 0, MB_POOL_TAG, mbseed, j & 3);
                int32_t smp = c->table[r % c->table_size];
                if (!smp) smp = c->vocab_size > 1 ? (int32_t)((r >> 8) % (c->vocab_size - 1) + 1) : 0;
                mb32_pool_add(P, j, smp);
            }
            mb32_pool_load(P, syn1, d);
            pool_no++;
            change_neg = 0;
            pool_loaded = 1;
        }
        const uint32_t b = pword(step, 0, 0, MB_WIN_TAG, mbseed, 0) % (uint32_t)win;
        neg_count++;
        const int I = mb32_step(MB_ORDER_KERNEL, d, win, neg, alpha, c->exp_table, b,
                                (int)(neg_count % (uint32_t)P->nbn), S, P, syn1, W.outs, W.gm, W.md);
        if (st) st->pairs += I;
        step++;
        S[0].pos++;
        S[1].pos++;
        for (int s = 0; s < 2; s++)
            if (S[s].pos >= S[s].len) { mb32_flush(&S[s], syn0, d, 0); S[s].len = 0; train_sen_num++; }
        if (train_sen_num >= 2) {
            mb32_pool_flush(P, syn1, d, 0);
            change_neg = 1;
            pool_loaded = 0;
            train_sen_num = 0;
        }
    }
    for (int s = 0; s < 2; s++) if (S[s].len) mb32_flush(&S[s], syn0, d, 0);
    if (pool_loaded) mb32_pool_flush(P, syn1, d, 0);
    mb32_work_free(&W);
    return 0;
}

/* ------------------------------------------- dsgl reference-stream mode -- */

#define DSGL_MAX_SENTENCE 1000 /* MAX_SENTENCE_LENGTH, dsgl.hpp:23 */

static unsigned long long dsgl_lcg(unsigned long long *nr) {
    *nr = *nr * (unsigned long long)25214903917ULL + 11;
    return *nr;
}

/* Reads one sentence of the compute thread's corpus slice (dsgl.hpp:903-937 /
 * 967-999): tokens up to a walk end (-1), the slice end or 1000 kept tokens;
 * the token that reaches the slice end is not kept; each token takes one LCG
 * draw and is discarded iff ran[w] < (draw & 0xFFFF) / 65536. */
static int dsgl_read(const dgo_dsgl_cfg *c, const int32_t *corpus, uint64_t end, uint64_t *cur,
                     unsigned long long *word_count, unsigned long long *nr, int32_t *sen) {
    int n = 0;
    for (;;) {
        const int32_t id = corpus[*cur];
        (*word_count)++;
        (*cur)++;
        if (id == -1 || *cur >= end) break;
        const int32_t w = c->v2w[id];
        if (c->sample > 0) {
            dsgl_lcg(nr);
            if (c->ran[w] < (float)(*nr & 0xFFFF) / 65536.f) continue;
        }
        sen[n++] = w;
        if (n >= DSGL_MAX_SENTENCE) break;
    }
    return n;
}

/* Train_SGNS_MPI's compute thread (dsgl.hpp:770-1407, MKL branch) at one rank
 * with one compute thread (-threads 2), followed literally: its LCG stream
 * seeded with the thread index 0 (dsgl.hpp:780) for subsampling, pools and
 * window shrinks, in the order the thread draws them; sentences from the token
 * stream; the linear learning-rate decay every 10,000 tokens (dsgl.hpp:889-897);
 * the reference's three GEMMs in the stand-in's order (MB_ORDER_GEMM); cached
 * rows and pools copied back (copy write-back); the sentences in flight when
 * the slice ends dropped (dsgl.hpp:1029-1045).  The step itself is mb32_step,
 * the one the device kernel's restatement uses.  wih / woh are the vocabulary-
 * order rows; *alpha_out gets the learning rate at the end. */
int dgo_dsgl_ref(const dgo_dsgl_cfg *c, const int32_t *corpus, uint64_t n_tokens, float *wih, float *woh,
                 float *alpha_out, dgo_sgns_stats *st) {
    const int d = c->d, neg = c->negative, win = c->window;
    if (d > 4096 || win < 1 || neg < 0 || n_tokens == 0) return -1;
    mb32_work W;
    const int pool_cap = DSGL_MAX_SENTENCE * (neg > 0 ? neg : 1);
    if (mb32_work_alloc(&W, DSGL_MAX_SENTENCE, pool_cap, d, neg, win)) {
        mb32_work_free(&W);
        return -2;
    }
    mb32_sentence *S = W.S;
    mb32_pool *P = &W.P;
    const float starting_alpha = c->alpha;
    float alpha = c->alpha;
    unsigned long long nr = 0, word_count = 0, last_word_count = 0, word_count_actual = 0;
    const uint64_t end = n_tokens;
    uint64_t cur = 0;
    int local_iter = c->iter, train_sen_num = 0, change_neg = 1;
    unsigned long long neg_count = 0;
    S[0].len = S[1].len = 0;
    for (;;) {
        if (word_count - last_word_count > 10000) {
            word_count_actual += word_count - last_word_count;
            last_word_count = word_count;
            alpha = starting_alpha * (1 - word_count_actual * 1ull / (float)(c->iter * c->train_words + 1));
            if (alpha < starting_alpha * 0.0001f) alpha = starting_alpha * 0.0001f;
        }
        for (int s = 0; s < 2; s++) {
            while (S[s].len == 0) {
                if (cur >= end) break;
                const int n = dsgl_read(c, corpus, end, &cur, &word_count, &nr, S[s].sen);
                if (st) st->trained += n;
                if (n <= 1) { S[s].len = 0; continue; }
                mb32_load(&S[s], n, wih, d);
            }
        }
        if (cur >= end) {
            word_count_actual += word_count - last_word_count;
            if (--local_iter == 0) break;
            word_count = 0;
            cur = 0;
            last_word_count = 0;
            S[0].len = S[1].len = 0;
            continue;
        }
        if (change_neg) {
            P->nbn = S[0].len > S[1].len ? S[0].len : S[1].len;
            P->np = 0;
            for (int j = 0; j < P->nbn * neg; j++) {
                dsgl_lcg(&nr);
                int32_t smp = c->table[(nr >> 16) % c->table_size];
                if (!smp) smp = (int32_t)(nr % (c->vocab_size - 1) + 1);
                mb32_pool_add(P, j, smp);
            }
            mb32_pool_load(P, woh, d);
            change_neg = 0;
        }
        dsgl_lcg(&nr);
        const uint32_t b = (uint32_t)(nr % (unsigned long long)win);
        neg_count++;
        const int I = mb32_step(c->device_order ? MB_ORDER_KERNEL : MB_ORDER_GEMM, d, win, neg, alpha, c->exp_table, b,
                                (int)(neg_count % (unsigned long long)P->nbn), S, P, woh, W.outs, W.gm, W.md);
        if (st) st->pairs += I;
        S[0].pos++;
        S[1].pos++;
        for (int s = 0; s < 2; s++)
            if (S[s].pos >= S[s].len) { mb32_flush(&S[s], wih, d, 1); S[s].len = 0; train_sen_num++; }
        if (train_sen_num >= 2) {
            mb32_pool_flush(P, woh, d, 1);
            change_neg = 1;
            train_sen_num = 0;
        }
    }
    if (st) st->words += word_count_actual;
    if (alpha_out) *alpha_out = alpha;
    mb32_work_free(&W);
    return 0;
}

/* InitUnigramTable of dsgl (dsgl.hpp:120-146): FP32 running share d1, the
 * index clamped before its share is added, and the power sum as its two-thread
 * OpenMP reduction forms it (iterations [0, ceil(n/2)) and the rest, summed
 * separately, then added). */
void dgo_unigram_table_dsgl(const uint32_t *cn, uint32_t vocab_size, uint64_t table_size, int threads,
                            int32_t *table) {
    double sum = 0.0;
    if (threads < 1) threads = 1;
    const uint32_t chunk = (vocab_size + (uint32_t)threads - 1) / (uint32_t)threads;
    for (int t = 0; t < threads; t++) {
        double part = 0.0;
        for (uint32_t i = (uint32_t)t * chunk; i < vocab_size && i < (uint32_t)(t + 1) * chunk; i++)
            part += pow((double)cn[i], (double)0.75f);
        sum += part;
    }
    uint32_t i = 0;
    float d1 = (float)(pow((double)cn[0], (double)0.75f) / sum);
    for (uint64_t a = 0; a < table_size; a++) {
        table[a] = (int32_t)i;
        if ((float)a / (float)table_size > d1) {
            i++;
            if (i >= vocab_size) i = vocab_size - 1;
            d1 = (float)((double)d1 + pow((double)cn[i], (double)0.75f) / sum);
        }
    }
}
