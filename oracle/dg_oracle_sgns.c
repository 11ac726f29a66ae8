/*
 * CPU restatement of the SGNS trainer.  TEST INFRASTRUCTURE ONLY (see
 * dg_oracle.h).  Rows are kept in FP64 so that the device's FP32 / BF16 error can
 * be stated against it; the order of every update follows the cited reference
 * lines, and the random choices use the same Philox counters as the device code.
 */
#include "dg_oracle.h"
#include "philox.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define EXP_TABLE_SIZE 1000 /* word2vec.cu:29 */
#define MAX_EXP 6           /* word2vec.cu:30 */

/* ---------------------------------------------------------------- vocab -- */

typedef struct { uint32_t cn, id; } vv;

static int vv_cmp(const void *a, const void *b) {
    const vv *x = (const vv *)a, *y = (const vv *)b;
    if (x->cn != y->cn) return x->cn > y->cn ? -1 : 1;
    return x->id < y->id ? -1 : (x->id > y->id);
}

/* ReadVocabFromDegree + SortVocab (word2vec.cu:791-809, 632-659): one word per
 * vertex with its count, sorted by count descending (ties: vertex id, where
 * qsort leaves the order unspecified), counts < min_count dropped except the
 * first word. */
int dgo_vocab_build(const uint32_t *counts, uint32_t v_num, int min_count, uint32_t *vocab_ids, uint32_t *vocab_cn,
                    int32_t *v2w, uint32_t *vocab_size, uint64_t *train_words) {
    vv *a = (vv *)malloc((size_t)(v_num ? v_num : 1) * sizeof(vv));
    if (!a) return -2;
    for (uint32_t v = 0; v < v_num; v++) { a[v].cn = counts[v]; a[v].id = v; }
    qsort(a, v_num, sizeof(vv), vv_cmp);
    for (uint32_t v = 0; v < v_num; v++) v2w[v] = -1;
    uint32_t n = 0;
    uint64_t tw = 0;
    for (uint32_t i = 0; i < v_num; i++) {
        if ((int64_t)a[i].cn < min_count && i != 0) continue;
        vocab_ids[n] = a[i].id;
        vocab_cn[n] = a[i].cn;
        v2w[a[i].id] = (int32_t)n;
        tw += a[i].cn;
        n++;
    }
    free(a);
    *vocab_size = n;
    *train_words = tw;
    return 0;
}

/* InitUnigramTable, word2vec.cu:537-556 (power 0.75). */
void dgo_unigram_table(const uint32_t *cn, uint32_t vocab_size, uint64_t table_size, int32_t *table) {
    double train_words_pow = 0;
    for (uint32_t a = 0; a < vocab_size; a++) train_words_pow += pow((double)cn[a], 0.75);
    uint32_t i = 0;
    double d1 = pow((double)cn[0], 0.75) / train_words_pow;
    for (uint64_t a = 0; a < table_size; a++) {
        table[a] = (int32_t)i;
        if (a / (double)table_size > d1) {
            i++;
            if (i < vocab_size) d1 += pow((double)cn[i], 0.75) / train_words_pow;
        }
        if (i >= vocab_size) i = vocab_size - 1;
    }
}

/* Subsampling keep thresholds: token kept iff (16 random bits) < thr[w].
 * word2vec.cu:1022-1026 (mode 0) and dsgl.hpp:931-937 (mode 1), in FP32. */
void dgo_keep_thresholds(const uint32_t *cn, uint32_t vocab_size, float sample, uint64_t train_words, int dsgl_form,
                         uint32_t *thr) {
    for (uint32_t w = 0; w < vocab_size; w++) {
        if (!(sample > 0)) { thr[w] = 65536; continue; }
        float ran;
        float sT = sample * (float)train_words;
        if (dsgl_form) {
            float ratio = sT / (float)cn[w];
            ran = sqrtf(ratio) + ratio;
        } else {
            ran = (sqrtf((float)cn[w] / sT) + 1) * sT / (float)cn[w];
        }
        /* discard iff ran < u / 65536.0f */
        uint32_t k = 0;
        if (ran != ran) k = 0;
        else if (ran >= 1.0f) k = 65536;
        else if (ran < 0.0f) k = 0;
        else {
            k = (uint32_t)floorf(ran * 65536.0f) + 1;
            if (k > 65536) k = 65536;
        }
        thr[w] = k;
    }
}

/* InitNet, word2vec.cu:870-873: input rows from the LCG, output rows zero. */
void dgo_init_rows(uint32_t vocab_size, int d, float *syn0) {
    unsigned long long next_random = 1;
    for (uint64_t a = 0; a < vocab_size; a++)
        for (int b = 0; b < d; b++) {
            next_random = next_random * (unsigned long long)25214903917ULL + 11;
            /* 0.5 and layer1_size promote the expression to double; the result is rounded to float */
            syn0[a * d + b] = (float)(((double)((next_random & 0xFFFF) / (float)65536) - 0.5) / (double)d);
        }
}

/* expTable, word2vec.cu:1569-1573. */
void dgo_exp_table(float *t) {
    for (int i = 0; i < EXP_TABLE_SIZE; i++) {
        t[i] = expf((i / (float)EXP_TABLE_SIZE * 2 - 1) * MAX_EXP);
        t[i] = t[i] / (t[i] + 1);
    }
    t[EXP_TABLE_SIZE] = 0.0f;
}

static uint32_t mix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}

/* ---------------------------------------------------------------- plain -- */

static uint32_t philox_word(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed, int word) {
    dgo_u32x4 ctr = {{c0, c1, c2, c3}};
    dgo_u32x4 x = dgo_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    return x.v[word];
}

/* g = (label - sigmoid(f)) * alpha through the table (word2vec.cu:383-388). */
static double grad(double f, int label, const float *exp_table, double alpha) {
    if (f > MAX_EXP) return (label - 1) * alpha;
    if (f < -MAX_EXP) return label * alpha;
    return (label - (double)exp_table[(int)((f + MAX_EXP) * (EXP_TABLE_SIZE / MAX_EXP / 2))]) * alpha;
}

/* Tokens of one walk after vocabulary lookup and subsampling. */
static uint32_t sentence(const dgo_sgns_cfg *c, const uint32_t *walk, uint32_t len, uint32_t wid, int32_t *sen,
                         dgo_sgns_stats *st) {
    uint32_t n = 0;
    for (uint32_t i = 0; i < len; i++) {
        int32_t w = c->v2w[walk[i]];
        if (st) st->words++;
        if (w < 0) continue;
        uint32_t u = philox_word(i, wid, c->pass, DGO_SUB_TAG, c->seed, 0) & 0xFFFFu;
        if (u >= c->keep_thr[w]) continue;
        sen[n++] = w;
    }
    if (st) st->trained += n;
    return n;
}

/* Negative `j` (1-based) of pair (position p, window slot a) of walk wid. */
static int32_t negative_sample(const dgo_sgns_cfg *c, uint32_t p, uint32_t a, uint32_t wid, int j) {
    uint32_t r = philox_word(p * (2 * c->window + 1) + a, wid, c->pass, DGO_NEG_TAG + (uint32_t)((j - 1) >> 2),
                             c->seed, (j - 1) & 3);
    int32_t t = c->table[r % c->table_size];
    if (t == 0) t = (int32_t)((r >> 8) % (c->vocab_size - 1) + 1); /* word2vec.cu:367 */
    return t;
}

/* skip_gram_kernel semantics (word2vec.cu:305-399), one sentence after another:
 * for each centre, a shrunk window b; for each context row syn0[ctx], the
 * positive target (the centre) and `negative` sampled targets update syn1 at
 * once and syn0[ctx] after the pair. */
int dgo_sgns_plain(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                   const uint32_t *walk_ids, double *syn0, double *syn1, dgo_sgns_stats *st) {
    const int d = c->d;
    int32_t *sen = (int32_t *)malloc(65536 * sizeof(int32_t));
    double *neu1e = (double *)malloc((size_t)d * sizeof(double));
    if (!sen || !neu1e) { free(sen); free(neu1e); return -2; }
    for (uint32_t k = 0; k < n_walks; k++) {
        const uint32_t wid = walk_ids ? walk_ids[k] : k;
        uint32_t len = (uint32_t)(offsets[k + 1] - offsets[k]);
        if (len > 65536) len = 65536;
        uint32_t n = sentence(c, verts + offsets[k], len, wid, sen, st);
        for (uint32_t p = 0; p < n; p++) {
            const int32_t word = sen[p];
            const uint32_t b = philox_word(p, wid, c->pass, DGO_WIN_TAG, c->seed, 0) % (uint32_t)c->window;
            for (uint32_t a = b; a < (uint32_t)(2 * c->window + 1) - b; a++) {
                if (a == (uint32_t)c->window) continue;
                int64_t cpos = (int64_t)p - c->window + a;
                if (cpos < 0 || cpos >= n) continue;
                const int32_t last = sen[cpos];
                double *l1 = syn0 + (size_t)last * d;
                for (int i = 0; i < d; i++) neu1e[i] = 0;
                if (st) st->pairs++;
                for (int j = 0; j <= c->negative; j++) {
                    int32_t target;
                    int label;
                    if (j == 0) { target = word; label = 1; }
                    else {
                        if (c->vocab_size < 2) continue;
                        target = negative_sample(c, p, a, wid, j);
                        if (target == word) continue;
                        label = 0;
                    }
                    double *l2 = syn1 + (size_t)target * d;
                    double f = 0;
                    for (int i = 0; i < d; i++) f += l1[i] * l2[i];
                    double g = grad(f, label, c->exp_table, c->alpha);
                    for (int i = 0; i < d; i++) neu1e[i] += g * l2[i];
                    for (int i = 0; i < d; i++) l2[i] += g * l1[i];
                }
                for (int i = 0; i < d; i++) l1[i] += neu1e[i];
            }
        }
    }
    free(sen);
    free(neu1e);
    return 0;
}

/* ------------------------------------------------------------ minibatch -- */

#define MB_MAX_SENT 32
#define MB_WIN_TAG 0x4D425749u
#define MB_POOL_TAG 0x4D42504Fu

typedef struct {
    int len, pos, ndist;
    int32_t sen[MB_MAX_SENT];
    int slot[MB_MAX_SENT];
    int32_t dist[MB_MAX_SENT];
    double *cache; /* ndist x d */
    double *init;
} mb_sentence;

/* Fills s from the next walks until one has >= 2 kept tokens (dsgl.hpp:903-1028). */
static int mb_fill(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                   uint32_t *next, mb_sentence *s, const double *syn0, dgo_sgns_stats *st) {
    while (s->len == 0) {
        if (*next >= n_walks) return 0;
        uint32_t w = (*next)++;
        uint32_t len = (uint32_t)(offsets[w + 1] - offsets[w]);
        if (len > MB_MAX_SENT) len = MB_MAX_SENT;
        int n = 0;
        for (uint32_t i = 0; i < len; i++) {
            int32_t word = c->v2w[verts[offsets[w] + i]];
            if (word < 0) continue;
            uint32_t u = philox_word(i, w, c->pass, DGO_SUB_TAG, c->seed, 0) & 0xFFFFu;
            if (u >= c->keep_thr[word]) continue;
            s->sen[n++] = word;
        }
        if (st) { st->words += len; st->trained += n; }
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
                for (int k = 0; k < c->d; k++)
                    s->cache[r * c->d + k] = s->init[r * c->d + k] = syn0[(size_t)s->dist[r] * c->d + k];
    }
    return 1;
}

static void mb_flush(const dgo_sgns_cfg *c, mb_sentence *s, double *syn0) {
    for (int r = 0; r < s->ndist; r++)
        for (int k = 0; k < c->d; k++)
            syn0[(size_t)s->dist[r] * c->d + k] += s->cache[r * c->d + k] - s->init[r * c->d + k];
}

/* dsgl.hpp Train_SGNS_MPI (MKL branch) as one worker over all walks, with the
 * device kernel's deviations: Philox draws, delta write-back of caches,
 * in-flight sentences and pool written back when the walks run out. */
int dgo_sgns_minibatch(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                       double *syn0, double *syn1, dgo_sgns_stats *st) {
    const int d = c->d, neg = c->negative, win = c->window;
    const uint32_t key0 = (uint32_t)c->seed ^ mix32(c->pass * 0x9E3779B9u + 0x632BE5ABu);
    const uint32_t key1 = (uint32_t)(c->seed >> 32);
    const uint64_t mbseed = ((uint64_t)key1 << 32) | key0;
    const int pool_cap = MB_MAX_SENT * (neg > 0 ? neg : 1);
    mb_sentence S[2];
    memset(S, 0, sizeof(S));
    for (int s = 0; s < 2; s++) {
        S[s].cache = (double *)malloc((size_t)MB_MAX_SENT * d * sizeof(double));
        S[s].init = (double *)malloc((size_t)MB_MAX_SENT * d * sizeof(double));
    }
    int32_t *pool_word = (int32_t *)malloc(pool_cap * sizeof(int32_t));
    int *pool_slot = (int *)malloc(pool_cap * sizeof(int));
    double *pool_cur = (double *)malloc((size_t)pool_cap * d * sizeof(double));
    double *pool_init = (double *)malloc((size_t)pool_cap * d * sizeof(double));
    const int MO = neg + 2, MI = 4 * win;
    double *outs = (double *)malloc((size_t)MO * d * sizeof(double));
    double *gm = (double *)malloc((size_t)MO * MI * sizeof(double));
    double *md = (double *)malloc((size_t)MO * d * sizeof(double));
    int in_row[256], out_word[64], out_meta[64], out_slot[64];
    uint32_t next = 0, step = 0, pool_no = 0, neg_count = 0;
    int train_sen_num = 0, change_neg = 1, pool_loaded = 0, np = 0, nbn = 1;
    for (;;) {
        int ok0 = mb_fill(c, offsets, verts, n_walks, &next, &S[0], syn0, st);
        int ok1 = ok0 ? mb_fill(c, offsets, verts, n_walks, &next, &S[1], syn0, st) : 0;
        if (!ok0 || !ok1) break;
        if (change_neg) {
            nbn = S[0].len > S[1].len ? S[0].len : S[1].len;
            np = 0;
            for (int j = 0; j < nbn * neg; j++) {
                uint32_t r = philox_word((uint32_t)j >> 2, pool_no, 0, MB_POOL_TAG, mbseed, j & 3);
                int32_t smp = c->table[r % c->table_size];
                if (!smp) smp = c->vocab_size > 1 ? (int32_t)((r >> 8) % (c->vocab_size - 1) + 1) : 0;
                int at = -1;
                for (int t = 0; t < np; t++) if (pool_word[t] == smp) { at = t; break; }
                if (at < 0) { at = np; pool_word[np++] = smp; }
                pool_slot[j] = at;
            }
            for (int r = 0; r < np; r++)
                for (int k = 0; k < d; k++)
                    pool_cur[(size_t)r * d + k] = pool_init[(size_t)r * d + k] = syn1[(size_t)pool_word[r] * d + k];
            pool_no++;
            change_neg = 0;
            pool_loaded = 1;
        }
        const uint32_t b = philox_word(step, 0, 0, MB_WIN_TAG, mbseed, 0) % (uint32_t)win;
        int ni = 0, first = 0;
        for (int s = 0; s < 2; s++) {
            for (int i = (int)b; i < 2 * win + 1 - (int)b; i++) {
                if (i == win) continue;
                int cpos = S[s].pos - win + i;
                if (cpos < 0) continue;
                if (cpos >= S[s].len) break;
                in_row[ni++] = s * MB_MAX_SENT + S[s].slot[cpos];
            }
            if (s == 0) first = ni;
        }
        neg_count++;
        int start = (int)(neg_count % (uint32_t)nbn), off = 1;
        out_word[0] = S[0].sen[S[0].pos]; out_meta[0] = 1; out_slot[0] = -1;
        for (int k = 0; k < neg; k++) {
            int ps = pool_slot[start * neg + k], smp = pool_word[ps], at = -1;
            for (int t = 0; t < off; t++) if (out_word[t] == smp) { at = t; break; }
            if (at < 0) { out_word[off] = smp; out_meta[off] = 1; out_slot[off] = ps; off++; }
            else out_meta[at]++;
        }
        out_meta[0] = 1;
        out_word[off] = S[1].sen[S[1].pos]; out_meta[off] = 1; out_slot[off] = -1;
        const int O = off + 1, I = ni;
        if (st) st->pairs += ni;
        for (int o = 0; o < O; o++)
            for (int k = 0; k < d; k++)
                outs[(size_t)o * d + k] = out_slot[o] < 0 ? syn1[(size_t)out_word[o] * d + k]
                                                          : pool_cur[(size_t)out_slot[o] * d + k];
#define IN_ROW(i) (in_row[i] < MB_MAX_SENT ? S[0].cache + (size_t)in_row[i] * d \
                                           : S[1].cache + (size_t)(in_row[i] - MB_MAX_SENT) * d)
        for (int o = 0; o < O; o++)
            for (int i = 0; i < I; i++) {
                const double *x = outs + (size_t)o * d, *y = IN_ROW(i);
                double f = 0;
                for (int k = 0; k < d; k++) f += x[k] * y[k];
                int label = i < first ? (o == 0) : (o == O - 1);
                gm[o * MI + i] = grad(f, label, c->exp_table, c->alpha) * out_meta[o];
            }
        for (int o = 0; o < O; o++)
            for (int k = 0; k < d; k++) {
                double acc = 0;
                for (int i = 0; i < I; i++) acc += gm[o * MI + i] * IN_ROW(i)[k];
                md[(size_t)o * d + k] = acc;
            }
        for (int k = 0; k < d; k++)
            for (int i = 0; i < I; i++) {
                double acc = 0;
                for (int o = 0; o < O; o++) acc += gm[o * MI + i] * outs[(size_t)o * d + k];
                IN_ROW(i)[k] += acc;
            }
#undef IN_ROW
        for (int k = 0; k < d; k++) {
            syn1[(size_t)out_word[0] * d + k] += md[k];
            syn1[(size_t)out_word[O - 1] * d + k] += md[(size_t)(O - 1) * d + k];
        }
        for (int o = 1; o < O - 1; o++)
            for (int k = 0; k < d; k++) pool_cur[(size_t)out_slot[o] * d + k] += md[(size_t)o * d + k];
        step++;
        S[0].pos++;
        S[1].pos++;
        for (int s = 0; s < 2; s++)
            if (S[s].pos >= S[s].len) { mb_flush(c, &S[s], syn0); S[s].len = 0; train_sen_num++; }
        if (train_sen_num >= 2) {
            for (int r = 0; r < np; r++)
                for (int k = 0; k < d; k++)
                    syn1[(size_t)pool_word[r] * d + k] += pool_cur[(size_t)r * d + k] - pool_init[(size_t)r * d + k];
            change_neg = 1;
            pool_loaded = 0;
            train_sen_num = 0;
        }
    }
    for (int s = 0; s < 2; s++) if (S[s].len) mb_flush(c, &S[s], syn0);
    if (pool_loaded)
        for (int r = 0; r < np; r++)
            for (int k = 0; k < d; k++)
                syn1[(size_t)pool_word[r] * d + k] += pool_cur[(size_t)r * d + k] - pool_init[(size_t)r * d + k];
    for (int s = 0; s < 2; s++) { free(S[s].cache); free(S[s].init); }
    free(pool_word); free(pool_slot); free(pool_cur); free(pool_init); free(outs); free(gm); free(md);
    return 0;
}
