/*
 * FP32 restatement of word2vec.cu's three negative-sampling trainers, with the
 * per-pair (per-centre) arithmetic shared between two forms.  TEST
 * INFRASTRUCTURE ONLY (see dg_oracle.h).
 *
 *  - Reference form (dgo_w2v_sentences): the kernels as the reference launches
 *    them on host-built sentences, one block per sentence, with the block's
 *    own LCG stream (word2vec.cu:319-321, 365-368, 415-417, 457-460), their
 *    reduction orders and the negative sets of __sgNegReuse passed in.  It is
 *    checked against the reference's kernels compiled for sm_100a
 *    (oracle/_ref/libref_w2v.so), one sentence per launch.
 *  - Device form (dgo_sgns_plain_f32 in dg_oracle_sgns32.c, dgo_sgns_cbow_f32 and
 *    dgo_sgns_negshare_f32 below): the same per-pair code over walks with the
 *    device kernels' Philox draws and warp reduction order, bit-exact against
 *    the deterministic device mode.
 *
 * Compiled with -ffp-contract=off: only the explicit fmaf calls fuse, at the
 * sites where nvcc contracts the reference's `x += a * b` (checked against the
 * reference's kernels); products handed to an atomicAdd are rounded first.
 */
#include "dg_oracle.h"
#include "philox.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define EXP_TABLE_SIZE 1000
#define MAX_EXP 6

/* ------------------------------------------------------- dot products -- */

/* Device kernels: lane l of a warp holds columns [l*v, l*v+v) (v = d/32), a
 * fused chain per lane, then an xor butterfly over 16 .. 1 lanes. */
static float dot_warp(const float *a, const float *b, int d) {
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

/* skip_gram_kernel / cbow_kernel (word2vec.cu:371-381, 435-444): F = half the
 * power of two >= d; f[x] = a[x] b[x] for x < F, then threads x >= F add their
 * product into f[x - F] (fused), then a shared-memory tree f[x] += f[x + i],
 * i = F/2 .. 1. */
static float dot_tree(const float *a, const float *b, int d) {
    int redu = 32;
    while (redu < d) redu *= 2;
    const int F = redu / 2;
    float f[512];
    for (int x = 0; x < F; x++) f[x] = x < d ? a[x] * b[x] : 0.f;
    for (int x = F; x < d; x++) f[x - F] = fmaf(a[x], b[x], f[x - F]);
    for (int i = F / 2; i > 0; i /= 2)
        for (int x = 0; x < i; x++) f[x] = f[x] + f[x + i];
    return f[0];
}

/* __sgNegReuse (word2vec.cu:263-266): lane l sums columns l, l+32, ... in a fused
 * chain; reduceInWarp (word2vec.cu:77-82) then adds, at offsets 16, 8, 4, 2, 1,
 * the value held by LANE `offset` (__shfl_sync with a source lane, not an xor or
 * down shuffle), so lane l ends with its own partial plus a sum common to all
 * lanes rather than the dot product.  `exact` = 1 sums the lanes instead. */
static void dot_lanes_reuse(const float *a, const float *b, int d, int exact, float out[32]) {
    float p[32], q[32];
    for (int l = 0; l < 32; l++) {
        float s = 0.f;
        for (int i = l; i < d; i += 32) s = fmaf(a[i], b[i], s);
        p[l] = s;
    }
    if (exact) {
        float s = 0.f;
        for (int l = 0; l < 32; l++) s += p[l];
        for (int l = 0; l < 32; l++) out[l] = s;
        return;
    }
    for (int o = 16; o; o >>= 1) {
        for (int l = 0; l < 32; l++) q[l] = p[l] + p[o];
        memcpy(p, q, sizeof(p));
    }
    memcpy(out, p, sizeof(p));
}

static float grad_table(float f, int label, const float *t, float alpha) {
    if (f > MAX_EXP) return (label - 1) * alpha;
    if (f < -MAX_EXP) return label * alpha;
    return (label - t[(int)((f + MAX_EXP) * (EXP_TABLE_SIZE / MAX_EXP / 2))]) * alpha;
}

static float dot_order(int order, const float *a, const float *b, int d) {
    return order == DGO_ORDER_REF ? dot_tree(a, b, d) : dot_warp(a, b, d);
}

/* ----------------------------------------------------- shared updates -- */

/* Hierarchical softmax over the centre's Huffman path (word2vec.cu:334-356,
 * 436-455): for each inner node point[k] with code bit code[k], f = x . syn1[node];
 * nodes with |f| >= MAX_EXP are skipped, else g = (1 - code - sigmoid(f)) alpha,
 * e += g syn1[node] (fused), syn1[node] += rounded g x.  The inner nodes index
 * the same output table as the words (the reference trains both with d_syn1). */
static void hs_path(int order, int d, float alpha, const float *exp_table, const float *x, const int32_t *point,
                    const int8_t *code, int n_hs, float *syn1, float *e) {
    for (int k = 0; k < n_hs; k++) {
        float *row = syn1 + (size_t)point[k] * d;
        const float f = dot_order(order, x, row, d);
        if (f <= -MAX_EXP || f >= MAX_EXP) continue;
        const float g = ((float)(1 - code[k]) - exp_table[(int)((f + MAX_EXP) * (EXP_TABLE_SIZE / MAX_EXP / 2))]) *
                        alpha;
        for (int i = 0; i < d; i++) {
            e[i] = fmaf(g, row[i], e[i]);
            const float u = g * x[i];
            row[i] = row[i] + u;
        }
    }
}

/* One (context, centre) pair of skip_gram_kernel (word2vec.cu:330-397): the
 * centre's hierarchical-softmax path first (n_hs nodes, none without -hs), then
 * for the positive target tg[0] and the negatives tg[1..nt), in order,
 * f = l1 . syn1[t], g = (label - sigmoid(f)) alpha, e += g syn1[t] (fused),
 * syn1[t] += rounded g l1; then l1 += e. */
void dgo_w2v_sg_pair(int order, int d, float alpha, const float *exp_table, float *l1, const int32_t *hs_point,
                     const int8_t *hs_code, int n_hs, const int32_t *tg, int nt, float *syn1, float *e) {
    for (int i = 0; i < d; i++) e[i] = 0.f;
    hs_path(order, d, alpha, exp_table, l1, hs_point, hs_code, n_hs, syn1, e);
    for (int t = 0; t < nt; t++) {
        float *row = syn1 + (size_t)tg[t] * d;
        const float g = grad_table(dot_order(order, l1, row, d), t == 0, exp_table, alpha);
        for (int i = 0; i < d; i++) {
            e[i] = fmaf(g, row[i], e[i]);
            const float u = g * l1[i];
            row[i] = row[i] + u;
        }
    }
    for (int i = 0; i < d; i++) l1[i] = l1[i] + e[i];
}

/* One centre of cbow_kernel (word2vec.cu:419-505): neu1 = the mean of the
 * context rows (summed in window order, then divided by their count), the
 * hierarchical-softmax path and the targets as in a skip-gram pair with neu1 in
 * place of l1, then e added to every context row in window order. */
void dgo_w2v_cbow_centre(int order, int d, float alpha, const float *exp_table, const int32_t *ctx, int cw,
                         const int32_t *hs_point, const int8_t *hs_code, int n_hs, const int32_t *tg, int nt,
                         float *syn0, float *syn1, float *neu1, float *e) {
    for (int i = 0; i < d; i++) { neu1[i] = 0.f; e[i] = 0.f; }
    for (int c = 0; c < cw; c++) {
        const float *r = syn0 + (size_t)ctx[c] * d;
        for (int i = 0; i < d; i++) neu1[i] = neu1[i] + r[i];
    }
    for (int i = 0; i < d; i++) neu1[i] = neu1[i] / (float)cw;
    hs_path(order, d, alpha, exp_table, neu1, hs_point, hs_code, n_hs, syn1, e);
    for (int t = 0; t < nt; t++) {
        float *row = syn1 + (size_t)tg[t] * d;
        const float g = grad_table(dot_order(order, neu1, row, d), t == 0, exp_table, alpha);
        for (int i = 0; i < d; i++) {
            e[i] = fmaf(g, row[i], e[i]);
            const float u = g * neu1[i];
            row[i] = row[i] + u;
        }
    }
    for (int c = 0; c < cw; c++) {
        float *r = syn0 + (size_t)ctx[c] * d;
        for (int i = 0; i < d; i++) r[i] = r[i] + e[i];
    }
}

/* One (context, centre) pair of __sgNegReuse (word2vec.cu:252-300): every target
 * (the shared negatives that differ from the centre, in order, then the centre
 * as the positive) takes its dot product with the unchanged context row l1;
 * e += rounded g syn1[t] (a shared-memory atomicAdd in the reference, so its
 * order there is the warps' arrival order), syn1[t] += g l1 (fused); then
 * l1 += e.  In the reference form (exact_sum == 0) each lane's columns use that
 * lane's own g (see dot_lanes_reuse) and the sigmoid is recomputed with exp(),
 * which is the expTable formula at the same index. */
void dgo_w2v_reuse_pair(int order, int exact_sum, int d, float alpha, const float *exp_table, float *l1, int32_t word,
                        const int32_t *negs, int n, float *syn1, float *e) {
    for (int i = 0; i < d; i++) e[i] = 0.f;
    for (int y = 0; y <= n; y++) {
        const int32_t t = y < n ? negs[y] : word;
        if (y < n && t == word) continue;
        const int label = y == n;
        float *row = syn1 + (size_t)t * d;
        float g[32];
        if (order == DGO_ORDER_REF) {
            float f[32];
            dot_lanes_reuse(l1, row, d, exact_sum, f);
            for (int l = 0; l < 32; l++) g[l] = grad_table(f[l], label, exp_table, alpha);
        } else {
            const float gg = grad_table(dot_warp(l1, row, d), label, exp_table, alpha);
            for (int l = 0; l < 32; l++) g[l] = gg;
        }
        for (int i = 0; i < d; i++) {
            const float u = g[i & 31] * row[i];
            e[i] = e[i] + u;
        }
        for (int i = 0; i < d; i++) row[i] = fmaf(g[i & 31], l1[i], row[i]);
    }
    for (int i = 0; i < d; i++) l1[i] = l1[i] + e[i];
}

/* The centre word's Huffman path (point, code, length) when the config trains
 * hierarchical softmax, else an empty path. */
#define HS_ARGS(c, word)                                                            \
    ((c)->hs ? (c)->hs_point + (c)->hs_off[word] : NULL),                           \
    ((c)->hs ? (c)->hs_code + (c)->hs_off[word] : NULL),                            \
    ((c)->hs ? (c)->hs_off[(word) + 1] - (c)->hs_off[word] : 0)

/* word2vec's Huffman coding restated (CreateBinaryTree, word2vec.cu:684-740):
 * merge the two smallest of the sorted counts and the new inner nodes, bit 1 for
 * the second; then each word's path from the root, laid out as the kernels read
 * it (InitVocabStructCUDA, word2vec.cu:511-535): off[n + 1] prefix of the code
 * lengths, point[] = the inner node (0 .. n-2) deciding each bit, code[] the
 * bits.  cn: counts in vocabulary order (most frequent first), n >= 2; point
 * and code hold n * 40 entries.  Returns the total length, or -1 when a code
 * would be longer than the reference's 40 (MAX_CODE_LENGTH). */
int64_t dgo_huffman(const uint64_t *cn, uint32_t n, int32_t *off, int32_t *point, int8_t *code) {
    if (n < 2) return -1;
    const uint64_t N = n;
    long long *count = (long long *)calloc(2 * N + 1, sizeof(long long));
    long long *binary = (long long *)calloc(2 * N + 1, sizeof(long long));
    long long *parent = (long long *)calloc(2 * N + 1, sizeof(long long));
    if (!count || !binary || !parent) { free(count); free(binary); free(parent); return -2; }
    for (uint64_t a = 0; a < N; a++) count[a] = (long long)cn[a];
    for (uint64_t a = N; a < 2 * N; a++) count[a] = (long long)1e15;
    long long p1 = (long long)N - 1, p2 = (long long)N;
    for (uint64_t a = 0; a + 1 < N; a++) {
        long long m[2];
        for (int k = 0; k < 2; k++) {
            if (p1 >= 0 && count[p1] < count[p2]) m[k] = p1--;
            else m[k] = p2++;
        }
        count[N + a] = count[m[0]] + count[m[1]];
        parent[m[0]] = (long long)(N + a);
        parent[m[1]] = (long long)(N + a);
        binary[m[1]] = 1;
    }
    int64_t total = 0;
    long long path[64];
    int8_t bits[64];
    off[0] = 0;
    for (uint64_t a = 0; a < N; a++) {
        int len = 0;
        long long b = (long long)a;
        while (len < 64) {
            bits[len] = (int8_t)binary[b];
            path[len] = b;
            len++;
            b = parent[b];
            if (b == (long long)(2 * N - 2)) break;
        }
        if (len > 40) { total = -1; break; }
        /* Bit k (from the root) is decided by point[k]: the root n - 2 first, then
         * the inner nodes on the way down. */
        for (int k = 0; k < len; k++) {
            code[total + k] = bits[len - 1 - k];
            point[total + k] = k == 0 ? (int32_t)(N - 2) : (int32_t)(path[len - k] - (long long)N);
        }
        total += len;
        off[a + 1] = (int32_t)total;
    }
    free(count); free(binary); free(parent);
    return total;
}

/* ------------------------------------------------------ reference form -- */

static unsigned long long lcg(unsigned long long x, unsigned long long a) { return x * a + 11; }

/* Negative draw of the reference kernels (word2vec.cu:365-368, 457-460). */
static int32_t lcg_negative(const dgo_w2v_cfg *c, unsigned long long *nr) {
    *nr = lcg(*nr, 25214903917ULL);
    int32_t t = c->table[(*nr >> 16) % c->table_size];
    if (t == 0) t = (int32_t)(*nr % (unsigned long long)(c->vocab_size - 1) + 1);
    return t;
}

int dgo_w2v_sentences(const dgo_w2v_cfg *c, const int32_t *sen, const int32_t *sent_off, uint32_t n_sent,
                      const int32_t *neg_samples, float *syn0, float *syn1) {
    const int d = c->d, w = c->window, n = c->negative;
    if (d < 1 || d > 512 || w < 1 || n < 0 || n > 64) return -1;
    float *e = (float *)malloc((size_t)d * sizeof(float)), *neu1 = (float *)malloc((size_t)d * sizeof(float));
    int32_t tg[65], ctx[256];
    if (!e || !neu1) { free(e); free(neu1); return -2; }
    for (uint32_t k = 0; k < n_sent; k++) {
        const int s = sent_off[k], t_end = sent_off[k + 1];
        unsigned long long nr = k; /* next_random = blockIdx.x */
        for (int p = s; p < t_end; p++) {
            const int32_t word = sen[p];
            if (word == -1) continue;
            if (c->kind == DGO_W2V_NEGREUSE) {
                for (int a = 0; a < 2 * w + 1; a++) {
                    if (a == w) continue;
                    const int cp = p - w + a;
                    if (cp < s || cp >= t_end || sen[cp] == -1) continue;
                    dgo_w2v_reuse_pair(DGO_ORDER_REF, c->exact_sum, d, c->alpha, c->exp_table,
                                       syn0 + (size_t)sen[cp] * d, word, neg_samples + (size_t)k * n, n, syn1, e);
                }
                continue;
            }
            nr = lcg(nr, 2514903917ULL); /* the reference's constant (one digit short of the LCG's) */
            const int b = (int)(nr % (unsigned long long)w);
            if (c->kind == DGO_W2V_SG) {
                for (int a = b; a < 2 * w + 1 - b; a++) {
                    if (a == w) continue;
                    const int cp = p - w + a;
                    if (cp < s || cp >= t_end || sen[cp] == -1) continue;
                    int nt = 0;
                    tg[nt++] = word;
                    for (int j = 0; j < n; j++) {
                        const int32_t t = lcg_negative(c, &nr);
                        if (t != word) tg[nt++] = t;
                    }
                    dgo_w2v_sg_pair(DGO_ORDER_REF, d, c->alpha, c->exp_table, syn0 + (size_t)sen[cp] * d,
                                    HS_ARGS(c, word), tg, nt, syn1, e);
                }
            } else {
                int cw = 0;
                for (int a = b; a < 2 * w + 1 - b; a++) {
                    if (a == w) continue;
                    const int cp = p - w + a;
                    if (cp < s || cp >= t_end || sen[cp] == -1) continue;
                    ctx[cw++] = sen[cp];
                }
                if (!cw) continue;
                int nt = 0;
                tg[nt++] = word;
                for (int j = 0; j < n; j++) {
                    const int32_t t = lcg_negative(c, &nr);
                    if (t != word) tg[nt++] = t;
                }
                dgo_w2v_cbow_centre(DGO_ORDER_REF, d, c->alpha, c->exp_table, ctx, cw, HS_ARGS(c, word), tg, nt, syn0,
                                    syn1, neu1, e);
            }
        }
    }
    free(e);
    free(neu1);
    return 0;
}

/* --------------------------------------------------------- device form -- */

static uint32_t pword(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed, int word) {
    dgo_u32x4 ctr = {{c0, c1, c2, c3}};
    dgo_u32x4 x = dgo_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    return x.v[word];
}

static int32_t philox_negative(const dgo_sgns_cfg *c, uint32_t c0, uint32_t wid, uint32_t tag, int j) {
    const uint32_t r = pword(c0, wid, c->pass, tag + (uint32_t)(j >> 2), c->seed, j & 3);
    int32_t t = c->table[r % c->table_size];
    if (t == 0) t = (int32_t)((r >> 8) % (c->vocab_size - 1) + 1);
    return t;
}

/* Kept tokens of walk w (vocabulary lookup + Philox subsampling draw), at most
 * 1024 of them, as the device's warp_sentence builds them. */
static uint32_t walk_sentence(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t w,
                              int32_t *sen, dgo_sgns_stats *st) {
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
    return n;
}

/* cbow_kernel's rule over walks, one centre after another: window shrink b from
 * (p, walk, pass, WIN tag), negatives j of centre p from (p, walk, pass,
 * CBOW tag + j/4) word j%4. */
int dgo_sgns_cbow_f32(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                      float *syn0, float *syn1, dgo_sgns_stats *st) {
    const int d = c->d, win = c->window;
    int32_t *sen = (int32_t *)malloc(1024 * sizeof(int32_t));
    float *e = (float *)malloc((size_t)d * sizeof(float)), *neu1 = (float *)malloc((size_t)d * sizeof(float));
    int32_t tg[65], ctx[256];
    if (!sen || !e || !neu1) { free(sen); free(e); free(neu1); return -2; }
    for (uint32_t w = 0; w < n_walks; w++) {
        const uint32_t n = walk_sentence(c, offsets, verts, w, sen, st);
        for (uint32_t p = 0; p < n; p++) {
            const int32_t word = sen[p];
            const uint32_t b = pword(p, w, c->pass, DGO_WIN_TAG, c->seed, 0) % (uint32_t)win;
            int cw = 0;
            for (uint32_t a = b; a < (uint32_t)(2 * win + 1) - b; a++) {
                if (a == (uint32_t)win) continue;
                const int64_t cp = (int64_t)p - win + a;
                if (cp < 0 || cp >= n) continue;
                ctx[cw++] = sen[cp];
            }
            if (!cw) continue;
            if (st) st->pairs += (uint64_t)cw;
            int nt = 0;
            tg[nt++] = word;
            if (c->vocab_size > 1)
                for (int j = 0; j < c->negative; j++) {
                    const int32_t t = philox_negative(c, p, w, DGO_CBOW_TAG, j);
                    if (t != word) tg[nt++] = t;
                }
            dgo_w2v_cbow_centre(DGO_ORDER_DEVICE, d, (float)c->alpha, c->exp_table, ctx, cw, HS_ARGS(c, word), tg, nt,
                                syn0, syn1, neu1, e);
        }
    }
    free(sen); free(e); free(neu1);
    return 0;
}

/* __sgNegReuse's rule over walks: one negative set per walk, j from (0, walk,
 * pass, SHARE tag + j/4) word j%4; the full window (no shrink); the warp sum as
 * the dot product. */
int dgo_sgns_negshare_f32(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                          float *syn0, float *syn1, dgo_sgns_stats *st) {
    const int d = c->d, win = c->window, neg = c->negative;
    int32_t *sen = (int32_t *)malloc(1024 * sizeof(int32_t));
    float *e = (float *)malloc((size_t)d * sizeof(float));
    int32_t negs[64];
    if (!sen || !e || neg > 64) { free(sen); free(e); return -2; }
    for (uint32_t w = 0; w < n_walks; w++) {
        const uint32_t n = walk_sentence(c, offsets, verts, w, sen, st);
        int nn = 0;
        if (c->vocab_size > 1)
            for (int j = 0; j < neg; j++) negs[nn++] = philox_negative(c, 0, w, DGO_SHARE_TAG, j);
        for (uint32_t p = 0; p < n; p++) {
            const int32_t word = sen[p];
            for (uint32_t a = 0; a < (uint32_t)(2 * win + 1); a++) {
                if (a == (uint32_t)win) continue;
                const int64_t cp = (int64_t)p - win + a;
                if (cp < 0 || cp >= n) continue;
                if (st) st->pairs++;
                dgo_w2v_reuse_pair(DGO_ORDER_DEVICE, 1, d, (float)c->alpha, c->exp_table, syn0 + (size_t)sen[cp] * d,
                                   word, negs, nn, syn1, e);
            }
        }
    }
    free(sen); free(e);
    return 0;
}
