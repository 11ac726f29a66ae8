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
    float *e = (float *)malloc(d * sizeof(float)), *pos = (float *)malloc(d * sizeof(float));
    if (!sen || !e || !pos) return -2;
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
            memcpy(pos, syn1 + (size_t)word * d, d * sizeof(float));
            for (uint32_t a = b; a < (uint32_t)(2 * c->window + 1) - b; a++) {
                if (a == (uint32_t)c->window) continue;
                int64_t cp = (int64_t)p - c->window + a;
                if (cp < 0 || cp >= n) continue;
                float *l1 = syn0 + (size_t)sen[cp] * d;
                for (int i = 0; i < d; i++) e[i] = 0.f;
                if (st) st->pairs++;
                float g = grad32(warp_dot(l1, pos, d), 1, c->exp_table, alpha);
                for (int i = 0; i < d; i++) { e[i] = fmaf(g, pos[i], e[i]); pos[i] = fmaf(g, l1[i], pos[i]); }
                if (c->vocab_size > 1)
                    for (int j = 1; j <= c->negative; j++) {
                        uint32_t r = pword(p * (2 * c->window + 1) + a, w, c->pass,
                                           DGO_NEG_TAG + (uint32_t)((j - 1) >> 2), c->seed, (j - 1) & 3);
                        int32_t t = c->table[r % c->table_size];
                        if (t == 0) t = (int32_t)((r >> 8) % (c->vocab_size - 1) + 1);
                        if (t == word) continue;
                        float *l2 = syn1 + (size_t)t * d;
                        g = grad32(warp_dot(l1, l2, d), 0, c->exp_table, alpha);
                        for (int i = 0; i < d; i++) {
                            e[i] = fmaf(g, l2[i], e[i]);
                            float u = g * l1[i];
                            l2[i] = l2[i] + u;
                        }
                    }
                for (int i = 0; i < d; i++) l1[i] = l1[i] + e[i];
            }
            memcpy(syn1 + (size_t)word * d, pos, d * sizeof(float));
        }
    }
    free(sen); free(e); free(pos);
    return 0;
}

typedef struct {
    int len, pos, ndist;
    int32_t sen[MB_MAX_SENT];
    int slot[MB_MAX_SENT];
    int32_t dist[MB_MAX_SENT];
    float cache[MB_MAX_SENT * 512];
    float init[MB_MAX_SENT * 512];
} mb32_sentence;

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

static void mb32_flush(const dgo_sgns_cfg *c, mb32_sentence *s, float *syn0) {
    for (int r = 0; r < s->ndist; r++)
        for (int k = 0; k < c->d; k++) {
            float *x = syn0 + (size_t)s->dist[r] * c->d + k;
            *x = *x + (s->cache[r * c->d + k] - s->init[r * c->d + k]);
        }
}

int dgo_sgns_minibatch_f32(const dgo_sgns_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                           float *syn0, float *syn1, dgo_sgns_stats *st) {
    const int d = c->d, neg = c->negative, win = c->window;
    const float alpha = (float)c->alpha;
    if (d > 512) return -1;
    const uint32_t key0 = (uint32_t)c->seed ^ mix32(c->pass * 0x9E3779B9u + 0x632BE5ABu);
    const uint64_t mbseed = ((uint64_t)(uint32_t)(c->seed >> 32) << 32) | key0;
    const int pool_cap = MB_MAX_SENT * (neg > 0 ? neg : 1);
    mb32_sentence *S = (mb32_sentence *)calloc(2, sizeof(mb32_sentence));
    int32_t *pool_word = (int32_t *)malloc(pool_cap * sizeof(int32_t));
    int *pool_slot = (int *)malloc(pool_cap * sizeof(int));
    float *pool_cur = (float *)malloc((size_t)pool_cap * d * sizeof(float));
    float *pool_init = (float *)malloc((size_t)pool_cap * d * sizeof(float));
    const int MO = neg + 2, MI = 4 * win;
    float *outs = (float *)malloc((size_t)MO * d * sizeof(float));
    float *gm = (float *)malloc((size_t)MO * MI * sizeof(float));
    float *md = (float *)malloc((size_t)MO * sizeof(float));
    int in_row[256], out_word[64], out_meta[64], out_slot[64];
    uint32_t next = 0, step = 0, pool_no = 0, neg_count = 0;
    int train_sen_num = 0, change_neg = 1, pool_loaded = 0, np = 0, nbn = 1;
    for (;;) {
        int ok0 = mb32_fill(c, offsets, verts, n_walks, &next, &S[0], syn0, st);
        int ok1 = ok0 ? mb32_fill(c, offsets, verts, n_walks, &next, &S[1], syn0, st) : 0;
        if (!ok0 || !ok1) break;
        if (change_neg) {
            nbn = S[0].len > S[1].len ? S[0].len : S[1].len;
            np = 0;
            for (int j = 0; j < nbn * neg; j++) {
                uint32_t r = pword((uint32_t)j >> 2, pool_no, 0, MB_POOL_TAG, mbseed, j & 3);
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
        const uint32_t b = pword(step, 0, 0, MB_WIN_TAG, mbseed, 0) % (uint32_t)win;
        int ni = 0, first = 0;
        for (int s = 0; s < 2; s++) {
            for (int i = (int)b; i < 2 * win + 1 - (int)b; i++) {
                if (i == win) continue;
                int cp = S[s].pos - win + i;
                if (cp < 0) continue;
                if (cp >= S[s].len) break;
                in_row[ni++] = s * MB_MAX_SENT + S[s].slot[cp];
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
#define ROW(i) (in_row[i] < MB_MAX_SENT ? S[0].cache + (size_t)in_row[i] * d \
                                        : S[1].cache + (size_t)(in_row[i] - MB_MAX_SENT) * d)
        for (int o = 0; o < O; o++)
            for (int i = 0; i < I; i++) {
                const float *x = outs + (size_t)o * d, *y = ROW(i);
                const float f = split_dot(x, y, d);
                int label = i < first ? (o == 0) : (o == O - 1);
                gm[o * MI + i] = grad32(f, label, c->exp_table, alpha) * (float)out_meta[o];
            }
        for (int k = 0; k < d; k++) {
            for (int o = 0; o < O; o++) {
                float acc = 0.f;
                for (int i = 0; i < I; i++) acc = fmaf(gm[o * MI + i], ROW(i)[k], acc);
                md[o] = acc;
            }
            for (int i = 0; i < I; i++) {
                float acc = 0.f;
                for (int o = 0; o < O; o++) acc = fmaf(gm[o * MI + i], outs[(size_t)o * d + k], acc);
                ROW(i)[k] = ROW(i)[k] + acc;
            }
            float *t1 = syn1 + (size_t)out_word[0] * d + k, *t2 = syn1 + (size_t)out_word[O - 1] * d + k;
            *t1 = *t1 + md[0];
            *t2 = *t2 + md[O - 1];
            for (int o = 1; o < O - 1; o++) {
                float *x = pool_cur + (size_t)out_slot[o] * d + k;
                *x = *x + md[o];
            }
        }
#undef ROW
        step++;
        S[0].pos++;
        S[1].pos++;
        for (int s = 0; s < 2; s++)
            if (S[s].pos >= S[s].len) { mb32_flush(c, &S[s], syn0); S[s].len = 0; train_sen_num++; }
        if (train_sen_num >= 2) {
            for (int r = 0; r < np; r++)
                for (int k = 0; k < d; k++) {
                    float *x = syn1 + (size_t)pool_word[r] * d + k;
                    *x = *x + (pool_cur[(size_t)r * d + k] - pool_init[(size_t)r * d + k]);
                }
            change_neg = 1;
            pool_loaded = 0;
            train_sen_num = 0;
        }
    }
    for (int s = 0; s < 2; s++) if (S[s].len) mb32_flush(c, &S[s], syn0);
    if (pool_loaded)
        for (int r = 0; r < np; r++)
            for (int k = 0; k < d; k++) {
                float *x = syn1 + (size_t)pool_word[r] * d + k;
                *x = *x + (pool_cur[(size_t)r * d + k] - pool_init[(size_t)r * d + k]);
            }
    free(S); free(pool_word); free(pool_slot); free(pool_cur); free(pool_init); free(outs); free(gm); free(md);
    return 0;
}
