/*
 * Bit-exact model of the staged-rows plain kernel (sgns_plain_pipe_kernel) run by
 * ONE warp, FP32 rows or BF16 rows with FP32 masters.  TEST INFRASTRUCTURE ONLY
 * (see dg_oracle.h).
 *
 * The kernel trains skip-gram pairs in the plain rule's order (word2vec.cu:358-397,
 * dgo_sgns_plain_f32) but copies the rows of pair m + S - 1 (its context row and
 * its negatives' rows) into shared memory while pair m trains.  With one warp
 * the result is fixed by program order: the copy of pair m is taken after the
 * updates of pairs 0 .. m - S (and before those of m - S + 1 ..), every later
 * update lands on the row itself.  The model replays exactly that:
 *  - pair m's context row and negative rows are the values at its copy time;
 *  - a context word used by one of the warp's previous S pairs is read from that
 *    pair's updated copy (the kernel's history slots, kept across walks);
 *  - the centre's output row is read when the centre starts and written back
 *    when it ends;
 *  - FP32 rows and masters receive updates as additions (the kernel's vector
 *    atomics); a BF16 row is overwritten with the warp's updated copy, rounded
 *    stochastically: 16 noise bits added below the kept mantissa, then
 *    truncated, the noise words drawn per row write from a salt exactly as the
 *    kernel's BfRows::store_bits does (one multiply-xorshift of the salt, then
 *    one LCG step per two elements).  Infinities and NaN are not expected.
 */
#include "dg_oracle.h"
#include "philox.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define EXP_TABLE_SIZE 1000
#define MAX_EXP 6
#define PIPE_SENTENCE 64 /* kPipeSentence */
#define FAST_NEG 8       /* kFastNeg */

static uint32_t pword(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed, int word) {
    dgo_u32x4 ctr = {{c0, c1, c2, c3}};
    dgo_u32x4 x = dgo_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    return x.v[word];
}

static uint32_t bf_mix(uint32_t h) {
    h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
    return h;
}

static float bits_f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t f_bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* FP32 -> BF16 with 16 noise bits added below the kept mantissa, truncated;
 * returned as the FP32 value of the BF16 result. */
static float bf16_sr(float x, uint32_t noise16) {
    uint32_t u = f_bits(x);
    if ((u & 0x7F800000u) != 0x7F800000u) u += noise16 & 0xFFFFu;
    return bits_f(u & 0xFFFF0000u);
}

static float grad(float f, int label, const float *t, float alpha) {
    if (f > MAX_EXP) return (label - 1) * alpha;
    if (f < -MAX_EXP) return label * alpha;
    return (label - t[(int)((f + MAX_EXP) * (EXP_TABLE_SIZE / MAX_EXP / 2))]) * alpha;
}

/* Warp dot: lane l holds columns [l*v, l*v+v), fused chain, xor butterfly. */
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

/* The kernel's write of an updated row: masters / FP32 rows get `delta` added;
 * a BF16 row gets `value` rounded with the per-lane noise of salt[lane]. */
static void row_update(const dgo_pipe_cfg *c, float *row, int32_t id, const float *delta, const float *value,
                       const uint32_t *salt) {
    const int d = c->d, v = d / 32;
    if (!c->bf16 || (uint32_t)id < c->n_master) {
        for (int i = 0; i < d; i++) row[i] = row[i] + delta[i];
        return;
    }
    for (int l = 0; l < 32; l++) {
        uint32_t x = salt[l] * 0x9E3779B1u;   /* the kernel's per-write noise word */
        x ^= x >> 16;
        for (int i = 0; i < v; i += 2) {
            row[l * v + i] = bf16_sr(value[l * v + i], x & 0xFFFFu);
            row[l * v + i + 1] = bf16_sr(value[l * v + i + 1], x >> 16);
            x = x * 0x9E3779B1u + 0x7F4A7C15u;
        }
    }
}

typedef struct {
    uint32_t q, s; /* centre, window slot */
    float *ctx;    /* staged context row */
    float *neg;    /* staged negative rows, NS x d */
} pipe_pair;

int dgo_sgns_pipe(const dgo_pipe_cfg *c, const uint64_t *offsets, const uint32_t *verts, uint32_t n_walks,
                  float *rows_in, float *rows_out, dgo_sgns_stats *st) {
    const int d = c->d, w = c->window, S = c->stages;
    const int NS = (c->negative == 5 && c->vocab_size > 1) ? 5 : FAST_NEG;
    const int neg = c->vocab_size > 1 ? c->negative : 0;
    const float alpha = c->alpha;
    if (!(d == 64 || d == 128) || S < 2 || S > 4 || neg > FAST_NEG || w < 1 || w > 15 || (c->bf16 && d != 128))
        return -1;
    const uint32_t key = c->seed_lo ^ bf_mix(c->pass * 0x9E3779B9u + 0x2F6B3A91u);
    const int npairs_max = PIPE_SENTENCE * 2 * 15;
    pipe_pair *pairs = (pipe_pair *)calloc(npairs_max, sizeof(pipe_pair));
    float *stage = (float *)malloc((size_t)npairs_max * (1 + NS) * d * sizeof(float));
    float *hist = (float *)malloc((size_t)S * d * sizeof(float));
    float *pos = (float *)malloc(d * 4), *pos0 = (float *)malloc(d * 4), *e = (float *)malloc(d * 4);
    float *l1 = (float *)malloc(d * 4), *upd = (float *)malloc(d * 4), *r = (float *)malloc(d * 4);
    float *v1 = (float *)malloc(d * 4);
    int32_t *hw = (int32_t *)malloc(S * sizeof(int32_t));
    int32_t *tb = (int32_t *)malloc((size_t)npairs_max * FAST_NEG * sizeof(int32_t));
    int32_t sen[PIPE_SENTENCE];
    uint32_t salt[32], base[32];
    int rc = 0;
    if (!pairs || !stage || !hist || !pos || !pos0 || !e || !l1 || !upd || !r || !v1 || !hw || !tb) {
        rc = -2;
        goto done;
    }
    for (int k = 0; k < S; k++) hw[k] = -1;
    uint32_t mm = 0;
    for (uint32_t wk = 0; wk < n_walks; wk++) {
        uint32_t len = (uint32_t)(offsets[wk + 1] - offsets[wk]);
        if (len > PIPE_SENTENCE) len = PIPE_SENTENCE;
        uint32_t n = 0;
        for (uint32_t i = 0; i < len; i++) {
            const int32_t word = c->v2w[verts[offsets[wk] + i]];
            if (word < 0) continue;
            if ((pword(i, wk, c->pass, DGO_SUB_TAG, c->seed, 0) & 0xFFFFu) >= c->keep_thr[word]) continue;
            sen[n++] = word;
        }
        if (st) { st->words += len; st->trained += n; }
        if (n < 2) continue;
        /* The walk's pairs in training order, with their negatives. */
        int np = 0;
        for (uint32_t q = 0; q < n; q++) {
            const uint32_t b = pword(q, wk, c->pass, DGO_WIN_TAG, c->seed, 0) % (uint32_t)w;
            const uint32_t wq = (uint32_t)w > q ? (uint32_t)w - q : 0u;
            const uint32_t lo = b > wq ? b : wq;
            const uint32_t hi0 = 2 * (uint32_t)w + 1 - b, hi1 = n + (uint32_t)w - q, hi = hi0 < hi1 ? hi0 : hi1;
            for (uint32_t s = lo; s < hi; s++) {
                if (s == (uint32_t)w) continue;
                pairs[np].q = q;
                pairs[np].s = s;
                for (int j = 0; j < NS; j++) {
                    int32_t t = -1;
                    if (j < neg) {
                        const uint32_t rr = pword(q * (2 * w + 1) + s, wk, c->pass,
                                                  DGO_NEG_TAG + (uint32_t)(j >> 2), c->seed, j & 3);
                        t = c->table[rr % c->table_size];
                        if (t == 0) t = (int32_t)((rr >> 8) % (c->vocab_size - 1) + 1);
                    }
                    tb[np * FAST_NEG + j] = t;
                }
                np++;
            }
        }
        if (st) st->pairs += (uint64_t)np;
        /* Copy of pair m: its context row and negative rows as they are now. */
#define COPY(m)                                                                                                  \
    do {                                                                                                         \
        pipe_pair *pp_ = &pairs[m];                                                                              \
        pp_->ctx = stage + (size_t)(m) * (1 + NS) * d;                                                           \
        pp_->neg = pp_->ctx + d;                                                                                 \
        memcpy(pp_->ctx, rows_in + (size_t)sen[pp_->q - w + pp_->s] * d, d * 4);                                 \
        for (int j_ = 0; j_ < neg; j_++)                                                                         \
            memcpy(pp_->neg + (size_t)j_ * d, rows_out + (size_t)tb[(m) * FAST_NEG + j_] * d, d * 4);            \
    } while (0)
        for (int m = 0; m < S - 1 && m < np; m++) COPY(m);
        int32_t word = sen[0];
        memcpy(pos, rows_out + (size_t)word * d, d * 4);
        memcpy(pos0, pos, d * 4);
        for (int m = 0; m < np; m++) {
            if (m + S - 1 < np) COPY(m + S - 1);
            const pipe_pair *P = &pairs[m];
            const uint32_t q = P->q, s = P->s;
            for (int l = 0; l < 32; l++)
                base[l] = bf_mix(key ^ bf_mix(wk * 0x01000193u + q * 0x2545F491u) ^ (uint32_t)l * 0x85EBCA6Bu);
            const int32_t last = sen[q - w + s];
            memcpy(l1, P->ctx, d * 4);
            for (int k = S - 1; k >= 0; k--)   /* the newest match wins */
                if (hw[k] == last) memcpy(l1, hist + (size_t)((mm + S - 1 - k) % S) * d, d * 4);
            const int32_t *t = tb + m * FAST_NEG;
            for (int i = 0; i < d; i++) e[i] = 0.f;
            {   /* the positive: the centre's output row, in registers */
                const float g = grad(dot_warp(l1, pos, d), 1, c->exp_table, alpha);
                for (int i = 0; i < d; i++) {
                    e[i] = fmaf(g, pos[i], e[i]);
                    const float u = g * l1[i];
                    pos[i] = pos[i] + u;
                }
            }
            /* Negatives in order, each from its staged copy; a repeat within the
             * pair sees the earlier copy's update. */
            for (int j = 0; j < neg; j++) {
                if (t[j] == word) continue;
                float *rj = P->neg + (size_t)j * d;
                memcpy(r, rj, d * 4);
                const float g = grad(dot_warp(l1, r, d), 0, c->exp_table, alpha);
                for (int i = 0; i < d; i++) {
                    e[i] = fmaf(g, r[i], e[i]);
                    upd[i] = g * l1[i];
                    r[i] = r[i] + upd[i];
                }
                for (int l = 0; l < 32; l++) salt[l] = base[l] + (uint32_t)t[j] * 0x27D4EB2Fu + s * 16u + (uint32_t)j;
                row_update(c, rows_out + (size_t)t[j] * d, t[j], upd, r, salt);
                for (int k = j + 1; k < neg; k++)
                    if (t[k] == t[j]) memcpy(P->neg + (size_t)k * d, r, d * 4);
            }
            /* The context row: e added (FP32 rows, masters) or l1 + e stored (BF16). */
            for (int i = 0; i < d; i++) v1[i] = l1[i] + e[i];
            for (int l = 0; l < 32; l++) salt[l] = base[l] + (uint32_t)last * 0x165667B1u + s * 16u + 15u;
            row_update(c, rows_in + (size_t)last * d, last, e, v1, salt);
            memcpy(hist + (size_t)(mm % S) * d, v1, d * 4);
            for (int k = S - 1; k > 0; k--) hw[k] = hw[k - 1];
            hw[0] = last;
            mm++;
            if (m + 1 == np || pairs[m + 1].q != q) {   /* the centre ends */
                for (int i = 0; i < d; i++) upd[i] = pos[i] - pos0[i];
                for (int l = 0; l < 32; l++) salt[l] = base[l] + (uint32_t)word * 0xD3A2646Cu + 0x5BD1E995u;
                row_update(c, rows_out + (size_t)word * d, word, upd, pos, salt);
                if (m + 1 < np) {
                    word = sen[pairs[m + 1].q];
                    memcpy(pos, rows_out + (size_t)word * d, d * 4);
                    memcpy(pos0, pos, d * 4);
                }
            }
        }
#undef COPY
    }
done:
    free(pairs); free(stage); free(hist); free(pos); free(pos0); free(e); free(l1); free(upd); free(r); free(v1);
    free(hw); free(tb);
    return rc;
}
