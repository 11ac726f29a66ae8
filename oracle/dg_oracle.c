/*
 * CPU restatement of the reference's walk hot path.  TEST INFRASTRUCTURE ONLY
 * (see dg_oracle.h).  Every function cites the reference lines it follows.
 * Compiled with -ffp-contract=off: each FP64 operation is one IEEE rounding,
 * in the order the reference's source writes it.
 */
#include "dg_oracle.h"
#include "philox.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define DGO_RAND_MAX 2147483647

/* ---------------------------------------------------------------- CSR ---- */

/* graph.hpp:642-824 with one partition: doubling (671-686) writes record i at
 * 2i and its transpose at 2i+1; degrees count sources (694-717); the shuffle to
 * the single partition keeps record order (shuffle_edges, 542-640); the CSR
 * buckets records by source in that order (build_edge_container, 509-540). */
int dgo_csr_build(const dgo_edge *edges, uint64_t n_edges, uint32_t v_num, int undirected, dgo_csr *out) {
    memset(out, 0, sizeof(*out));
    uint64_t m = undirected ? 2 * n_edges : n_edges;
    for (uint64_t i = 0; i < n_edges; i++)
        if (edges[i].src >= v_num || edges[i].dst >= v_num) return -1;
    out->v_num = v_num;
    out->m = m;
    out->offsets = (uint64_t *)calloc((size_t)v_num + 1, sizeof(uint64_t));
    out->nbr = (uint32_t *)malloc((size_t)(m ? m : 1) * sizeof(uint32_t));
    out->data = (float *)malloc((size_t)(m ? m : 1) * sizeof(float));
    out->out_deg = (uint32_t *)calloc(v_num, sizeof(uint32_t));
    out->in_deg = (uint32_t *)calloc(v_num, sizeof(uint32_t));
    if (!out->offsets || !out->nbr || !out->data || !out->out_deg || !out->in_deg) return -2;
    for (uint64_t i = 0; i < n_edges; i++) {
        out->out_deg[edges[i].src]++;
        out->in_deg[edges[i].dst]++;
        if (undirected) {
            out->out_deg[edges[i].dst]++;
            out->in_deg[edges[i].src]++;
        }
    }
    for (uint32_t v = 0; v < v_num; v++) out->offsets[v + 1] = out->offsets[v] + out->out_deg[v];
    uint64_t *cursor = (uint64_t *)malloc((size_t)v_num * sizeof(uint64_t) + 8);
    memcpy(cursor, out->offsets, (size_t)v_num * sizeof(uint64_t));
    for (uint64_t i = 0; i < n_edges; i++) {
        const dgo_edge *e = &edges[i];
        uint64_t at = cursor[e->src]++;
        out->nbr[at] = e->dst;
        out->data[at] = e->data;
        if (undirected) {
            at = cursor[e->dst]++;
            out->nbr[at] = e->src;
            out->data[at] = e->data;
        }
    }
    free(cursor);
    return 0;
}

void dgo_csr_free(dgo_csr *g) {
    free(g->offsets); free(g->nbr); free(g->data); free(g->out_deg); free(g->in_deg);
    memset(g, 0, sizeof(*g));
}

/* ------------------------------------------------------- Correlation ---- */

typedef struct { double H, S, EH, ES, EHS, EHH, ESS, N, R; } dgo_corr;

/* Correlation::SnSn_div_Snp1Snp1, walk.hpp:284-289 */
static double sn_ratio(double Sn, double k) {
    double Snp1 = Sn + k;
    return pow(Sn / Snp1, Sn) * pow(1.0 / Snp1, k);
}

/* Correlation::FjFj_div_FiFi, walk.hpp:291-295 */
static double fj_ratio(double fi, double k) {
    double fj = fi + k;
    return pow(fj / fi, fi) * pow(fj, k);
}

/* Correlation::iterateHn, walk.hpp:297-304: the log2 argument is a function of
 * the two small integers (Sn, fi) only. */
static double entropy_term(double Sn, double fi) {
    return fi == 0 ? log2(sn_ratio(Sn, 1.0)) : log2(sn_ratio(Sn, 1.0) * fj_ratio(fi, 1.0));
}

/* Correlation::iterate, walk.hpp:317-354, step_k = 1 */
static void corr_iterate(dgo_corr *c, double fi, dgo_walk_stats *st) {
    double t = entropy_term(c->S, fi);
    double Hnp1 = (c->S * c->H - t) / (c->S + 1.0);
    double Snp1 = c->S + 1.0;
    double Np1 = c->N + 1.0;
    double EH = c->EH + (Hnp1 - c->EH) / Np1;
    double ES = c->ES + (Snp1 - c->ES) / Np1;
    double EHS = c->EHS + (Hnp1 * Snp1 - c->EHS) / Np1;
    double EHH = c->EHH + (Hnp1 * Hnp1 - c->EHH) / Np1;
    double ESS = c->ESS + (Snp1 * Snp1 - c->ESS) / Np1;
    double DH = EHH - EH * EH;
    double DS = ESS - ES * ES;
    double e = EHS - EH * ES;
    c->R = e == 0.0 ? 0.0 : e / sqrt(DH * DS);
    c->H = Hnp1; c->S = Snp1; c->EH = EH; c->ES = ES; c->EHS = EHS; c->EHH = EHH; c->ESS = ESS; c->N = Np1;
    if (st && pow(c->R, 2) != c->R * c->R) st->pow_sq_mismatch++;
}

/* Termination test, walk.hpp:868-872 / 979-984 / 1011-1016 (R = 0.999, walk.hpp:24). */
static int corr_stop(const dgo_corr *c, uint32_t step, uint32_t min_len) {
    return step > min_len && (pow(c->R, 2) < 0.999 || c->R < 0);
}

/* ------------------------------------------------------------- walks ---- */

typedef struct { uint32_t *v; uint64_t n, cap; } dgo_vec;

static int vec_push(dgo_vec *a, uint32_t x) {
    if (a->n == a->cap) {
        uint64_t nc = a->cap ? 2 * a->cap : 1024;
        uint32_t *nv = (uint32_t *)realloc(a->v, (size_t)nc * sizeof(uint32_t));
        if (!nv) return -1;
        a->v = nv; a->cap = nc;
    }
    a->v[a->n++] = x;
    return 0;
}

/* Prior visits of v in the current walk: the unordered_map counter of
 * walk.hpp:816/849/965/994 (post-increment, so the value before this visit). */
static double prior_visits(const uint32_t *walk, uint64_t len, uint32_t v) {
    uint32_t c = 0;
    for (uint64_t i = 0; i < len; i++) c += walk[i] == v;
    return (double)c;
}

/* One walker to completion, walk.hpp:845-1024 with every vertex local. */
static int walk_one(const dgo_csr *g, const dgo_walk_params *p, uint32_t round, uint32_t wid,
                    dgo_vec *out, dgo_walk_stats *st) {
    uint64_t base = out->n;
    uint32_t cur = wid % g->v_num;                       /* walk.hpp:505 */
    if (vec_push(out, cur)) return -1;                   /* step-0 footprint, walk.hpp:667 */
    dgo_corr c = {0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 1.0, 1.0, 1.0}; /* walk.hpp:853-855 */
    uint32_t step = 0;
    uint32_t attempt = 0;
    for (;;) {
        uint32_t deg = g->out_deg[cur];
        if (deg == 0) break;                             /* walk.hpp:887-892 */
        uint32_t slot, k = 0;
        if (p->rng_mode == DGO_RNG_PHILOX) {
            dgo_u32x4 ctr = {{attempt, wid, round, DGO_WALK_TAG}};
            dgo_u32x4 x = dgo_philox4x32_10(ctr, (uint32_t)p->seed, (uint32_t)(p->seed >> 32));
            slot = dgo_scale64(((uint64_t)x.v[1] << 32) | x.v[0], deg);
            k = x.v[2] & 0x7fffffffu;
        } else {
            slot = p->cand_cb(p->cb_ctx, deg);            /* walk.hpp:899 */
        }
        attempt++;
        if (st) st->draws++;
        uint64_t row = g->offsets[cur];
        uint64_t e = row + slot;
        if (deg == 2 && g->nbr[row] == cur) break;       /* walk.hpp:900-902 */
        if (step == 0 && g->nbr[e] == cur) continue;     /* walk.hpp:904-906 */
        if (p->rng_mode != DGO_RNG_PHILOX) k = p->acc_cb(p->cb_ctx); /* walk.hpp:928 */
        int cn = (int)g->data[e];                        /* walk.hpp:920 */
        double pr = (double)k / (double)DGO_RAND_MAX;
        int sd = (int)g->out_deg[cur];
        int dd = (int)g->out_deg[g->nbr[e]];
        int hi = sd > dd ? sd : dd, lo = sd < dd ? sd : dd;
        double p_accept = (1 / ((double)(sd - cn))) * ((double)hi) / lo; /* walk.hpp:933 */
        double p_norm = tanh(p_accept);                  /* walk.hpp:934 */
        int trace = p_norm <= pr;                        /* walk.hpp:938-942 */
        if (st) {
            if (trace) st->traces++;
            if (fabs(p_norm - pr) < 1e-12) st->near_ties++;
        }
        uint32_t dst = g->nbr[e];
        step++;                                          /* walk.hpp:961-977 */
        double fi = prior_visits(out->v + base, out->n - base, dst);
        if (vec_push(out, dst)) return -1;
        corr_iterate(&c, fi, st);
        if (corr_stop(&c, step, p->min_len)) break;
        if (trace) {                                     /* walk.hpp:986-1017 */
            step++;
            fi = prior_visits(out->v + base, out->n - base, cur);
            if (vec_push(out, cur)) return -1;
            corr_iterate(&c, fi, st);
            if (corr_stop(&c, step, p->min_len)) break;
        } else {
            cur = dst;                                   /* walk.hpp:1018-1023 */
        }
    }
    if (st) {
        uint64_t len = out->n - base;
        st->footprints += len;
        st->steps += len - 1;
        if (len > st->max_len) st->max_len = (uint32_t)len;
    }
    return 0;
}

int dgo_walk_round(const dgo_csr *g, const dgo_walk_params *p, uint32_t round, uint32_t n_walkers,
                   dgo_paths *out, dgo_walk_stats *stats) {
    memset(out, 0, sizeof(*out));
    if (g->v_num == 0) return -1;
    if (p->rng_mode == DGO_RNG_CALLBACK && (!p->cand_cb || !p->acc_cb)) return -1;
    dgo_vec v = {0, 0, 0};
    out->offsets = (uint64_t *)malloc(((size_t)n_walkers + 1) * sizeof(uint64_t));
    if (!out->offsets) return -2;
    out->offsets[0] = 0;
    for (uint32_t w = 0; w < n_walkers; w++) {
        if (walk_one(g, p, round, w, &v, stats)) { free(v.v); return -2; }
        out->offsets[w + 1] = v.n;
    }
    out->n_walks = n_walkers;
    out->total = v.n;
    out->verts = v.v ? v.v : (uint32_t *)malloc(4);
    return 0;
}

/* The walks of selected walker ids only (same per-walker semantics; Philox mode),
 * for spot checks of full-size rounds. */
int dgo_walk_ids(const dgo_csr *g, const dgo_walk_params *p, uint32_t round, const uint32_t *ids, uint32_t n_ids,
                 dgo_paths *out, dgo_walk_stats *stats) {
    memset(out, 0, sizeof(*out));
    if (g->v_num == 0 || p->rng_mode != DGO_RNG_PHILOX) return -1;
    dgo_vec v = {0, 0, 0};
    out->offsets = (uint64_t *)malloc(((size_t)n_ids + 1) * sizeof(uint64_t));
    if (!out->offsets) return -2;
    out->offsets[0] = 0;
    for (uint32_t i = 0; i < n_ids; i++) {
        if (walk_one(g, p, round, ids[i], &v, stats)) { free(v.v); return -2; }
        out->offsets[i + 1] = v.n;
    }
    out->n_walks = n_ids;
    out->total = v.n;
    out->verts = v.v ? v.v : (uint32_t *)malloc(4);
    return 0;
}

void dgo_paths_free(dgo_paths *p) {
    free(p->offsets); free(p->verts);
    memset(p, 0, sizeof(*p));
}

/* PathSet::dump, path.hpp:67-119 (one segment: one worker thread). */
int dgo_write_walks(const char *path, const dgo_paths *p) {
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    for (uint32_t w = 0; w < p->n_walks; w++) {
        for (uint64_t i = p->offsets[w]; i < p->offsets[w + 1]; i++) fprintf(f, " %u", p->verts[i]);
        fprintf(f, "\n");
    }
    return fclose(f) ? -1 : 0;
}

/* walk.hpp:694-725 */
double dgo_relative_entropy(const uint32_t *out_deg, const uint32_t *freq, uint32_t v_num) {
    uint64_t words_sum = 0, degree_sum = 0;
    for (uint32_t i = 0; i < v_num; i++) { words_sum += freq[i]; degree_sum += out_deg[i]; }
    double h = 0.0;
    for (uint32_t i = 0; i < v_num; i++) {
        double pi = (double)out_deg[i] / degree_sum;
        double qi = (double)freq[i] / words_sum;
        h += pi * (log(pi) - log(qi));
    }
    return h;
}

/* Smallest k with t <= k / 2147483647.0, i.e. the first Philox draw for which
 * the reference's `p_norm <= p` holds (walk.hpp:928-942). */
static uint32_t threshold_of(double t) {
    if (t != t) return 0x80000000u;          /* NaN: never <= p */
    if (t <= 0.0) return 0;
    if (t > 1.0) return 0x80000000u;
    double guess = ceil(t * (double)DGO_RAND_MAX);
    int64_t k = (int64_t)guess;
    if (k > DGO_RAND_MAX) k = DGO_RAND_MAX;
    while (k > 0 && t <= (double)(k - 1) / (double)DGO_RAND_MAX) k--;
    while (k <= DGO_RAND_MAX && !(t <= (double)k / (double)DGO_RAND_MAX)) k++;
    return (uint32_t)k;
}

void dgo_thresholds(const dgo_csr *g, uint32_t *thr) {
    for (uint32_t v = 0; v < g->v_num; v++) {
        int sd = (int)g->out_deg[v];
        for (uint64_t e = g->offsets[v]; e < g->offsets[v + 1]; e++) {
            int cn = (int)g->data[e];
            int dd = (int)g->out_deg[g->nbr[e]];
            int hi = sd > dd ? sd : dd, lo = sd < dd ? sd : dd;
            double p_accept = (1 / ((double)(sd - cn))) * ((double)hi) / lo;
            thr[e] = threshold_of(tanh(p_accept));
        }
    }
}

uint64_t dgo_entropy_table_size(uint32_t max_sn) {
    return (uint64_t)max_sn * (max_sn + 1) / 2 + max_sn;
}

void dgo_entropy_table(uint32_t max_sn, double *out) {
    for (uint32_t s = 1; s <= max_sn; s++)
        for (uint32_t f = 0; f <= s; f++)
            out[(uint64_t)s * (s + 1) / 2 + f - 1] = entropy_term((double)s, (double)f);
}

/* Known-answer hook for the Philox restatement. */
void dgo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    dgo_u32x4 c = {{ctr[0], ctr[1], ctr[2], ctr[3]}};
    dgo_u32x4 r = dgo_philox4x32_10(c, key[0], key[1]);
    for (int i = 0; i < 4; i++) out[i] = r.v[i];
}
