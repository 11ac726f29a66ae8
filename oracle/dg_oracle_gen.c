/*
 * CPU restatement of the device graph generator and link-prediction split
 * (gdistger-re_b200/csrc/dg_gen.cu) -- test infrastructure only, the checker of
 * dg_edges_chung_lu / dg_edges_split at sizes the CPU finishes in seconds.
 *
 * The reference has no generator (its graphs come from files) and splits on the
 * host with src/tools/gtrain.cpp:226-386; the split rule restated here is that
 * tool's hold-out rule in the parallel form the device code uses.
 */
#include "dg_oracle.h"
#include "philox.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define GEN_TAG 0x4347454Eu
#define ISO_TAG 0x4349534Fu
#define NEG_TAG 0x4C504E47u
#define NO_EDGE (~0ull)

static uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

typedef struct {
    uint32_t n, half, mask;
    uint64_t key;
} perm_t;

static perm_t make_perm(uint32_t n, uint64_t seed) {
    uint32_t bits = 2;
    while (bits < 32 && (1ull << bits) < n) bits++;
    if (bits & 1) bits++;
    perm_t p = {n, bits / 2, (1u << (bits / 2)) - 1, mix64(seed ^ 0x5045524D5045524Dull)};
    return p;
}

static uint32_t perm_apply(const perm_t *p, uint32_t x) {
    do {
        uint32_t l = x >> p->half, r = x & p->mask;
        for (uint32_t k = 0; k < 4; k++) {
            const uint32_t f = (uint32_t)mix64((uint64_t)r ^ (p->key + (uint64_t)k * 0x9E3779B97F4A7C15ull)) & p->mask;
            const uint32_t t = l ^ f;
            l = r;
            r = t;
        }
        x = (l << p->half) | r;
    } while (x >= p->n);
    return x;
}

static double uniform53(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

/* First i with cdf[i] > u, clamped to n - 1 (plain binary search over the whole CDF). */
static uint32_t sample(const double *cdf, uint32_t n, double u) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] > u) hi = mid;
        else lo = mid + 1;
    }
    return lo < n ? lo : n - 1;
}

static int cmp_u64(const void *a, const void *b) {
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

static uint64_t sort_unique(uint64_t *k, uint64_t n) {
    qsort(k, n, sizeof(uint64_t), cmp_u64);
    uint64_t w = 0;
    for (uint64_t i = 0; i < n; i++) {
        if (k[i] == NO_EDGE) break;
        if (w == 0 || k[w - 1] != k[i]) k[w++] = k[i];
    }
    return w;
}

static uint64_t pair_key(uint32_t a, uint32_t b) {
    return a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
}

/* Expected degrees, capped and rescaled, then the normalised CDF -- sequential
 * double sums in the same order as the library's host code. */
static void cdf_of(uint32_t n, uint64_t m, double beta, double cap, double *cdf) {
    double *w = (double *)malloc(sizeof(double) * n);
    const double gamma = 1.0 / (beta - 1.0);
    double total = 0.0;
    for (uint32_t i = 0; i < n; i++) {
        w[i] = pow((double)i + 1.0, -gamma);
        total += w[i];
    }
    const double target = 2.0 * (double)m;
    for (uint32_t i = 0; i < n; i++) w[i] *= target / total;
    if (cap > 0) {
        for (int it = 0; it < 8; it++) {
            total = 0.0;
            for (uint32_t i = 0; i < n; i++) {
                w[i] = w[i] < cap ? w[i] : cap;
                total += w[i];
            }
            for (uint32_t i = 0; i < n; i++) w[i] *= target / total;
        }
        for (uint32_t i = 0; i < n; i++) w[i] = w[i] < cap ? w[i] : cap;
    }
    double acc = 0.0;
    for (uint32_t i = 0; i < n; i++) {
        acc += w[i];
        cdf[i] = acc;
    }
    for (uint32_t i = 0; i < n; i++) cdf[i] /= acc;
    free(w);
}

/* keys must hold m + n entries; returns the number of unique undirected pairs. */
uint64_t dgo_chung_lu(uint32_t n, uint64_t m, double beta, double cap, uint64_t seed, uint64_t *keys) {
    double *cdf = (double *)malloc(sizeof(double) * n);
    cdf_of(n, m, beta, cap, cdf);
    const perm_t perm = make_perm(n, seed);
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (uint64_t j = 0; j < m; j++) {
        dgo_u32x4 c = {{(uint32_t)j, (uint32_t)(j >> 32), 0u, GEN_TAG}};
        const dgo_u32x4 x = dgo_philox4x32_10(c, k0, k1);
        const uint32_t s = sample(cdf, n, uniform53(x.v[0], x.v[1]));
        const uint32_t d = sample(cdf, n, uniform53(x.v[2], x.v[3]));
        keys[j] = s == d ? NO_EDGE : pair_key(perm_apply(&perm, s), perm_apply(&perm, d));
    }
    uint64_t e = sort_unique(keys, m);
    uint32_t *deg = (uint32_t *)calloc(n, sizeof(uint32_t));
    for (uint64_t i = 0; i < e; i++) {
        deg[keys[i] >> 32]++;
        deg[(uint32_t)keys[i]]++;
    }
    uint64_t add = 0;
    for (uint32_t v = 0; v < n; v++) {
        if (deg[v]) continue;
        dgo_u32x4 c = {{v, 0u, 1u, ISO_TAG}};
        const dgo_u32x4 x = dgo_philox4x32_10(c, k0, k1);
        uint32_t p = perm_apply(&perm, sample(cdf, n, uniform53(x.v[0], x.v[1])));
        if (p == v) p = (v + 1) % n;
        keys[e + add++] = pair_key(v, p);
    }
    if (add) e = sort_unique(keys, e + add);
    free(deg);
    free(cdf);
    return e;
}

float dgo_edge_data(uint64_t key, uint64_t seed, int weighted) {
    if (!weighted) return 1.0f;
    const uint64_t ds = mix64(seed ^ 0x4441544144415441ull);
    return 1.0f - (float)(mix64(key ^ ds) >> 40) * (1.0f / 16777216.0f);
}

static int has_key(const uint64_t *keys, uint64_t n, uint64_t key) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (keys[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && keys[lo] == key;
}

/* Split of sorted unique keys[0, n): writes the kept keys back in order
 * (returns their count), the held-out pairs to pos_u/pos_v (key order) and the
 * negatives to neg_u/neg_v; *n_pos = *n_neg = held-out count.  Arrays sized n. */
uint64_t dgo_lp_split(uint64_t *keys, uint64_t n, uint32_t v_num, double frac, uint64_t seed, uint32_t *pos_u,
                      uint32_t *pos_v, uint32_t *neg_u, uint32_t *neg_v, uint64_t *n_pos) {
    const uint64_t hseed = mix64(seed ^ 0x53504C4953504C49ull);
    uint32_t *deg = (uint32_t *)calloc(v_num, sizeof(uint32_t));
    uint32_t *cand = (uint32_t *)calloc(v_num, sizeof(uint32_t));
    unsigned char *isc = (unsigned char *)malloc(n ? n : 1);
    for (uint64_t i = 0; i < n; i++) {
        const uint32_t a = (uint32_t)(keys[i] >> 32), b = (uint32_t)keys[i];
        deg[a]++;
        deg[b]++;
        isc[i] = (double)(mix64(keys[i] ^ hseed) >> 11) * (1.0 / 9007199254740992.0) < frac;
        if (isc[i]) {
            cand[a]++;
            cand[b]++;
        }
    }
    uint64_t np = 0, nk = 0;
    uint64_t *full = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    memcpy(full, keys, sizeof(uint64_t) * n);
    for (uint64_t i = 0; i < n; i++) {
        const uint32_t a = (uint32_t)(full[i] >> 32), b = (uint32_t)full[i];
        if (isc[i] && deg[a] - cand[a] >= 1 && deg[b] - cand[b] >= 1) {
            pos_u[np] = a;
            pos_v[np] = b;
            np++;
        } else {
            keys[nk++] = full[i];
        }
    }
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (uint64_t j = 0; j < np; j++) {
        neg_u[j] = neg_v[j] = 0xFFFFFFFFu;
        for (uint32_t t = 0; t < 64; t++) {
            dgo_u32x4 c = {{(uint32_t)j, (uint32_t)(j >> 32), t, NEG_TAG}};
            const dgo_u32x4 x = dgo_philox4x32_10(c, k0, k1);
            const uint32_t a = (uint32_t)(((uint64_t)x.v[0] * v_num) >> 32);
            const uint32_t b = (uint32_t)(((uint64_t)x.v[1] * v_num) >> 32);
            if (a == b || has_key(full, n, pair_key(a, b))) continue;
            neg_u[j] = a;
            neg_v[j] = b;
            break;
        }
    }
    *n_pos = np;
    free(full);
    free(isc);
    free(cand);
    free(deg);
    return nk;
}
