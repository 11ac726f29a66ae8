// Minibatch SGNS with shared negatives: the update rule of dsgl.hpp
// Train_SGNS_MPI (dsgl.hpp:783-1407) on BF16 rows with FP32 accumulation.
//
// One CTA is one dsgl worker: it owns a contiguous slice of the walks and keeps
// two sentences in flight.  Per step (one position in each sentence):
//   inputs  I <= 2 * 2 * window : context rows of both centres, same shrink b
//                                 (dsgl.hpp:1097-1127), from per-sentence caches;
//   outputs O <= negative + 2   : centre 1, the step's group of the shared
//                                 negative pool (duplicates merged with a count,
//                                 dsgl.hpp:1131-1156), centre 2;
//   corr (O x I) = outputs . inputs^T -> g = (label - sigmoid) * alpha * count,
//   row 0 positive against sentence-1 columns, row O-1 against sentence-2
//   columns (dsgl.hpp:1241-1274);
//   outputs += corr . inputs,  inputs += corr^T . outputs (dsgl.hpp:1290-1311).
//
// The worker's NW warps split the columns: warp w owns the contiguous block
// [w*32*v, (w+1)*32*v), lane l of it v columns (v = size / (32 NW)).  Everything
// but the corr dots is column-local, so the warps only meet once per batch of
// 32 dots: each warp reduces its partial sums with a recursive-halving transpose
// (31 shuffles for 32 sums; lane j ends with dot j, summed in the tree of an xor
// butterfly), the NW partials are added in warp order, and every warp derives
// the same gradients.  Output rows of a step sit in registers.  Sentence caches
// live in shared memory (FP32); the negative pool lives in this worker's slice of
// a global scratch area (FP32).  Caches are written back as deltas when a
// sentence ends (inputs) or after two sentences (pool).  BF16 rows are rounded
// stochastically; the hottest rows (lowest vocabulary ids) are FP32 masters
// updated with atomics.
//
// The contractions are O x I x d = 7 x 40 x 128 per step for the reference
// configuration.  They run on FP32 CUDA cores: the step is a dependent chain of
// row loads, products and cache updates that the next step waits on, bound by
// latency rather than arithmetic, and FP32 fused chains keep the deterministic
// mode bit-exact against the restatement (a tensor core's accumulation order is
// unspecified and its operands would be rounded to BF16 / TF32).
#include "dg_sgns.h"

#include <algorithm>
#include <cmath>
#include <mutex>

namespace dgs {

constexpr int kMbMaxSent = 32;               // tokens per sentence (= cache rows per sentence)
constexpr int kMbHash = 512;                 // pool dedup table (>= 2 x pool capacity)
constexpr uint32_t kMbWinTag = 0x4D425749u;  // "MBWI": window shrink of step s
constexpr uint32_t kMbPoolTag = 0x4D42504Fu; // "MBPO": negative pool sample j of pool p

struct MbArgs {
    float *scratch;            // per worker: pool_cur, pool_init (pool_cap x d each), sent_init (2 x 32 x d)
    uint64_t scratch_stride;   // floats per worker
    uint32_t pool_cap;         // kMbMaxSent * negative
    int max_in;                // 4 * window
    uint32_t smem;             // bytes per worker
};

// Warps per worker for a row size: each lane owns two columns (one for d = 32).
constexpr int mb_warps(int d) { return d >= 64 ? d / 64 : 1; }
// Workers per SM the register budget is sized for (shared memory allows about
// as many): enough residency to reach the staleness bound on large vocabularies.
constexpr int mb_min_blocks(int d) { return d <= 32 ? 16 : d == 64 ? 8 : d == 128 ? 5 : 3; }
// Register cap per thread: the most that mb_min_blocks workers per SM leave.
// Registers are allocated per SM sub-partition (four per SM, 16,384 each), so
// the cap is 16,384 / (32 x the warps one sub-partition holds); size 128: five
// two-warp workers, three warps per sub-partition, 168 registers.
constexpr int mb_max_regs(int d) {
    return 16384 / (32 * ((mb_warps(d) * mb_min_blocks(d) + 3) / 4)) / 8 * 8 > 255
               ? 255
               : 16384 / (32 * ((mb_warps(d) * mb_min_blocks(d) + 3) / 4)) / 8 * 8;
}

__device__ __forceinline__ uint32_t mix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}

// FP32 -> BF16 with stochastic rounding: add 16 random bits below the kept
// mantissa and truncate (unbiased in expectation).
__device__ __forceinline__ __nv_bfloat16 bf16_sr(float x, uint32_t noise) {
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7F800000u) != 0x7F800000u) u += noise & 0xFFFFu;
    return __ushort_as_bfloat16((unsigned short)(u >> 16));
}

// V consecutive columns of one row, owned by one lane.
template <int V>
struct Cols {
    float v[V];
};

template <int V>
__device__ __forceinline__ void ld_cols(const float *p, Cols<V> &c) {
    if constexpr (V % 4 == 0) {
#pragma unroll
        for (int i = 0; i < V; i += 4) {
            const float4 t = *reinterpret_cast<const float4 *>(p + i);
            c.v[i] = t.x; c.v[i + 1] = t.y; c.v[i + 2] = t.z; c.v[i + 3] = t.w;
        }
    } else if constexpr (V == 2) {
        const float2 t = *reinterpret_cast<const float2 *>(p);
        c.v[0] = t.x; c.v[1] = t.y;
    } else {
        c.v[0] = p[0];
    }
}

template <int V>
__device__ __forceinline__ void st_cols(float *p, const Cols<V> &c) {
    if constexpr (V % 4 == 0) {
#pragma unroll
        for (int i = 0; i < V; i += 4)
            *reinterpret_cast<float4 *>(p + i) = make_float4(c.v[i], c.v[i + 1], c.v[i + 2], c.v[i + 3]);
    } else if constexpr (V == 2) {
        *reinterpret_cast<float2 *>(p) = make_float2(c.v[0], c.v[1]);
    } else {
        p[0] = c.v[0];
    }
}

// Rows of a table: BF16 storage, with FP32 masters for rows < n_master.
template <int V>
struct MbRows {
    __nv_bfloat16 *bf;
    float *master;
    uint32_t n_master;
    int d;
    __device__ __forceinline__ void get(int32_t w, int col, Cols<V> &c) const {
        if ((uint32_t)w < n_master) {
            const float *p = master + (size_t)w * d + col;
#pragma unroll
            for (int i = 0; i < V; i++) c.v[i] = __ldcg(p + i);
        } else {
            const __nv_bfloat16 *p = bf + (size_t)w * d + col;
#pragma unroll
            for (int i = 0; i < V; i++) c.v[i] = __bfloat162float(p[i]);
        }
    }
    __device__ __forceinline__ bool is_master(int32_t w) const { return (uint32_t)w < n_master; }
    // The current BF16 value of a non-master row (masters need no read: they are
    // updated with atomics).
    __device__ __forceinline__ void load_old(int32_t w, int col, Cols<V> &old) const {
        if ((uint32_t)w >= n_master) {
            const __nv_bfloat16 *p = bf + (size_t)w * d + col;
#pragma unroll
            for (int i = 0; i < V; i++) old.v[i] = __bfloat162float(p[i]);
        }
    }
    // row[w][col..col+V) += delta, given the row's value `old` (unused for masters).
    __device__ __forceinline__ void apply(int32_t w, int col, const Cols<V> &old, const Cols<V> &delta,
                                          uint32_t salt) const {
        if ((uint32_t)w < n_master) {
            float *p = master + (size_t)w * d + col;
            if constexpr (V == 2) {
                atomicAdd(reinterpret_cast<float2 *>(p), make_float2(delta.v[0], delta.v[1]));
            } else {
#pragma unroll
                for (int i = 0; i < V; i++) atomicAdd(p + i, delta.v[i]);
            }
        } else {
            __nv_bfloat16 *p = bf + (size_t)w * d + col;
#pragma unroll
            for (int i = 0; i < V; i++)
                p[i] = bf16_sr(old.v[i] + delta.v[i], mix32(salt + (uint32_t)i * 0x9E3779B9u));
        }
    }
};

__device__ __forceinline__ float mb_grad(float f, int label, const float *exp_table, float alpha) {
    if (f > kMaxExp) return (label - 1) * alpha;
    if (f < -kMaxExp) return label * alpha;
    return (label - exp_table[(int)((f + kMaxExp) * (kExpTableSize / kMaxExp / 2))]) * alpha;
}

// Shared memory of one worker (floats first, then ints).
constexpr uint32_t mb_smem_bytes(int d, int out, int max_in, uint32_t pool_cap) {
    return (uint32_t)((2u * kMbMaxSent * d + (uint32_t)mb_warps(d) * max_in * out + 2u * mb_warps(d) * 32u) * 4 +
                      (6u * kMbMaxSent + (uint32_t)max_in + 2u * pool_cap + kMbHash + 3u * out + 16u) * 4);
}

// D: row size; OUT: output slots per step (>= negative + 2, a divisor of 32).
template <int D, int OUT>
__global__ void __launch_bounds__(32 * mb_warps(D)) __maxnreg__(mb_max_regs(D)) sgns_mb_kernel(SgnsArgs a, WalkSet ws, MbArgs m) {
    constexpr int NW = mb_warps(D);
    constexpr int V = D / (32 * NW);
    constexpr int IPB = 32 / OUT;                   // inputs per batch of 32 corr dots
    // Rows whose loads are issued together by the fills and flushes (4: the
    // step fits the 168-register cap without spilling; 8 needed 192).
    constexpr int kRowBatch = 4;
    extern __shared__ __align__(16) float smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int col = warp * 32 * V + lane * V;
    const int MI = m.max_in;
    float *cache = smem;                            // [2][kMbMaxSent][D]
    float *gm = cache + 2 * kMbMaxSent * D + warp * MI * OUT;   // this warp's copy, [MI][OUT]
    float *xs = cache + 2 * kMbMaxSent * D + NW * MI * OUT;     // [2][NW][32] partial dots
    int *ip = reinterpret_cast<int *>(xs + 2 * NW * 32);
    int *sen = ip;                                  // [2][kMbMaxSent] vocabulary ids
    int *slot = sen + 2 * kMbMaxSent;               // [2][kMbMaxSent] token -> cache row
    int *dist = slot + 2 * kMbMaxSent;              // [2][kMbMaxSent] cache row -> word
    int *in_row = dist + 2 * kMbMaxSent;            // [MI] cache row (+ kMbMaxSent for sentence 2)
    int *pool_slot = in_row + MI;                   // [pool_cap] sample -> pool slot
    int *pool_word = pool_slot + m.pool_cap;        // [pool_cap] pool slot -> word
    int *hash = pool_word + m.pool_cap;             // [kMbHash] word -> pool slot (dedup)
    int *out_word = hash + kMbHash;                 // [OUT]
    int *out_meta = out_word + OUT;                 // [OUT]
    int *out_slot = out_meta + OUT;                 // [OUT] pool slot, -1 for centres
    int *shr = out_slot + OUT;                      // [16] scalars: 0-1 len, 2-3 ndist, 4 npool, 5 O, 6 I, 7 first

    const uint32_t worker = blockIdx.x;
    const uint32_t W = ws.n_walks, G = gridDim.x;
    const uint32_t w_begin = (uint32_t)((uint64_t)W * worker / G), w_end = (uint32_t)((uint64_t)W * (worker + 1) / G);
    float *pool_cur = m.scratch + (uint64_t)worker * m.scratch_stride;
    float *pool_init = pool_cur + (uint64_t)m.pool_cap * D;
    float *sent_init = pool_init + (uint64_t)m.pool_cap * D;   // [2][kMbMaxSent][D]
    const uint32_t key0 = a.seed_lo ^ mix32(a.pass * 0x9E3779B9u + 0x632BE5ABu), key1 = a.seed_hi;
    const MbRows<V> in_rows{a.in_bf, a.in_master, a.n_master, D};
    const MbRows<V> out_rows{a.out_bf, a.out_master, a.n_master, D};
    const float alpha = a.alpha;
    const int window = a.window, negative = a.negative;

    // Worker state, identical in every thread.
    // Indexed only by constants (the loops over the two sentences are unrolled),
    // so these stay in registers rather than in a local-memory stack frame.
    int len[2] = {0, 0}, pos[2] = {0, 0};
    int nbn = 1;
    unsigned long long n_words = 0, n_trained = 0, n_pairs = 0, n_rows = 0;
    uint32_t next_walk = w_begin;
    uint32_t step = 0, pool_no = 0, neg_count = 0;
    int train_sen_num = 0;
    bool change_neg = true, pool_loaded = false;

    auto salt_of = [&](int32_t w, uint32_t extra) {
        return mix32(key0 ^ mix32((uint32_t)w * 0x01000193u + (uint32_t)col) ^ (step * 0x2545F491u) ^ extra);
    };
    // Writes cache s back as a delta against the rows it was loaded from.
    // Rows of one flush are distinct, so all their reads are issued before any write.
    auto flush_sentence = [&](int s) {
        const int nd = shr[2 + s];
        for (int r0 = 0; r0 < nd; r0 += kRowBatch) {
            Cols<V> cur[kRowBatch], ini[kRowBatch], old[kRowBatch];
#pragma unroll
            for (int u = 0; u < kRowBatch; u++)
                if (r0 + u < nd) {
                    ld_cols<V>(cache + (s * kMbMaxSent + r0 + u) * D + col, cur[u]);
                    ld_cols<V>(sent_init + ((uint64_t)s * kMbMaxSent + r0 + u) * D + col, ini[u]);
                    in_rows.load_old(dist[s * kMbMaxSent + r0 + u], col, old[u]);
                }
#pragma unroll
            for (int u = 0; u < kRowBatch; u++)
                if (r0 + u < nd) {
#pragma unroll
                    for (int i = 0; i < V; i++) cur[u].v[i] -= ini[u].v[i];
                    const int w = dist[s * kMbMaxSent + r0 + u];
                    in_rows.apply(w, col, old[u], cur[u], salt_of(w, 0x11u + s));
                }
        }
    };
    auto flush_pool = [&]() {
        const int np = shr[4];
        for (int r0 = 0; r0 < np; r0 += kRowBatch) {
            Cols<V> cur[kRowBatch], ini[kRowBatch], old[kRowBatch];
#pragma unroll
            for (int u = 0; u < kRowBatch; u++)
                if (r0 + u < np) {
                    ld_cols<V>(pool_cur + (uint64_t)(r0 + u) * D + col, cur[u]);
                    ld_cols<V>(pool_init + (uint64_t)(r0 + u) * D + col, ini[u]);
                    out_rows.load_old(pool_word[r0 + u], col, old[u]);
                }
#pragma unroll
            for (int u = 0; u < kRowBatch; u++)
                if (r0 + u < np) {
#pragma unroll
                    for (int i = 0; i < V; i++) cur[u].v[i] -= ini[u].v[i];
                    out_rows.apply(pool_word[r0 + u], col, old[u], cur[u], salt_of(pool_word[r0 + u], 0x55u));
                }
        }
    };

    for (;;) {
        // ---- fill empty sentence slots (dsgl.hpp:903-1028); warp 0 builds, all load ----
#pragma unroll
        for (int s = 0; s < 2; s++) {
            while (len[s] == 0 && next_walk < w_end) {
                const uint32_t walk = next_walk++;
                uint64_t begin;
                uint32_t wl;
                ws.range(walk, begin, wl);
                if (wl > kMbMaxSent) wl = kMbMaxSent;
                if (warp == 0) {
                    const uint32_t wid = ws.ids ? ws.ids[walk] : walk + ws.id_base;
                    bool keep = false;
                    int32_t w = -1;
                    if ((uint32_t)lane < wl) {
                        w = a.v2w[ws.verts[begin + lane]];
                        if (w >= 0) {
                            const uint32_t u = philox4x32_10(make_uint4((uint32_t)lane, wid, a.pass, kSubTag),
                                                             a.seed_lo, a.seed_hi).x & 0xFFFFu;
                            keep = u < a.keep_thr[w];
                        }
                    }
                    const uint32_t mask = __ballot_sync(0xffffffffu, keep);
                    const int n = __popc(mask);
                    if (keep) sen[s * kMbMaxSent + __popc(mask & ((1u << lane) - 1))] = w;
                    __syncwarp();
                    // distinct words in first-occurrence order (dsgl.hpp:948-956)
                    int nd = 0;
                    for (int t = 0; t < n; t++) {
                        const int wt = sen[s * kMbMaxSent + t];
                        const uint32_t hit =
                            __ballot_sync(0xffffffffu, lane < nd && dist[s * kMbMaxSent + lane] == wt);
                        int r;
                        if (hit) {
                            r = __ffs(hit) - 1;
                        } else {
                            r = nd;
                            if (lane == 0) dist[s * kMbMaxSent + nd] = wt;
                            nd++;
                        }
                        if (lane == 0) slot[s * kMbMaxSent + t] = r;
                        __syncwarp();
                    }
                    if (lane == 0) {
                        shr[s] = n <= 1 ? 0 : n;   // dsgl.hpp:941-945
                        shr[2 + s] = nd;
                        shr[8 + s] = n;
                    }
                }
                __syncthreads();
                len[s] = shr[s];
                pos[s] = 0;
                n_words += wl;
                n_trained += shr[8 + s];
                if (len[s] != 0) {
                    const int nd = shr[2 + s];
                    for (int r0 = 0; r0 < nd; r0 += kRowBatch) {
                        Cols<V> c[kRowBatch];
#pragma unroll
                        for (int u = 0; u < kRowBatch; u++)
                            if (r0 + u < nd) in_rows.get(dist[s * kMbMaxSent + r0 + u], col, c[u]);
#pragma unroll
                        for (int u = 0; u < kRowBatch; u++)
                            if (r0 + u < nd) {
                                st_cols<V>(cache + (s * kMbMaxSent + r0 + u) * D + col, c[u]);
                                st_cols<V>(sent_init + ((uint64_t)s * kMbMaxSent + r0 + u) * D + col, c[u]);
                            }
                    }
                }
                __syncthreads();
            }
        }
        if (len[0] == 0 || len[1] == 0) break;   // slice exhausted (dsgl.hpp:1029-1049)

        // ---- shared negative pool (dsgl.hpp:1052-1083) ----
        if (change_neg) {
            nbn = max(len[0], len[1]);
            if (warp == 0) {
                const int total = nbn * negative;
                for (int h = lane; h < kMbHash; h += 32) hash[h] = -1;
                __syncwarp();
                int np = 0;
                for (int base = 0; base < total; base += 32) {
                    const int j = base + lane;
                    int32_t smp = -1;
                    if (j < total) {
                        const uint4 x =
                            philox4x32_10(make_uint4((uint32_t)j >> 2, pool_no, worker, kMbPoolTag), key0, key1);
                        const uint32_t q = j & 3;
                        const uint32_t r = q == 0 ? x.x : q == 1 ? x.y : q == 2 ? x.z : x.w;
                        smp = a.table[r % a.table_size];
                        if (!smp) smp = a.vocab_size > 1 ? (int32_t)((r >> 8) % (a.vocab_size - 1) + 1) : 0;
                    }
                    // Pool slots in sample order (first occurrence keeps its slot).
                    const int cnt = min(32, total - base);
                    for (int t = 0; t < cnt; t++) {
                        const int w = __shfl_sync(0xffffffffu, smp, t);
                        if (lane == 0) {
                            uint32_t h = mix32((uint32_t)w) & (kMbHash - 1);
                            int at = -1;
                            for (int probe = 0; probe < kMbHash; probe++) {
                                const int e = hash[h];
                                if (e < 0) {
                                    at = np;
                                    hash[h] = np;
                                    pool_word[np++] = w;
                                    break;
                                }
                                if (pool_word[e] == w) {
                                    at = e;
                                    break;
                                }
                                h = (h + 1) & (kMbHash - 1);
                            }
                            pool_slot[base + t] = at;
                        }
                    }
                    np = __shfl_sync(0xffffffffu, np, 0);
                }
                if (lane == 0) shr[4] = np;
            }
            __syncthreads();
            const int np = shr[4];
            for (int r0 = 0; r0 < np; r0 += kRowBatch) {
                Cols<V> c[kRowBatch];
#pragma unroll
                for (int u = 0; u < kRowBatch; u++)
                    if (r0 + u < np) out_rows.get(pool_word[r0 + u], col, c[u]);
#pragma unroll
                for (int u = 0; u < kRowBatch; u++)
                    if (r0 + u < np) {
                        st_cols<V>(pool_cur + (uint64_t)(r0 + u) * D + col, c[u]);
                        st_cols<V>(pool_init + (uint64_t)(r0 + u) * D + col, c[u]);
                    }
            }
            pool_no++;
            change_neg = false;
            pool_loaded = true;
        }

        // ---- step bookkeeping: inputs and outputs (dsgl.hpp:1089-1160), by warp 0 ----
        neg_count++;
        if (warp == 0) {
            const uint32_t b = philox4x32_10(make_uint4(step, worker, 0, kMbWinTag), key0, key1).x % (uint32_t)window;
            int ni = 0;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                for (int base = (int)b; base < 2 * window + 1 - (int)b; base += 32) {
                    const int i = base + lane;
                    const int c = pos[s] - window + i;
                    const bool ok = i < 2 * window + 1 - (int)b && i != window && c >= 0 && c < len[s];
                    const uint32_t mask = __ballot_sync(0xffffffffu, ok);
                    if (ok) in_row[ni + __popc(mask & ((1u << lane) - 1))] = s * kMbMaxSent + slot[s * kMbMaxSent + c];
                    ni += __popc(mask);
                }
                if (s == 0 && lane == 0) shr[7] = ni;
            }
            const int start = (int)(neg_count % (uint32_t)nbn);
            const int t1 = sen[pos[0]];
            int ps = -1, smp = -1;
            if (lane < negative) {
                ps = pool_slot[start * negative + lane];
                smp = pool_word[ps];
            }
            const uint32_t same = __match_any_sync(0xffffffffu, smp);
            const bool lead = lane < negative && (int)(__ffs(same) - 1) == lane && smp != t1;
            const uint32_t leads = __ballot_sync(0xffffffffu, lead);
            if (lead) {
                const int o = 1 + __popc(leads & ((1u << lane) - 1));
                out_word[o] = smp;
                out_meta[o] = __popc(same);
                out_slot[o] = ps;
            }
            if (lane == 0) {
                const int O = 2 + __popc(leads);
                out_word[0] = t1;
                out_meta[0] = 1;                     // dsgl.hpp:1153-1154
                out_slot[0] = -1;
                out_word[O - 1] = sen[kMbMaxSent + pos[1]];
                out_meta[O - 1] = 1;
                out_slot[O - 1] = -1;
                shr[5] = O;
                shr[6] = ni;
            }
        }
        __syncthreads();
        const int O = shr[5], I = shr[6], first = shr[7];
        n_pairs += I;
        n_rows += I + O;

        // ---- output rows into registers (centres from the tables, negatives from the pool) ----
        Cols<V> x[OUT];
#pragma unroll
        for (int o = 0; o < OUT; o++) {
            if (o < O) {
                if (out_slot[o] < 0) out_rows.get(out_word[o], col, x[o]);
                else ld_cols<V>(pool_cur + (uint64_t)out_slot[o] * D + col, x[o]);
            } else {
#pragma unroll
                for (int k = 0; k < V; k++) x[o].v[k] = 0.f;
            }
        }

        // ---- corr = outputs . inputs^T, gradients (dsgl.hpp:1241-1274) ----
        int parity = 0;
        for (int i0 = 0; i0 < I; i0 += IPB, parity ^= 1) {
            float s[32];
#pragma unroll
            for (int bi = 0; bi < IPB; bi++) {
                Cols<V> y;
                if (i0 + bi < I) ld_cols<V>(cache + in_row[i0 + bi] * D + col, y);
                else {
#pragma unroll
                    for (int k = 0; k < V; k++) y.v[k] = 0.f;
                }
#pragma unroll
                for (int o = 0; o < OUT; o++) {
                    float acc = 0.f;
#pragma unroll
                    for (int k = 0; k < V; k++) acc = fmaf(x[o].v[k], y.v[k], acc);
                    s[bi * OUT + o] = acc;
                }
            }
            // Recursive halving: lane j ends with this warp's partial of dot j.
#pragma unroll
            for (int w = 16; w >= 1; w >>= 1) {
                const bool upper = (lane & w) != 0;
#pragma unroll
                for (int k = 0; k < w; k++) {
                    const float send = upper ? s[k] : s[k + w];
                    const float keep = upper ? s[k + w] : s[k];
                    s[k] = keep + __shfl_xor_sync(0xffffffffu, send, w);
                }
            }
            float f = s[0];
            if (NW > 1) {
                xs[(parity * NW + warp) * 32 + lane] = f;
                __syncthreads();
                f = xs[parity * NW * 32 + lane];
#pragma unroll
                for (int w = 1; w < NW; w++) f += xs[(parity * NW + w) * 32 + lane];
            }
            const int bi = lane / OUT, o = lane % OUT, i = i0 + bi;
            if (i < I && o < O) {
                const int label = i < first ? (o == 0) : (o == O - 1);
                gm[i * OUT + o] = mb_grad(f, label, a.exp_table, alpha) * (float)out_meta[o];
            }
        }
        __syncwarp();

        // ---- outputs += corr . inputs (dsgl.hpp:1290-1295), from the inputs before their update ----
        Cols<V> md[OUT];
#pragma unroll
        for (int o = 0; o < OUT; o++)
#pragma unroll
            for (int k = 0; k < V; k++) md[o].v[k] = 0.f;
        // Gradient column of input i: OUT consecutive floats, fetched as float4s.
        auto g_column = [&](int i, float (&g)[OUT]) {
#pragma unroll
            for (int o = 0; o < OUT; o += 4) {
                const float4 t = *reinterpret_cast<const float4 *>(gm + i * OUT + o);
                g[o] = t.x; g[o + 1] = t.y; g[o + 2] = t.z; g[o + 3] = t.w;
            }
        };
        for (int i = 0; i < I; i++) {
            Cols<V> y;
            ld_cols<V>(cache + in_row[i] * D + col, y);
            float g[OUT];
            g_column(i, g);
#pragma unroll
            for (int o = 0; o < OUT; o++) {
                if (o >= O) break;
#pragma unroll
                for (int k = 0; k < V; k++) md[o].v[k] = fmaf(g[o], y.v[k], md[o].v[k]);
            }
        }
        // ---- inputs += corr^T . outputs (dsgl.hpp:1303-1350), in input order ----
        for (int i = 0; i < I; i++) {
            Cols<V> acc;
#pragma unroll
            for (int k = 0; k < V; k++) acc.v[k] = 0.f;
            float g[OUT];
            g_column(i, g);
#pragma unroll
            for (int o = 0; o < OUT; o++) {
                if (o >= O) break;
#pragma unroll
                for (int k = 0; k < V; k++) acc.v[k] = fmaf(g[o], x[o].v[k], acc.v[k]);
            }
            float *row = cache + in_row[i] * D + col;
            Cols<V> c;
            ld_cols<V>(row, c);
#pragma unroll
            for (int k = 0; k < V; k++) c.v[k] += acc.v[k];
            st_cols<V>(row, c);
        }
        // Centre rows in order (centre 1, then centre 2), updated from their values
        // staged at the start of the step; pool rows from registers.
        {
            const int32_t w1 = out_word[0];
            out_rows.apply(w1, col, x[0], md[0], salt_of(w1, 0x77u));
        }
#pragma unroll
        for (int o = 1; o < OUT; o++) {
            if (o == O - 1) {
                const int32_t w2 = out_word[o];
                Cols<V> base = x[o];
                if (w2 == out_word[0] && !out_rows.is_master(w2)) {
                    // The same BF16 row as centre 1: continue from what was just stored.
                    out_rows.load_old(w2, col, base);
                }
                out_rows.apply(w2, col, base, md[o], salt_of(w2, 0x78u));
            } else if (o < O - 1) {
                // x[o] holds this pool row as staged at the start of the step and
                // only this worker writes its columns, so no re-load is needed.
#pragma unroll
                for (int k = 0; k < V; k++) x[o].v[k] += md[o].v[k];
                st_cols<V>(pool_cur + (uint64_t)out_slot[o] * D + col, x[o]);
            }
        }

        // ---- advance; write back finished sentences and spent pools (dsgl.hpp:1398-1424) ----
        step++;
        pos[0]++;
        pos[1]++;
#pragma unroll
        for (int s = 0; s < 2; s++)
            if (pos[s] >= len[s]) {
                flush_sentence(s);
                len[s] = 0;
                train_sen_num++;
            }
        if (train_sen_num >= 2) {
            flush_pool();
            change_neg = true;
            pool_loaded = false;
            train_sen_num = 0;
        }
        __syncthreads();   // bookkeeping arrays are rewritten next step
    }
    // Slice exhausted: keep the updates of the sentence still in flight and of
    // the pool (dsgl drops them; here they are written back).
#pragma unroll
    for (int s = 0; s < 2; s++)
        if (len[s] != 0) flush_sentence(s);
    if (pool_loaded) flush_pool();
    if (tid == 0) {
        atomicAdd(&a.stats[0], n_words);
        atomicAdd(&a.stats[1], n_trained);
        atomicAdd(&a.stats[2], n_pairs);
        atomicAdd(&a.stats[3], n_rows);
    }
}

// Launch geometry shared by both entry points.
struct MbPlan {
    MbArgs m{};
    int out = 8;
    int threads = 32;
    int per_sm = 0;
};

template <int D, int OUT>
static int mb_setup(MbPlan &plan) {
    plan.threads = 32 * mb_warps(D);
    DG_CUDA(cudaFuncSetAttribute(sgns_mb_kernel<D, OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)plan.m.smem));
    DG_CUDA(cudaFuncSetAttribute(sgns_mb_kernel<D, OUT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
    DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&plan.per_sm, sgns_mb_kernel<D, OUT>, plan.threads,
                                                          plan.m.smem));
    return DG_OK;
}

template <int OUT>
static int mb_setup_d(int d, MbPlan &plan) {
    switch (d) {
    case 32: return mb_setup<32, OUT>(plan);
    case 64: return mb_setup<64, OUT>(plan);
    case 128: return mb_setup<128, OUT>(plan);
    default: return mb_setup<256, OUT>(plan);
    }
}

static int mb_plan(int d, int negative, int window, MbPlan &plan) {
    DG_CHECK(d == 32 || d == 64 || d == 128 || d == 256, DG_ERR_ARG,
             "size %d not supported in minibatch mode (32, 64, 128, 256)", d);
    DG_CHECK(negative >= 0 && negative <= 14, DG_ERR_ARG, "minibatch mode supports negative <= 14 (got %d)", negative);
    DG_CHECK(window >= 1 && window <= 64, DG_ERR_ARG, "window %d out of range [1, 64]", window);
    plan.out = negative + 2 <= 8 ? 8 : 16;
    MbArgs &m = plan.m;
    m.pool_cap = (uint32_t)kMbMaxSent * (uint32_t)std::max(negative, 1);
    m.max_in = 4 * window;
    m.scratch_stride = (uint64_t)m.pool_cap * d * 2 + 2ull * kMbMaxSent * d;
    m.smem = mb_smem_bytes(d, plan.out, m.max_in, m.pool_cap);
    int rc = plan.out == 8 ? mb_setup_d<8>(d, plan) : mb_setup_d<16>(d, plan);
    if (rc) return rc;
    DG_CHECK(plan.per_sm >= 1, DG_ERR_ARG, "minibatch kernel does not fit (%u bytes of shared memory)", m.smem);
    return DG_OK;
}

template <int OUT>
static void mb_launch_out(int d, unsigned workers, const MbPlan &plan, cudaStream_t s, const SgnsArgs &a,
                          const WalkSet &ws, const MbArgs &m) {
    const size_t smem = plan.m.smem;
    switch (d) {
    case 32: sgns_mb_kernel<32, OUT><<<workers, 32 * mb_warps(32), smem, s>>>(a, ws, m); break;
    case 64: sgns_mb_kernel<64, OUT><<<workers, 32 * mb_warps(64), smem, s>>>(a, ws, m); break;
    case 128: sgns_mb_kernel<128, OUT><<<workers, 32 * mb_warps(128), smem, s>>>(a, ws, m); break;
    default: sgns_mb_kernel<256, OUT><<<workers, 32 * mb_warps(256), smem, s>>>(a, ws, m); break;
    }
}

static void mb_launch(int d, unsigned workers, const MbPlan &plan, cudaStream_t s, const SgnsArgs &a,
                      const WalkSet &ws, const MbArgs &m) {
    if (plan.out == 8) mb_launch_out<8>(d, workers, plan, s, a, ws, m);
    else mb_launch_out<16>(d, workers, plan, s, a, ws, m);
    dg::note_launch();
}

// Every worker trains on snapshot copies (its negative pool, its two sentences)
// and writes them back as deltas, so a row held by k workers at once receives k
// deltas computed from one stale value: the hottest row's effective step grows
// with the number of workers holding it.  On the 10,000-vertex power-law graph
// (hottest row in 64% of pools) about 190 concurrent holders trained stably and
// about 380 diverged (rows grew until sigmoid saturated, link-prediction AUC fell
// from 0.71 to 0.45).  The bound keeps the expected number of holders of the
// hottest input row and of the hottest output row at kMbMaxHolders.
constexpr double kMbMaxHolders = 128.0;

void hot_row_shares(const std::vector<uint32_t> &cn, const std::vector<uint32_t> &keep_thr, double &p_neg,
                    double &p_tok) {
    // Negatives: unigram^0.75 (word2vec.cu:141-160).
    double z = 0.0, top = 0.0;
    for (uint32_t c : cn) {
        const double p = std::pow((double)c, 0.75);
        z += p;
        top = std::max(top, p);
    }
    p_neg = z > 0 ? top / z : 0.0;
    // Tokens: frequency after subsampling.
    double kept = 0.0, kept_top = 0.0;
    for (size_t w = 0; w < cn.size(); w++) {
        const double k = (double)cn[w] * std::min(1.0, keep_thr[w] / 65536.0);
        kept += k;
        kept_top = std::max(kept_top, k);
    }
    p_tok = kept > 0 ? kept_top / kept : 0.0;
}

uint32_t mb_worker_bound(const std::vector<uint32_t> &cn, const std::vector<uint32_t> &keep_thr, int negative) {
    if (cn.empty()) return 1;
    double p_neg, p_tok;
    hot_row_shares(cn, keep_thr, p_neg, p_tok);
    // A worker holds a pool of kMbMaxSent x negative draws and two sentences of kMbMaxSent tokens.
    const double hold_out = 1.0 - std::pow(1.0 - p_neg, (double)kMbMaxSent * std::max(negative, 1));
    const double hold_in = 1.0 - std::pow(1.0 - p_tok, 2.0 * kMbMaxSent);
    const double hold = std::max(hold_out, hold_in);
    if (hold <= 0.0) return 0xFFFFFFFFu;
    return (uint32_t)std::max(1.0, std::min(4.0e9, std::floor(kMbMaxHolders / hold)));
}

int launch_minibatch(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws) {
    MbPlan plan;
    int rc = mb_plan(s->p.size, a.negative, a.window, plan);
    if (rc) return rc;
    uint32_t workers = a.deterministic ? 1u : (uint32_t)(dg::sm_count(s->device) * plan.per_sm);
    if (!a.deterministic) workers = std::min(workers, s->p.workers ? s->p.workers : s->mb_workers);
    if (workers > ws.n_walks / 2 + 1) workers = std::max(1u, ws.n_walks / 2);
    const uint64_t need = plan.m.scratch_stride * workers;
    if (s->scratch.n < need) DG_CUDA(s->scratch.alloc(need));
    MbArgs m = plan.m;
    m.scratch = s->scratch.p;
    mb_launch(s->p.size, workers, plan, s->stream, a, ws, m);
    DG_CUDA(cudaGetLastError());
    return DG_OK;
}

}  // namespace dgs

// ---------------------------------------------------------------------------
// Allocation-free entry point: the minibatch trainer with its per-worker
// scratch (negative pools and cache snapshots) in a fixed device array that is
// part of this library, so that a call performs no device or host allocation.
// It serves callers that must not allocate: a host framework whose memory pool
// owns the device memory and forbids foreign cudaMalloc, or a latency-bound loop
// that cannot pay cudaMalloc / cudaFree (which can synchronise the device) or
// handle an allocation failure in the middle of training.
// ---------------------------------------------------------------------------
namespace dgs {
namespace {

// Scratch shared by every call on a device (held by each GPU that loads the library).
constexpr size_t kNoAllocScratchBytes = 16u << 20;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchBytes / sizeof(float)];
static __device__ __align__(256) unsigned long long g_noalloc_stats[4];

// Device address of the scratch array, looked up once per device (the host-side
// name of a __device__ array is not a device address).
struct NoAllocSetup {
    std::mutex mu;
    float *scratch[kNoAllocMaxDevices] = {};
    unsigned long long *stats[kNoAllocMaxDevices] = {};
};
NoAllocSetup &noalloc_setup() {
    static NoAllocSetup s;
    return s;
}

int noalloc_pointers(int device, float **scratch, unsigned long long **stats) {
    DG_CHECK(device >= 0 && device < kNoAllocMaxDevices, DG_ERR_ARG, "device %d beyond the %d supported", device,
             kNoAllocMaxDevices);
    NoAllocSetup &s = noalloc_setup();
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.scratch[device]) {
        void *p = nullptr, *q = nullptr;
        DG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        DG_CUDA(cudaGetSymbolAddress(&q, g_noalloc_stats));
        s.scratch[device] = static_cast<float *>(p);
        s.stats[device] = static_cast<unsigned long long *>(q);
    }
    *scratch = s.scratch[device];
    *stats = s.stats[device];
    return DG_OK;
}

}  // namespace
}  // namespace dgs

extern "C" int dg_sgns_minibatch_train_noalloc(const dg_sgns_minibatch_args *x, void *stream, dg_train_info *info) {
    using namespace dgs;
    DG_CHECK(x, DG_ERR_ARG, "dg_sgns_minibatch_train_noalloc: NULL arguments");
    DG_CHECK(x->verts && x->offsets && x->v2w && x->keep_thr && x->table && x->exp_table, DG_ERR_ARG,
             "dg_sgns_minibatch_train_noalloc: walk or table pointer is NULL");
    DG_CHECK(x->in_bf16 && x->out_bf16 && (x->n_master == 0 || (x->in_master && x->out_master)), DG_ERR_ARG,
             "dg_sgns_minibatch_train_noalloc: row pointer is NULL");
    DG_CHECK(x->vocab_size > 0 && x->table_size > 0 && x->table_size < (1ull << 32), DG_ERR_ARG,
             "empty vocabulary or unigram table");
    const int d = x->size;
    MbPlan plan;
    int rc = mb_plan(d, x->negative, x->window, plan);
    if (rc) return rc;
    int device = 0;
    DG_CUDA(cudaGetDevice(&device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (s) {
        // The scratch address and the worker count are those of the current
        // device, so the stream must belong to it.
        int stream_device = -1;
        DG_CUDA(cudaStreamGetDevice(s, &stream_device));
        DG_CHECK(stream_device == device, DG_ERR_ARG,
                 "dg_sgns_minibatch_train_noalloc: the stream belongs to device %d but device %d is current",
                 stream_device, device);
    }
    float *scratch = nullptr;
    unsigned long long *stats = nullptr;
    rc = noalloc_pointers(device, &scratch, &stats);
    if (rc) return rc;
    const uint64_t per_worker = plan.m.scratch_stride * sizeof(float);
    const uint64_t max_workers = kNoAllocScratchBytes / per_worker;
    DG_CHECK(max_workers >= 1, DG_ERR_ARG,
             "size %d with negative %d needs %llu bytes of scratch per worker, more than the %zu-byte static area",
             d, x->negative, (unsigned long long)per_worker, kNoAllocScratchBytes);
    uint64_t workers = x->deterministic ? 1 : (uint64_t)dg::sm_count(device) * plan.per_sm;
    workers = std::min<uint64_t>(workers, max_workers);
    // workers = 0: kMbMaxHolders workers, the staleness bound that holds whatever
    // the vocabulary (even if every worker held the hottest row); the handle
    // path's bound for a given vocabulary is what dg_sgns_get_info reports.
    if (!x->deterministic) workers = std::min<uint64_t>(workers, x->workers ? x->workers : (uint64_t)kMbMaxHolders);
    if (workers > x->n_walks / 2 + 1) workers = std::max<uint64_t>(1, x->n_walks / 2);

    SgnsArgs a{};
    a.v2w = x->v2w;
    a.keep_thr = x->keep_thr;
    a.table = x->table;
    a.exp_table = x->exp_table;
    a.in_bf = reinterpret_cast<__nv_bfloat16 *>(x->in_bf16);
    a.out_bf = reinterpret_cast<__nv_bfloat16 *>(x->out_bf16);
    a.in_master = x->in_master;
    a.out_master = x->out_master;
    a.n_master = x->n_master;
    a.stats = stats;
    a.table_size = x->table_size;
    a.vocab_size = x->vocab_size;
    a.window = x->window;
    a.negative = x->negative;
    a.d = d;
    a.alpha = x->alpha;
    a.pass = x->pass;
    a.seed_lo = (uint32_t)x->seed;
    a.seed_hi = (uint32_t)(x->seed >> 32);
    a.deterministic = x->deterministic;
    WalkSet ws{};
    ws.verts = x->verts;
    ws.offsets = x->offsets;
    ws.n_walks = x->n_walks;
    MbArgs m = plan.m;
    m.scratch = scratch;

    DG_CUDA(cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), s));  // counters start at zero every call
    mb_launch(d, (unsigned)workers, plan, s, a, ws, m);
    DG_CUDA(cudaGetLastError());
    if (info) {
        unsigned long long st[4];
        DG_CUDA(cudaMemcpyAsync(st, stats, sizeof(st), cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        info->words = st[0];
        info->trained = st[1];
        info->pairs = st[2];
        info->train_ms = 0.0;
        info->rows = st[3];
    }
    return DG_OK;
}
