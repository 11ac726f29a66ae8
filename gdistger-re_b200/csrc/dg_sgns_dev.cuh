// Warp-level building blocks of the SGNS kernels (dg_sgns.cu, dg_sgns_w2v.cu):
// a row slice per lane, vector loads / stores / atomics, warp dot products,
// the sigmoid-table gradient and the walk-to-sentence step.
#pragma once

#include "dg_sgns.h"

namespace dgs {

template <int VEC>
struct RowVec {
    float v[VEC];
};

template <int VEC>
__device__ __forceinline__ void load_row(const float *p, RowVec<VEC> &r) {
    if constexpr (VEC % 4 == 0) {
#pragma unroll
        for (int i = 0; i < VEC; i += 4) {
            const float4 t = __ldcg(reinterpret_cast<const float4 *>(p + i));
            r.v[i] = t.x; r.v[i + 1] = t.y; r.v[i + 2] = t.z; r.v[i + 3] = t.w;
        }
    } else if constexpr (VEC == 2) {
        const float2 t = __ldcg(reinterpret_cast<const float2 *>(p));
        r.v[0] = t.x; r.v[1] = t.y;
    } else {
        r.v[0] = __ldcg(p);
    }
}

template <int VEC>
__device__ __forceinline__ void store_row(float *p, const RowVec<VEC> &r) {
    if constexpr (VEC % 4 == 0) {
#pragma unroll
        for (int i = 0; i < VEC; i += 4)
            __stcg(reinterpret_cast<float4 *>(p + i), make_float4(r.v[i], r.v[i + 1], r.v[i + 2], r.v[i + 3]));
    } else if constexpr (VEC == 2) {
        __stcg(reinterpret_cast<float2 *>(p), make_float2(r.v[0], r.v[1]));
    } else {
        __stcg(p, r.v[0]);
    }
}

// p[i] += r[i] with 16-byte vector atomics (sm_90+).
template <int VEC>
__device__ __forceinline__ void add_row(float *p, const RowVec<VEC> &r) {
    if constexpr (VEC % 4 == 0) {
#pragma unroll
        for (int i = 0; i < VEC; i += 4)
            atomicAdd(reinterpret_cast<float4 *>(p + i), make_float4(r.v[i], r.v[i + 1], r.v[i + 2], r.v[i + 3]));
    } else if constexpr (VEC == 2) {
        atomicAdd(reinterpret_cast<float2 *>(p), make_float2(r.v[0], r.v[1]));
    } else {
        atomicAdd(p, r.v[0]);
    }
}

template <int VEC>
__device__ __forceinline__ float warp_dot(const RowVec<VEC> &a, const RowVec<VEC> &b) {
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < VEC; i++) s = fmaf(a.v[i], b.v[i], s);
    // Butterfly: lanes i and i^o add the same two values (in swapped order, which
    // float addition does not see), so every lane ends with the same sum.
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}


// g = (label - sigmoid(f)) * alpha through expTable (word2vec.cu:383-388), with
// the reference's integer-division index scale (EXP_TABLE_SIZE / MAX_EXP / 2 = 83).
__device__ __forceinline__ float sg_grad(float f, int label, const float *exp_table, float alpha) {
    if (f > kMaxExp) return (label - 1) * alpha;
    if (f < -kMaxExp) return label * alpha;
    return (label - __ldg(exp_table + (int)((f + kMaxExp) * (kExpTableSize / kMaxExp / 2)))) * alpha;
}

// Brings [p, p + bytes) into L2 (bytes a multiple of 16, p 16-byte aligned).  A
// hint only: it holds no registers and orders nothing.
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(bytes));
}

__device__ __forceinline__ uint4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    return philox4x32_10(make_uint4(c0, c1, c2, c3), k0, k1);
}

// Builds the walk's sentence in shared memory: vocabulary lookup + subsampling
// (word2vec.cu:1011-1029 with a Philox draw in place of rand()).  Returns its length.
// At most CAP tokens of a walk are used.
template <uint32_t CAP = kMaxSentence>
__device__ __forceinline__ uint32_t warp_sentence(const WalkSet &ws, uint32_t walk, const SgnsArgs &a, int32_t *sen,
                                                  uint32_t &words) {
    const uint32_t lane = threadIdx.x & 31;
    uint64_t begin;
    uint32_t len;
    ws.range(walk, begin, len);
    if (len > CAP) len = CAP;
    words = len;
    uint32_t n = 0;
    for (uint32_t base = 0; base < len; base += 32) {
        const uint32_t i = base + lane;
        bool keep = false;
        int32_t w = -1;
        if (i < len) {
            w = a.v2w[ws.verts[begin + i]];
            if (w >= 0) {
                const uint32_t u = philox(i, ws.ids ? ws.ids[walk] : walk + ws.id_base, a.pass, kSubTag, a.seed_lo,
                                          a.seed_hi).x & 0xFFFFu;
                keep = u < a.keep_thr[w];
            }
        }
        const uint32_t mask = __ballot_sync(0xffffffffu, keep);
        if (keep) sen[n + __popc(mask & ((1u << lane) - 1))] = w;
        n += __popc(mask);
    }
    __syncwarp();
    return n;
}

// ------------------------------------------------------------ BF16 rows

__device__ __forceinline__ uint32_t bf_mix(uint32_t h) {
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}

// FP32 -> BF16 with stochastic rounding: 16 random bits added below the kept
// mantissa, then truncation (unbiased in expectation; infinities and NaN kept).
__device__ __forceinline__ uint16_t bf16_sr_bits(float x, uint32_t noise) {
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7F800000u) != 0x7F800000u) u += noise & 0xFFFFu;
    return (uint16_t)(u >> 16);
}

// A row of the BF16 tables: FP32 masters for ids < n_master, BF16 otherwise.
// Lane l owns columns [l*VEC, l*VEC + VEC).
template <int VEC>
struct BfRows {
    __nv_bfloat16 *bf;
    float *master;
    uint32_t n_master;
    int d;
    __device__ __forceinline__ void load(int32_t w, uint32_t lane, RowVec<VEC> &r) const {
        if ((uint32_t)w < n_master) {
            load_row<VEC>(master + (size_t)w * d + lane * VEC, r);
            return;
        }
        const uint16_t *p = reinterpret_cast<const uint16_t *>(bf + (size_t)w * d + lane * VEC);
        if constexpr (VEC == 8) {
            const uint4 t = __ldcg(reinterpret_cast<const uint4 *>(p));
            const uint32_t q[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
            for (int i = 0; i < 4; i++) {
                r.v[2 * i] = __uint_as_float(q[i] << 16);
                r.v[2 * i + 1] = __uint_as_float(q[i] & 0xFFFF0000u);
            }
        } else if constexpr (VEC == 4) {
            const uint2 t = __ldcg(reinterpret_cast<const uint2 *>(p));
            r.v[0] = __uint_as_float(t.x << 16);
            r.v[1] = __uint_as_float(t.x & 0xFFFF0000u);
            r.v[2] = __uint_as_float(t.y << 16);
            r.v[3] = __uint_as_float(t.y & 0xFFFF0000u);
        } else {
            const uint32_t t = __ldcg(reinterpret_cast<const unsigned int *>(p));
            r.v[0] = __uint_as_float(t << 16);
            r.v[1] = __uint_as_float(t & 0xFFFF0000u);
        }
    }
    // One multiply-xorshift of the salt per row write (the salts already differ
    // by row, pair and lane); each 32-bit word of noise rounds two elements (low
    // half for the even element, high half for the odd one), the next word comes
    // from one LCG step.  The rounding is bf16_sr_bits, done by the stochastic-
    // rounding convert (cvt.rs.bf16x2.f32: upper result = a rounded with
    // rbits[31:16], lower = b with rbits[15:0]), which gives bf16_sr_bits'
    // result for every non-NaN input (infinities kept; a NaN stays a NaN).
    __device__ __forceinline__ void store_bits(int32_t w, uint32_t lane, const RowVec<VEC> &r, uint32_t salt) const {
        uint32_t word[VEC / 2];
        uint32_t x = salt * 0x9E3779B1u;
        x ^= x >> 16;
#pragma unroll
        for (int i = 0; i < VEC; i += 2) {
            asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(word[i / 2]) : "f"(r.v[i + 1]), "f"(r.v[i]), "r"(x));
            x = x * 0x9E3779B1u + 0x7F4A7C15u;
        }
        uint16_t *p = reinterpret_cast<uint16_t *>(bf + (size_t)w * d + lane * VEC);
        if constexpr (VEC == 8) {
            __stcg(reinterpret_cast<uint4 *>(p), make_uint4(word[0], word[1], word[2], word[3]));
        } else if constexpr (VEC == 4) {
            __stcg(reinterpret_cast<uint2 *>(p), make_uint2(word[0], word[1]));
        } else {
            __stcg(reinterpret_cast<unsigned int *>(p), word[0]);
        }
    }
    // Hogwild write of an updated row: FP32 masters (the hottest rows, where
    // writers collide) receive `delta` by vector atomics; a BF16 row is stored
    // as the warp's updated copy `value` (loaded at the start of the pair, so an
    // update another warp made to the same cold row in that window is lost, as
    // in any Hogwild scheme), rounded stochastically -- a store, not a
    // read-modify-write, so the warp does not wait on it.
    __device__ __forceinline__ void update(int32_t w, uint32_t lane, const RowVec<VEC> &delta,
                                           const RowVec<VEC> &value, uint32_t salt) const {
        if ((uint32_t)w < n_master) add_row<VEC>(master + (size_t)w * d + lane * VEC, delta);
        else store_bits(w, lane, value, salt);
    }
    // row = value (one writer: deterministic mode).
    __device__ __forceinline__ void put(int32_t w, uint32_t lane, const RowVec<VEC> &v, uint32_t salt) const {
        if ((uint32_t)w < n_master) store_row<VEC>(master + (size_t)w * d + lane * VEC, v);
        else store_bits(w, lane, v, salt);
    }
};

}  // namespace dgs
