// SGNS loss and its hand-written backward (adjoint) over explicit minibatches.
//
// The loss that word2vec.cu's skip_gram_kernel (word2vec.cu:305-399) and dsgl's
// minibatch update (dsgl.hpp:1241-1311) climb with their fused updates:
//
//   L = sum over pairs p = (i, o) in minibatch b of
//         softplus(-v_i . u_o) + sum over the minibatch's negatives k of softplus(v_i . u_k)
//
// (softplus(x) = -log sigmoid(-x)), v = input rows, u = output rows.  Its
// gradient, with s = v_i . u_o and s_k = v_i . u_k:
//
//   dL/dv_i += (sigmoid(s) - 1) u_o + sum_k sigmoid(s_k) u_k
//   dL/du_o += (sigmoid(s) - 1) v_i
//   dL/du_k += sigmoid(s_k) v_i                (summed over the minibatch's pairs)
//
// Unlike the fused Hogwild updates, nothing is written to the rows while the
// gradient is formed, and the result does not depend on thread scheduling: every
// contribution is computed by one warp in a fixed order and added to 64-bit
// fixed-point accumulators (value x 2^40) with integer atomics, which are
// associative.  Contributions must stay below 2^20 in magnitude (a flag turns a
// larger or non-finite one into DG_ERR_ARG); sums below 2^23.  The step kernel
// then applies rows -= alpha * gradient, rounding to nearest (FP32 rows, FP32
// masters, BF16 rows).
//
// Layout: one warp per minibatch (grid-stride), lane l owns columns
// [l*V, l*V + V) of every row (V = size / 32); the minibatch's negative rows and
// their gradient sums sit in this warp's slice of shared memory.
#include "dg_sgns.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace dgs {
namespace {

constexpr int kAdjMaxNeg = 16;
constexpr int kAdjFixedNeg = 5;                          // negative count with its own kernel instance
constexpr float kFixScale = 1099511627776.0f;           // 2^40
constexpr double kFixInv = 1.0 / 1099511627776.0;       // 2^-40
constexpr float kFixMaxTerm = 1048576.0f;               // 2^20
constexpr int kAdjThreads = 256;
constexpr int kAdjGraphSteps = 16;                     // gradient steps per replayed graph

struct AdjArgs {
    const uint32_t *inputs, *outputs, *negatives;   // whole arrays, indexed by global pair / minibatch
    uint64_t n_pairs, n_batches;
    uint64_t b_begin, b_end;                          // minibatches of this launch (when step is NULL)
    const AdjStep *step;                              // else: the step's minibatches, read on the device
    uint32_t batch;
    int negative;
    const float *in_f32, *out_f32;              // plain form rows (else NULL)
    const __nv_bfloat16 *in_bf, *out_bf;        // BF16 storage rows
    const float *in_master, *out_master;        // FP32 rows of the hottest words
    uint32_t n_master;
    unsigned long long *acc_in, *acc_out;       // vocab x size fixed-point sums
    double *batch_loss;                         // [n_batches]
    unsigned int *flag;
};

template <int V>
__device__ __forceinline__ void adj_load(const float *f32, const __nv_bfloat16 *bf, const float *master,
                                         uint32_t n_master, uint32_t w, int col, float (&x)[V]) {
    constexpr int D = 32 * V;
    if (f32 || w < n_master) {
        const float *p = (f32 ? f32 : master) + (size_t)w * D + col;
#pragma unroll
        for (int c = 0; c < V; c++) x[c] = p[c];
    } else {
        const __nv_bfloat16 *p = bf + (size_t)w * D + col;
#pragma unroll
        for (int c = 0; c < V; c++) x[c] = __bfloat162float(p[c]);
    }
}

template <int V>
__device__ __forceinline__ float adj_dot(const float (&a)[V], const float (&b)[V]) {
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < V; c++) s = fmaf(a[c], b[c], s);
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;  // identical in every lane: the butterfly adds the same operands in the same order
}

__device__ __forceinline__ double softplus(double x) { return fmax(x, 0.0) + log1p(exp(-fabs(x))); }

__device__ __forceinline__ void fix_add(unsigned long long *p, float x, unsigned int *flag) {
    if (!(fabsf(x) < kFixMaxTerm)) {   // also catches NaN
        atomicOr(flag, 1u);
        return;
    }
    atomicAdd(p, (unsigned long long)__float2ll_rn(x * kFixScale));
}

__device__ __forceinline__ float fix_value(unsigned long long q) { return (float)((double)(long long)q * kFixInv); }

// NEG > 0: the negative count fixed at compile time (a.negative == NEG); the
// 1 + NEG dot products of a pair are then reduced together (warp_sums_split,
// bit-identical to adj_dot) and each lane group evaluates one sigmoid.
// NEG == 0: any count up to kAdjMaxNeg, one target after the other.
template <int V, int NEG>
__global__ void __launch_bounds__(kAdjThreads) sgns_adjoint_kernel(AdjArgs a) {
    constexpr int D = 32 * V;
    extern __shared__ __align__(16) float adj_smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, col = lane * V;
    const int neg = NEG > 0 ? NEG : a.negative;
    float *uk = adj_smem + (size_t)wib * 2 * neg * D;   // [neg][D] negative rows
    float *gk = uk + (size_t)neg * D;                    // [neg][D] their gradient sums
    uint64_t n_pairs = a.n_pairs, b_begin = a.b_begin, b_end = a.b_end;
    if (a.step) {
        const AdjStep st = *a.step;
        n_pairs = st.n_pairs;
        b_begin = st.step * st.k;
        if (b_begin >= st.n_batches) return;   // a graph's steps past the round's end
        b_end = min(b_begin + st.k, st.n_batches);
    }
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t b = b_begin + (uint64_t)blockIdx.x * (blockDim.x / 32) + wib; b < b_end; b += warps) {
        const uint64_t p0 = b * a.batch, p1 = min(p0 + a.batch, n_pairs);
        for (int k = 0; k < neg; k++) {
            float x[V];
            adj_load<V>(a.out_f32, a.out_bf, a.out_master, a.n_master, a.negatives[b * neg + k], col, x);
#pragma unroll
            for (int c = 0; c < V; c++) {
                uk[k * D + col + c] = x[c];
                gk[k * D + col + c] = 0.f;
            }
        }
        double loss = 0.0;
        // Consecutive pairs usually share their output row (the contexts of one
        // centre): its row stays in registers and its gradient is summed in
        // order over the run, then added to the accumulator once.
        uint32_t run_o = 0xFFFFFFFFu;
        float uo[V], duo[V];
        for (uint64_t p = p0; p < p1; p++) {
            const uint32_t i = a.inputs[p], o = a.outputs[p];
            if (o != run_o) {
                if (run_o != 0xFFFFFFFFu) {
#pragma unroll
                    for (int c = 0; c < V; c++) fix_add(a.acc_out + (size_t)run_o * D + col + c, duo[c], a.flag);
                }
                adj_load<V>(a.out_f32, a.out_bf, a.out_master, a.n_master, o, col, uo);
#pragma unroll
                for (int c = 0; c < V; c++) duo[c] = 0.f;
                run_o = o;
            }
            float v[V], dv[V];
            adj_load<V>(a.in_f32, a.in_bf, a.in_master, a.n_master, i, col, v);
            if constexpr (NEG > 0) {
                constexpr int M = pow2_at_least(NEG + 1);
                constexpr int GROUP = 32 / M;
                float f[M], u[NEG][V];
                {
                    float s0 = 0.f;
#pragma unroll
                    for (int c = 0; c < V; c++) s0 = fmaf(v[c], uo[c], s0);
                    f[0] = s0;
                }
#pragma unroll
                for (int k = 0; k < NEG; k++) {
                    float sk = 0.f;
#pragma unroll
                    for (int c = 0; c < V; c++) {
                        u[k][c] = uk[k * D + col + c];
                        sk = fmaf(v[c], u[k][c], sk);
                    }
                    f[k + 1] = sk;
                }
#pragma unroll
                for (int k = NEG + 1; k < M; k++) f[k] = 0.f;
                const float mine = warp_sums_split<M>(f, (uint32_t)lane);
                const int jm = lane / GROUP;
                // sigmoid(s) - 1 for the positive target, sigmoid(s_k) for negative k
                const float gm = jm == 0 ? -1.f / (1.f + expf(mine)) : jm <= NEG ? 1.f / (1.f + expf(-mine)) : 0.f;
                float g[NEG + 1];
#pragma unroll
                for (int k = 0; k <= NEG; k++) g[k] = __shfl_sync(0xffffffffu, gm, k * GROUP);
                if (a.batch_loss) {   // the loss in the sequential order (every lane holds every sum)
                    loss += softplus(-(double)__shfl_sync(0xffffffffu, mine, 0));
#pragma unroll
                    for (int k = 0; k < NEG; k++) loss += softplus((double)__shfl_sync(0xffffffffu, mine, (k + 1) * GROUP));
                }
#pragma unroll
                for (int c = 0; c < V; c++) {
                    dv[c] = __fmul_rn(g[0], uo[c]);
                    duo[c] = fmaf(g[0], v[c], duo[c]);
                }
#pragma unroll
                for (int k = 0; k < NEG; k++) {
#pragma unroll
                    for (int c = 0; c < V; c++) {
                        dv[c] = fmaf(g[k + 1], u[k][c], dv[c]);
                        gk[k * D + col + c] = fmaf(g[k + 1], v[c], gk[k * D + col + c]);
                    }
                }
#pragma unroll
                for (int c = 0; c < V; c++) fix_add(a.acc_in + (size_t)i * D + col + c, dv[c], a.flag);
                continue;
            }
            const float s = adj_dot<V>(v, uo);
            const float g = -1.f / (1.f + expf(s));   // sigmoid(s) - 1
            if (a.batch_loss) loss += softplus(-(double)s);
#pragma unroll
            for (int c = 0; c < V; c++) {
                dv[c] = __fmul_rn(g, uo[c]);
                duo[c] = fmaf(g, v[c], duo[c]);
            }
            for (int k = 0; k < neg; k++) {
                float u[V];
#pragma unroll
                for (int c = 0; c < V; c++) u[c] = uk[k * D + col + c];
                const float sk = adj_dot<V>(v, u);
                const float gn = 1.f / (1.f + expf(-sk));   // sigmoid(s_k)
                if (a.batch_loss) loss += softplus((double)sk);
#pragma unroll
                for (int c = 0; c < V; c++) {
                    dv[c] = fmaf(gn, u[c], dv[c]);
                    gk[k * D + col + c] = fmaf(gn, v[c], gk[k * D + col + c]);
                }
            }
#pragma unroll
            for (int c = 0; c < V; c++) fix_add(a.acc_in + (size_t)i * D + col + c, dv[c], a.flag);
        }
        if (run_o != 0xFFFFFFFFu) {
#pragma unroll
            for (int c = 0; c < V; c++) fix_add(a.acc_out + (size_t)run_o * D + col + c, duo[c], a.flag);
        }
        for (int k = 0; k < neg; k++) {
            const uint32_t w = a.negatives[b * neg + k];
#pragma unroll
            for (int c = 0; c < V; c++) fix_add(a.acc_out + (size_t)w * D + col + c, gk[k * D + col + c], a.flag);
        }
        if (lane == 0 && a.batch_loss) a.batch_loss[b] = loss;
    }
}

// Shared negatives of minibatch b (adjoint mode): unigram-table draws keyed by
// (b, pass), with the replacement of row 0 that word2vec.cu:365-368 and
// dsgl.hpp:1064-1066 both apply.
constexpr uint32_t kAdjNegTag = 0x41444E47u;  // "ADNG"

__global__ void adj_negatives(const int32_t *table, uint64_t table_size, uint32_t vocab_size, uint32_t pass,
                              uint32_t k0, uint32_t k1, uint64_t n_batches, int negative, uint32_t *neg) {
    const uint64_t n = n_batches * (uint64_t)negative;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = i / negative;
        const uint32_t k = (uint32_t)(i % negative);
        const uint4 r = philox4x32_10(make_uint4((uint32_t)b, (uint32_t)(b >> 32), pass, kAdjNegTag + k), k0, k1);
        int32_t t = table[r.x % table_size];
        if (t == 0 && vocab_size > 1) t = (int32_t)(r.y % (vocab_size - 1) + 1);
        neg[i] = (uint32_t)t;
    }
}

// rows -= alpha * gradient for the rows one step touched, clearing their
// accumulators for the next step.  A row that occurs several times is applied
// once: the first visitor's exchange takes the whole sum, later ones read 0.
// The step's contributions are complete when this kernel starts.
// The step's minibatches [b0, b1) and pairs [p0, p1) come from the step record.
__global__ void adjoint_apply_rows(unsigned long long *acc_in, unsigned long long *acc_out, const uint32_t *inputs,
                                   const uint32_t *outputs, const uint32_t *negatives, uint32_t batch, int negative,
                                   int d, const AdjStep *step, float *in_f32, float *out_f32, __nv_bfloat16 *in_bf,
                                   __nv_bfloat16 *out_bf, float *in_master, float *out_master, uint32_t n_master) {
    const AdjStep st = *step;
    const uint64_t b0 = st.step * st.k;
    if (b0 >= st.n_batches) return;
    const uint64_t b1 = min(b0 + st.k, st.n_batches);
    const uint64_t p0 = b0 * batch, p1 = min(b1 * batch, st.n_pairs);
    const uint64_t n_pairs = p1 - p0, n_neg = (b1 - b0) * (uint64_t)negative;
    const uint32_t *in_ids = inputs + p0, *out_ids = outputs + p0, *negs = negatives + b0 * negative;
    const float alpha = st.alpha;
    const uint64_t n = (2 * n_pairs + n_neg) * (uint64_t)d;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t occ = i / d;
        const uint32_t c = (uint32_t)(i % d);
        const bool input = occ < n_pairs;
        const uint32_t row = input ? in_ids[occ] : occ < 2 * n_pairs ? out_ids[occ - n_pairs] : negs[occ - 2 * n_pairs];
        const uint64_t k = (uint64_t)row * d + c;
        const unsigned long long q = atomicExch(input ? acc_in + k : acc_out + k, 0ull);
        if (q == 0) continue;
        const float step = __fmul_rn(alpha, fix_value(q));
        float *f32 = input ? in_f32 : out_f32;
        if (f32) {
            f32[k] = __fsub_rn(f32[k], step);
        } else if (row < n_master) {
            float *m = input ? in_master : out_master;
            m[k] = __fsub_rn(m[k], step);
        } else {
            __nv_bfloat16 *bf = input ? in_bf : out_bf;
            bf[k] = __float2bfloat16_rn(__fsub_rn(__bfloat162float(bf[k]), step));
        }
    }
}

__global__ void adj_advance(AdjStep *step) {
    if (threadIdx.x == 0 && blockIdx.x == 0) step->step++;
}

__global__ void adjoint_to_f32(const unsigned long long *acc, uint64_t n, float *out) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        out[k] = fix_value(acc[k]);
}

// rows -= alpha * gradient, rounded to nearest in the rows' storage.
__global__ void adjoint_apply(const unsigned long long *acc, uint64_t n, float alpha, float *f32, __nv_bfloat16 *bf,
                              float *master, uint64_t n_master_elems) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const float step = __fmul_rn(alpha, fix_value(acc[k]));
        if (f32) {
            f32[k] = __fsub_rn(f32[k], step);
        } else if (k < n_master_elems) {
            master[k] = __fsub_rn(master[k], step);
        } else {
            bf[k] = __float2bfloat16_rn(__fsub_rn(__bfloat162float(bf[k]), step));
        }
    }
}

// Launch geometry of the gradient kernel for up to n_batches minibatches per launch.
struct AdjLaunch {
    unsigned blocks = 1;
    int threads = 32;
    size_t smem = 0;
};

template <int V>
int adjoint_config(dg_sgns *s, int negative, uint64_t n_batches, AdjLaunch &l) {
    const size_t per_warp = (size_t)2 * negative * 32 * V * sizeof(float);
    int warps = kAdjThreads / 32;
    while (warps > 1 && per_warp * warps > 96 * 1024) warps /= 2;
    l.smem = per_warp * warps;
    l.threads = warps * 32;
    void (*kern)(AdjArgs) = negative == kAdjFixedNeg ? sgns_adjoint_kernel<V, kAdjFixedNeg> : sgns_adjoint_kernel<V, 0>;
    DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)l.smem));
    int per_sm = 0;
    DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, l.threads, l.smem));
    const uint64_t need = (n_batches + warps - 1) / warps;
    l.blocks = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>(need, (uint64_t)dg::sm_count(s->device) * std::max(per_sm, 1)));
    return DG_OK;
}

int adjoint_configure(dg_sgns *s, int negative, uint64_t n_batches, AdjLaunch &l) {
    switch (s->p.size) {
    case 32: return adjoint_config<1>(s, negative, n_batches, l);
    case 64: return adjoint_config<2>(s, negative, n_batches, l);
    case 128: return adjoint_config<4>(s, negative, n_batches, l);
    case 256: return adjoint_config<8>(s, negative, n_batches, l);
    case 512: return adjoint_config<16>(s, negative, n_batches, l);
    default: return dg::fail(DG_ERR_ARG, "size %d not supported", s->p.size);
    }
}

// Kernel launch only (no runtime calls besides the launch: safe inside a stream capture).
template <int V>
static void adjoint_enqueue_v(dg_sgns *s, const AdjLaunch &l, const AdjArgs &a) {
    if (a.negative == kAdjFixedNeg) sgns_adjoint_kernel<V, kAdjFixedNeg><<<l.blocks, l.threads, l.smem, s->stream>>>(a);
    else sgns_adjoint_kernel<V, 0><<<l.blocks, l.threads, l.smem, s->stream>>>(a);
}

void adjoint_enqueue(dg_sgns *s, const AdjLaunch &l, const AdjArgs &a) {
    switch (s->p.size) {
    case 32: adjoint_enqueue_v<1>(s, l, a); break;
    case 64: adjoint_enqueue_v<2>(s, l, a); break;
    case 128: adjoint_enqueue_v<4>(s, l, a); break;
    case 256: adjoint_enqueue_v<8>(s, l, a); break;
    default: adjoint_enqueue_v<16>(s, l, a); break;
    }
}

AdjArgs adjoint_args(dg_sgns *s, const uint32_t *inputs, const uint32_t *outputs, const uint32_t *negatives,
                     uint64_t n_pairs, uint32_t batch, int negative) {
    AdjArgs a{};
    a.inputs = inputs;
    a.outputs = outputs;
    a.negatives = negatives;
    a.n_pairs = n_pairs;
    a.n_batches = (n_pairs + batch - 1) / batch;
    a.b_begin = 0;
    a.b_end = a.n_batches;
    a.step = nullptr;
    a.batch = batch;
    a.negative = negative;
    const bool plain = dgs::fp32_rows(s);
    a.in_f32 = plain ? s->syn0.p : nullptr;
    a.out_f32 = plain ? s->syn1.p : nullptr;
    a.in_bf = s->in_bf.p;
    a.out_bf = s->out_bf.p;
    a.in_master = s->in_master.p;
    a.out_master = s->out_master.p;
    a.n_master = plain ? 0 : s->n_master;
    a.acc_in = s->adj_in.p;
    a.acc_out = s->adj_out.p;
    a.batch_loss = nullptr;
    a.flag = s->adj_flag.p;
    return a;
}

int adjoint_buffers(dg_sgns *s) {
    const uint64_t n = (uint64_t)s->vocab_size * s->p.size;
    if (s->adj_in.n != n) {
        DG_CUDA(s->adj_in.alloc(n));
        DG_CUDA(s->adj_out.alloc(n));
        s->adj_dirty = true;
    }
    if (s->adj_flag.n == 0) DG_CUDA(s->adj_flag.alloc(1));
    return DG_OK;
}

// The gradient of one set of device-resident minibatches, added to the
// accumulators (batch_loss may be NULL).  Asynchronous on the trainer's stream.
int adjoint_grad(dg_sgns *s, const uint32_t *inputs, const uint32_t *outputs, const uint32_t *negatives,
                 uint64_t n_pairs, uint32_t batch, int negative, double *batch_loss) {
    const uint64_t n_batches = (n_pairs + batch - 1) / batch;
    if (n_batches == 0) return DG_OK;
    AdjArgs a = adjoint_args(s, inputs, outputs, negatives, n_pairs, batch, negative);
    a.batch_loss = batch_loss;
    AdjLaunch l;
    int rc = adjoint_configure(s, negative, n_batches, l);
    if (rc) return rc;
    adjoint_enqueue(s, l, a);
    dg::note_launch();
    DG_CUDA(cudaGetLastError());
    return DG_OK;
}

// Uploads the pairs, clears the accumulators and runs the adjoint kernel.
int adjoint_run(dg_sgns *s, const dg_sgns_pairs *pp, double *loss) {
    DG_CHECK(pp, DG_ERR_ARG, "NULL pairs");
    DG_CHECK(pp->batch >= 1, DG_ERR_ARG, "batch must be >= 1");
    DG_CHECK(pp->negative >= 0 && pp->negative <= kAdjMaxNeg, DG_ERR_ARG, "negative %d out of range [0, %d]",
             pp->negative, kAdjMaxNeg);
    DG_CHECK(pp->n_pairs == 0 || (pp->inputs && pp->outputs), DG_ERR_ARG, "NULL pair arrays");
    const uint64_t n_batches = (pp->n_pairs + pp->batch - 1) / pp->batch;
    const uint64_t n_neg = n_batches * (uint64_t)pp->negative;
    DG_CHECK(n_neg == 0 || pp->negatives, DG_ERR_ARG, "NULL negatives");
    for (uint64_t p = 0; p < pp->n_pairs; p++)
        DG_CHECK(pp->inputs[p] < s->vocab_size && pp->outputs[p] < s->vocab_size, DG_ERR_ARG,
                 "pair %llu has a row id beyond the vocabulary (%u rows)", (unsigned long long)p, s->vocab_size);
    for (uint64_t k = 0; k < n_neg; k++)
        DG_CHECK(pp->negatives[k] < s->vocab_size, DG_ERR_ARG, "negative %llu is beyond the vocabulary (%u rows)",
                 (unsigned long long)k, s->vocab_size);
    int rc = adjoint_buffers(s);
    if (rc) return rc;
    const uint64_t n = (uint64_t)s->vocab_size * s->p.size;
    dg::DevArray<uint32_t> d_in, d_out, d_neg;
    dg::DevArray<double> d_loss;
    DG_CUDA(d_in.alloc(pp->n_pairs));
    DG_CUDA(d_out.alloc(pp->n_pairs));
    DG_CUDA(d_neg.alloc(n_neg));
    DG_CUDA(d_loss.alloc(n_batches));
    if (pp->n_pairs) {
        DG_CUDA(cudaMemcpyAsync(d_in.p, pp->inputs, pp->n_pairs * 4, cudaMemcpyHostToDevice, s->stream));
        DG_CUDA(cudaMemcpyAsync(d_out.p, pp->outputs, pp->n_pairs * 4, cudaMemcpyHostToDevice, s->stream));
    }
    if (n_neg) DG_CUDA(cudaMemcpyAsync(d_neg.p, pp->negatives, n_neg * 4, cudaMemcpyHostToDevice, s->stream));
    DG_CUDA(cudaMemsetAsync(s->adj_in.p, 0, n * 8, s->stream));
    DG_CUDA(cudaMemsetAsync(s->adj_out.p, 0, n * 8, s->stream));
    DG_CUDA(cudaMemsetAsync(s->adj_flag.p, 0, 4, s->stream));
    s->adj_dirty = true;
    rc = adjoint_grad(s, d_in.p, d_out.p, d_neg.p, pp->n_pairs, pp->batch, pp->negative, d_loss.p);
    if (rc) return rc;
    std::vector<double> bl(n_batches);
    unsigned int flag = 0;
    if (n_batches) DG_CUDA(cudaMemcpyAsync(bl.data(), d_loss.p, n_batches * 8, cudaMemcpyDeviceToHost, s->stream));
    DG_CUDA(cudaMemcpyAsync(&flag, s->adj_flag.p, 4, cudaMemcpyDeviceToHost, s->stream));
    DG_CUDA(cudaStreamSynchronize(s->stream));
    DG_CHECK(flag == 0, DG_ERR_ARG, "a gradient contribution is not finite or exceeds 2^20 in magnitude");
    if (loss) {
        double t = 0.0;
        for (double x : bl) t += x;   // minibatch order
        *loss = t;
    }
    return DG_OK;
}

}  // namespace

// A step of K minibatches gives the hottest row about
// K * (2 * batch * p_tok + negative * p_neg) contributions, all computed from
// the same row values; like the minibatch trainer's concurrent snapshots
// (dg_sgns_mb.cu), too many of them make that row overshoot.  The bound keeps
// them at kAdjMaxHot.
constexpr double kAdjMaxHot = 256.0;

uint32_t adjoint_step_bound(const std::vector<uint32_t> &cn, const std::vector<uint32_t> &keep_thr, int batch,
                            int negative) {
    if (cn.empty()) return 1;
    double p_neg, p_tok;
    hot_row_shares(cn, keep_thr, p_neg, p_tok);
    const double per_batch = 2.0 * batch * p_tok + negative * p_neg;
    const double cap = (double)(1u << 20);
    if (per_batch <= 0.0) return (uint32_t)cap;
    return (uint32_t)std::max(1.0, std::min(cap, std::floor(kAdjMaxHot / per_batch)));
}

// Adjoint mode: the pass's pairs (the plain trainer's pairs), cut into
// minibatches of batch_size pairs sharing `negative` negatives, trained by
// gradient steps of adj_step_batches minibatches (or params.workers): gradient
// at the current rows by the backward kernel, then rows -= alpha * gradient.
// Every step is deterministic, so the whole pass is.
int adjoint_train(dg_sgns *s, const SgnsArgs &a, const WalkSet &ws, uint64_t &n_pairs) {
    n_pairs = 0;
    const int neg = a.vocab_size > 1 ? a.negative : 0;
    DG_CHECK(neg <= kAdjMaxNeg, DG_ERR_ARG, "adjoint mode supports negative <= %d", kAdjMaxNeg);
    int rc = adjoint_buffers(s);
    if (rc) return rc;
    const int d = s->p.size;
    if (s->adj_dirty) {
        const uint64_t n = (uint64_t)s->vocab_size * d;
        DG_CUDA(cudaMemsetAsync(s->adj_in.p, 0, n * 8, s->stream));
        DG_CUDA(cudaMemsetAsync(s->adj_out.p, 0, n * 8, s->stream));
        s->adj_dirty = false;
    }
    DG_CUDA(cudaMemsetAsync(s->adj_flag.p, 0, 4, s->stream));
    rc = adjoint_pairs(s, a, ws, n_pairs);
    if (rc) return rc;
    if (n_pairs == 0) return DG_OK;
    const uint32_t batch = s->p.batch_size > 0 ? (uint32_t)s->p.batch_size : (uint32_t)(2 * a.window + 1);
    const uint64_t n_batches = (n_pairs + batch - 1) / batch;
    const uint64_t n_neg = n_batches * (uint64_t)neg;
    if (s->adj_neg.n < n_neg) DG_CUDA(s->adj_neg.alloc(n_neg + n_neg / 8));
    const unsigned grid = (unsigned)(dg::sm_count(s->device) * 8);
    if (n_neg) {
        adj_negatives<<<grid, 256, 0, s->stream>>>(a.table, a.table_size, a.vocab_size, a.pass, a.seed_lo,
                                                   a.seed_hi, n_batches, neg, s->adj_neg.p);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
    }
    const uint64_t k = s->p.workers ? s->p.workers : s->adj_step_batches;
    // Step parameters live on the device; the captured graph of kAdjGraphSteps
    // steps (gradient, step, advance) reads them, so it is replayed as is every
    // round and recaptured only when a buffer it points at moves.
    if (s->adj_step.n == 0) DG_CUDA(s->adj_step.alloc(1));
    const AdjStep h{n_pairs, n_batches, k, a.alpha, 0};
    DG_CUDA(cudaMemcpyAsync(s->adj_step.p, &h, sizeof(h), cudaMemcpyHostToDevice, s->stream));
    const void *key[3] = {s->adj_pin.p, s->adj_pout.p, s->adj_neg.p};
    if (!s->adj_exec || s->adj_exec_k != k || memcmp(key, s->adj_exec_key, sizeof(key)) != 0) {
        if (s->adj_exec) {
            cudaGraphExecDestroy(s->adj_exec);
            s->adj_exec = nullptr;
        }
        const bool plain = dgs::fp32_rows(s);
        AdjArgs ga = adjoint_args(s, s->adj_pin.p, s->adj_pout.p, s->adj_neg.p, 0, batch, neg);
        ga.step = s->adj_step.p;
        AdjLaunch l;
        rc = adjoint_configure(s, neg, k, l);
        if (rc) return rc;
        DG_CUDA(cudaStreamSynchronize(s->stream));
        DG_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < kAdjGraphSteps; i++) {
            adjoint_enqueue(s, l, ga);
            adjoint_apply_rows<<<grid, 256, 0, s->stream>>>(
                s->adj_in.p, s->adj_out.p, s->adj_pin.p, s->adj_pout.p, s->adj_neg.p, batch, neg, d, s->adj_step.p,
                plain ? s->syn0.p : nullptr, plain ? s->syn1.p : nullptr, s->in_bf.p, s->out_bf.p, s->in_master.p,
                s->out_master.p, plain ? 0u : s->n_master);
            adj_advance<<<1, 32, 0, s->stream>>>(s->adj_step.p);
        }
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s->stream, &graph);
        DG_CUDA(ce);
        const cudaError_t ie = cudaGraphInstantiate(&s->adj_exec, graph, 0);
        cudaGraphDestroy(graph);
        DG_CUDA(ie);
        memcpy(s->adj_exec_key, key, sizeof(key));
        s->adj_exec_k = k;
    }
    const uint64_t n_steps = (n_batches + k - 1) / k;
    for (uint64_t done = 0; done < n_steps; done += kAdjGraphSteps) {
        DG_CUDA(cudaGraphLaunch(s->adj_exec, s->stream));
        dg::note_launches(3 * kAdjGraphSteps);
    }
    unsigned int flag = 0;
    DG_CUDA(cudaMemcpyAsync(&flag, s->adj_flag.p, 4, cudaMemcpyDeviceToHost, s->stream));
    DG_CUDA(cudaStreamSynchronize(s->stream));
    if (flag) s->adj_dirty = true;
    DG_CHECK(flag == 0, DG_ERR_ARG, "a gradient contribution is not finite or exceeds 2^20 in magnitude");
    return DG_OK;
}

}  // namespace dgs

extern "C" int dg_sgns_loss_grad(dg_sgns *s, const dg_sgns_pairs *pairs, double *loss, float *grad_in,
                                 float *grad_out) {
    DG_CHECK(s, DG_ERR_ARG, "dg_sgns_loss_grad: NULL trainer");
    DG_CHECK(s->out_size == s->p.size, DG_ERR_ARG, "dg_sgns_loss_grad: size %d is stored padded; use 32 .. 512, "
             "a power of two", s->out_size);
    dg::DeviceGuard guard(s->device);
    int rc = dgs::adjoint_run(s, pairs, loss);
    if (rc) return rc;
    const uint64_t n = (uint64_t)s->vocab_size * s->p.size;
    if (!grad_in && !grad_out) return DG_OK;
    dg::DevArray<float> tmp;
    DG_CUDA(tmp.alloc(n));
    for (int k = 0; k < 2; k++) {
        float *host = k == 0 ? grad_in : grad_out;
        if (!host) continue;
        dgs::adjoint_to_f32<<<dg::sm_count(s->device) * 4, 256, 0, s->stream>>>(k == 0 ? s->adj_in.p : s->adj_out.p,
                                                                              n, tmp.p);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
        DG_CUDA(cudaMemcpyAsync(host, tmp.p, n * 4, cudaMemcpyDeviceToHost, s->stream));
        DG_CUDA(cudaStreamSynchronize(s->stream));
    }
    return DG_OK;
}

extern "C" int dg_sgns_adjoint_step(dg_sgns *s, const dg_sgns_pairs *pairs, float alpha, double *loss) {
    DG_CHECK(s, DG_ERR_ARG, "dg_sgns_adjoint_step: NULL trainer");
    DG_CHECK(s->out_size == s->p.size, DG_ERR_ARG, "dg_sgns_adjoint_step: size %d is stored padded; use 32 .. 512, "
             "a power of two", s->out_size);
    DG_CHECK(std::isfinite(alpha), DG_ERR_ARG, "alpha must be finite");
    dg::DeviceGuard guard(s->device);
    int rc = dgs::adjoint_run(s, pairs, loss);
    if (rc) return rc;
    const uint64_t n = (uint64_t)s->vocab_size * s->p.size;
    const bool plain = dgs::fp32_rows(s);
    const uint64_t nm = plain ? 0 : (uint64_t)s->n_master * s->p.size;
    for (int k = 0; k < 2; k++) {
        dgs::adjoint_apply<<<dg::sm_count(s->device) * 4, 256, 0, s->stream>>>(
            k == 0 ? s->adj_in.p : s->adj_out.p, n, alpha, plain ? (k == 0 ? s->syn0.p : s->syn1.p) : nullptr,
            k == 0 ? s->in_bf.p : s->out_bf.p, k == 0 ? s->in_master.p : s->out_master.p, nm);
        dg::note_launch();
        DG_CUDA(cudaGetLastError());
    }
    DG_CUDA(cudaStreamSynchronize(s->stream));
    return DG_OK;
}
