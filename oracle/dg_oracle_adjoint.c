/*
 * FP64 reference of the SGNS loss and its gradient over explicit minibatches --
 * test infrastructure only (the checker of the device adjoint kernel).
 *
 * Loss: the objective that word2vec.cu's skip_gram_kernel (word2vec.cu:305-399)
 * and dsgl's minibatch update (dsgl.hpp:1241-1311) descend with their fused
 * updates, with the exact logistic sigmoid:
 *   L = sum over pairs (i, o) of softplus(-v_i . u_o)
 *       + sum over the pair's minibatch negatives k of softplus(v_i . u_k).
 * Gradient: dL/dv_i += (s(v.u_o) - 1) u_o + sum_k s(v.u_k) u_k,
 *           dL/du_o += (s(v.u_o) - 1) v_i,  dL/du_k += s(v.u_k) v_i.
 *
 * only_table / only_row (row >= 0) restrict the sum to the pairs whose terms
 * depend on that row (table 0: pairs with input == row; table 1: pairs with
 * output == row or with row among their minibatch's negatives), for central
 * finite differences that do not drown in the rest of the sum.
 */
#include "dg_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

static double softplus(double x) { return fmax(x, 0.0) + log1p(exp(-fabs(x))); }
static double sigmoid(double x) { return x >= 0 ? 1.0 / (1.0 + exp(-x)) : exp(x) / (1.0 + exp(x)); }

static double dot(const double *a, const double *b, int d) {
    double s = 0.0;
    for (int c = 0; c < d; c++) s += a[c] * b[c];
    return s;
}

int dgo_sgns_loss_grad(const double *in, const double *out, int d, uint32_t vocab_size, const uint32_t *inputs,
                       const uint32_t *outputs, const uint32_t *negatives, uint64_t n_pairs, uint32_t batch,
                       int negative, int only_table, int64_t only_row, double *loss, double *grad_in,
                       double *grad_out) {
    if (batch < 1 || negative < 0 || d < 1) return -1;
    if (grad_in) memset(grad_in, 0, sizeof(double) * (size_t)vocab_size * d);
    if (grad_out) memset(grad_out, 0, sizeof(double) * (size_t)vocab_size * d);
    double total = 0.0;
    for (uint64_t p = 0; p < n_pairs; p++) {
        const uint64_t b = p / batch;
        const uint32_t i = inputs[p], o = outputs[p];
        const uint32_t *neg = negatives + b * (uint64_t)negative;
        if (i >= vocab_size || o >= vocab_size) return -1;
        if (only_row >= 0) {
            int hit = 0;
            if (only_table == 0) {
                hit = i == (uint32_t)only_row;
            } else {
                hit = o == (uint32_t)only_row;
                for (int k = 0; k < negative && !hit; k++) hit = neg[k] == (uint32_t)only_row;
            }
            if (!hit) continue;
        }
        const double *v = in + (size_t)i * d, *uo = out + (size_t)o * d;
        const double s = dot(v, uo, d);
        total += softplus(-s);
        const double g = sigmoid(s) - 1.0;
        for (int c = 0; c < d; c++) {
            if (grad_in) grad_in[(size_t)i * d + c] += g * uo[c];
            if (grad_out) grad_out[(size_t)o * d + c] += g * v[c];
        }
        for (int k = 0; k < negative; k++) {
            const uint32_t w = neg[k];
            if (w >= vocab_size) return -1;
            const double *uk = out + (size_t)w * d;
            const double sk = dot(v, uk, d);
            total += softplus(sk);
            const double gk = sigmoid(sk);
            for (int c = 0; c < d; c++) {
                if (grad_in) grad_in[(size_t)i * d + c] += gk * uk[c];
                if (grad_out) grad_out[(size_t)w * d + c] += gk * v[c];
            }
        }
    }
    if (loss) *loss = total;
    return 0;
}
