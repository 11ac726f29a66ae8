/*
 * Stand-in for the two MKL entry points the reference's dsgl trainer calls
 * (include/dsgl.hpp:1241, 1290, 1309 cblas_sgemm; 540 mkl_set_num_threads), used
 * ONLY to build the CPU checker oracle/_ref/ref_embed.  Plain row-major GEMM:
 * C = alpha * op(A) * op(B) + beta * C, summed in k order.  Test infrastructure.
 */
#ifndef DG_REF_SHIM_MKL_H
#define DG_REF_SHIM_MKL_H

enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

inline void mkl_set_num_threads(int) {}

inline void cblas_sgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, int M, int N, int K,
                        float alpha, const float *A, int lda, const float *B, int ldb, float beta, float *C,
                        int ldc) {
    (void)layout;  // the reference only uses row-major
    for (int i = 0; i < M; i++) {
        for (int j = 0; j < N; j++) {
            float s = 0.f;
            for (int k = 0; k < K; k++) {
                const float a = ta == CblasNoTrans ? A[i * lda + k] : A[k * lda + i];
                const float b = tb == CblasNoTrans ? B[k * ldb + j] : B[j * ldb + k];
                s += a * b;
            }
            C[i * ldc + j] = beta == 0.f ? alpha * s : alpha * s + beta * C[i * ldc + j];
        }
    }
}

#endif
