/*
 * The reference's own word2vec.cu CUDA kernels, compiled unmodified for sm_100a
 * as the checker of the SGNS restatement (oracle/dg_oracle_w2v.c).  TEST
 * INFRASTRUCTURE ONLY: built into oracle/_ref/libref_w2v.so by `make -C oracle
 * ref` from src/word2vec.cu where it lies (the translation unit below includes
 * it), with the project-written hnswlib stand-in of oracle/ref_shim/.  The
 * shipped library never links it.
 *
 * ref_w2v_launch() sets the globals the reference's launchers read and calls
 * those launchers themselves: sgKernel (word2vec.cu:905-949: skip_gram_kernel,
 * or __sgNegReuse when reuseNeg is set) and cbowKernel (word2vec.cu:879-903),
 * with reduSize computed as TrainModelThread computes it (word2vec.cu:971-973).
 * All pointers are device pointers owned by the caller; the table must hold
 * the reference's fixed table_size (1e8, word2vec.cu:66) entries.
 * ref_w2v_huffman() runs the reference's host-side Huffman coding.
 */
#include "word2vec.cu"

extern "C" {

/* kind: 0 skip_gram_kernel, 1 cbow_kernel, 2 __sgNegReuse.  Returns 0, or the
 * CUDA error code of the launch / synchronisation. */
int ref_w2v_launch(int kind, int d, int win, int neg, int use_hs, long long vocab_sz, float lr,
                   const float *exp_table, const int *unigram, const int *codelen, const int *point,
                   const char *code, float *rows_in, float *rows_out, int *sentences, int *sentence_offsets,
                   int *neg_samples, int cnt_sentence) {
    layer1_size = d;
    window = win;
    negative = neg;
    hs = use_hs;
    vocab_size = vocab_sz;
    reuseNeg = kind == 2 ? 1 : 0;
    d_expTable = const_cast<float *>(exp_table);
    d_table = const_cast<int *>(unigram);
    d_vocab_codelen = const_cast<int *>(codelen);
    d_vocab_point = const_cast<int *>(point);
    d_vocab_code = const_cast<char *>(code);
    d_syn0 = rows_in;
    d_syn1 = rows_out;
    int reduSize = 32;
    while (reduSize < layer1_size) reduSize *= 2;
    if (kind == 1)
        cbowKernel(sentences, sentence_offsets, lr, cnt_sentence, reduSize);
    else
        sgKernel(sentences, sentence_offsets, neg_samples, lr, cnt_sentence, reduSize);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

/* The reference's own Huffman coding (CreateBinaryTree, word2vec.cu:684-740) of
 * n words with counts cn (in vocabulary order, most frequent first): host code,
 * no GPU.  Writes codelen[n] and, per word, MAX_CODE_LENGTH (40) entries of
 * point[] and code[] (only the first codelen are meaningful).  Returns 0. */
int ref_w2v_huffman(const long long *cn, long long n, int *codelen_out, int *point_out, char *code_out) {
    vocab_size = n;
    vocab = (struct vocab_word *)calloc(n + 1, sizeof(struct vocab_word));
    for (long long a = 0; a < n; a++) {
        vocab[a].cn = cn[a];
        vocab[a].code = (char *)calloc(MAX_CODE_LENGTH, sizeof(char));
        vocab[a].point = (int *)calloc(MAX_CODE_LENGTH, sizeof(int));
    }
    CreateBinaryTree();
    for (long long a = 0; a < n; a++) {
        codelen_out[a] = vocab[a].codelen;
        for (int j = 0; j < MAX_CODE_LENGTH; j++) {
            point_out[a * MAX_CODE_LENGTH + j] = vocab[a].point[j];
            code_out[a * MAX_CODE_LENGTH + j] = vocab[a].code[j];
        }
        free(vocab[a].code);
        free(vocab[a].point);
    }
    free(vocab);
    vocab = nullptr;
    return 0;
}

/* The reference's fixed unigram-table size (word2vec.cu:66). */
int ref_w2v_table_size(void) { return table_size; }

}  // extern "C"
