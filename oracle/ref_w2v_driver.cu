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
 * ref_w2v_huffman() runs the reference's host-side Huffman coding;
 * ref_w2v_vocab(), ref_w2v_unigram() and ref_w2v_init_rows() its vocabulary,
 * unigram table and initial rows.
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

/* The reference's vocabulary from vertex degrees: ReadVocabFromDegree
 * (word2vec.cu:791-809; word = the vertex id as text, count = its degree) with
 * SortVocab (word2vec.cu:629-659: the C library's qsort by count, min_count cut,
 * train_words), after main's allocations (word2vec.cu:1569-1570).  Host code, no
 * GPU.  Writes, in vocabulary order, each word's vertex id and count (at most
 * cap entries), the vocabulary size and train_words.  The vocabulary stays in
 * place for ref_w2v_unigram and ref_w2v_init_rows.  Returns 0, or -1 when cap
 * is smaller than the vocabulary. */
int ref_w2v_vocab(const unsigned *deg, unsigned v_num, int min_cnt, long long cap, unsigned *id_out,
                  long long *cn_out, long long *size_out, long long *train_words_out) {
    min_count = min_cnt;
    vocab_max_size = 1000;
    vocab_size = 0;
    vocab = (struct vocab_word *)calloc(vocab_max_size, sizeof(struct vocab_word));
    if (!vocab_hash) vocab_hash = (int *)calloc(vocab_hash_size, sizeof(int));
    std::vector<vertex_id_t> degrees(deg, deg + v_num);
    ReadVocabFromDegree(degrees);
    *size_out = vocab_size;
    *train_words_out = train_words;
    if (vocab_size > cap) return -1;
    for (long long a = 0; a < vocab_size; a++) {
        id_out[a] = (unsigned)strtoul(vocab[a].word, nullptr, 10);
        cn_out[a] = vocab[a].cn;
    }
    return 0;
}

/* InitUnigramTable (word2vec.cu:537-556) over the vocabulary of the last
 * ref_w2v_vocab call; copies its host table (table_size entries) to table_out.
 * Needs a GPU (the function also uploads the table).  Returns 0 or the CUDA
 * error code. */
int ref_w2v_unigram(int *table_out) {
    InitUnigramTable();
    memcpy(table_out, table, (size_t)table_size * sizeof(int));
    free(table);
    table = nullptr;
    cudaFree(d_table);
    d_table = nullptr;
    return (int)cudaGetLastError();
}

/* InitNet (word2vec.cu:844-878) for the last vocabulary with d columns and
 * negative sampling: copies the host syn0 (vocab_size x d, the LCG-initialised
 * input rows) to rows_out.  Needs a GPU (InitNet uploads the rows and the
 * Huffman codes).  Returns 0 or the CUDA error code. */
int ref_w2v_init_rows(int d, float *rows_out) {
    layer1_size = d;
    negative = 5;
    hs = 0;
    InitNet();
    memcpy(rows_out, syn0, (size_t)vocab_size * d * sizeof(float));
    free(syn0);
    free(syn1neg);
    free(last_emb);
    syn0 = syn1neg = last_emb = nullptr;
    cudaFree(d_syn0);
    cudaFree(d_syn1);
    d_syn0 = d_syn1 = nullptr;
    return (int)cudaGetLastError();
}

}  // extern "C"
