/*
 * Runs the reference's UNMODIFIED dsgl trainer (include/dsgl.hpp:1464, MKL
 * branch, with the naive-GEMM and one-rank MPI stand-ins of oracle/ref_shim/)
 * on a given corpus and dumps its exact rows, as the pin of the minibatch
 * restatement (dgo_dsgl_ref in oracle/dg_oracle_dsgl.c).  TEST INFRASTRUCTURE
 * ONLY: built into oracle/_ref/ref_dsgl by `make -C oracle ref`.
 *
 * Determinism: with -threads 2, dsgl runs one model-sync thread and one compute
 * thread (dsgl.hpp:533-544); the compute thread's random stream is the LCG
 * seeded with its global thread index 0 (dsgl.hpp:780), so the run is fixed by
 * its inputs as long as no model sync overlaps training.  At one rank a sync
 * copies rows out and back unchanged (dsgl.hpp:700-747), but it could
 * overwrite a row the compute thread updates meanwhile; the caller passes a
 * -sync-period well above the training time, so the only sync runs after the
 * compute thread has finished.
 *
 * Input  (--corpus): u32 n_vertices, i32 counts[n] (vertex_cn), u64 n_tokens,
 *                    i32 tokens[n_tokens] (vertex ids, walks ended by -1).
 * Output (--dump):   u64 vocab_size, u64 size, u32 ids[vocab] (v_vocab order),
 *                    f32 Wih[vocab * size], f32 Woh[vocab * size], f32 alpha.
 * All other arguments are passed to dsgl() unchanged (-size -window -negative
 * -sample -alpha -iter -threads -sync-period -eoutput ...).
 */
#define USE_MKL 1
#include "walk.hpp"
#include "dsgl.hpp"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

static bool read_all(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n; }

int main(int argc, char **argv) {
    std::string corpus_path, dump_path;
    for (int i = 1; i + 1 < argc; i++) {
        if (!strcmp(argv[i], "--corpus")) corpus_path = argv[i + 1];
        if (!strcmp(argv[i], "--dump")) dump_path = argv[i + 1];
    }
    if (corpus_path.empty() || dump_path.empty()) {
        fprintf(stderr, "usage: ref_dsgl --corpus in.bin --dump out.bin [dsgl flags]\n");
        return 2;
    }
    FILE *f = fopen(corpus_path.c_str(), "rb");
    if (!f) { perror("corpus"); return 1; }
    uint32_t n = 0;
    uint64_t nt = 0;
    std::vector<int> counts;
    std::vector<int> tokens;
    bool ok = read_all(f, &n, 4);
    if (ok) { counts.resize(n); ok = read_all(f, counts.data(), 4ull * n); }
    if (ok) ok = read_all(f, &nt, 8);
    if (ok) { tokens.resize(nt); ok = read_all(f, tokens.data(), 4ull * nt); }
    fclose(f);
    if (!ok) { fprintf(stderr, "corpus: short read\n"); return 1; }

    MPI_Instance mpi_instance(&argc, &argv);
    WalkEngine<real_t, uint32_t> engine;
    engine.local_corpus = tokens;
    std::vector<int> vertex_cn(counts);
    std::vector<vertex_id_t> order(n);
    for (uint32_t v = 0; v < n; v++) order[v] = v;
    dsgl(argc, argv, &vertex_cn, &order, &engine);

    FILE *o = fopen(dump_path.c_str(), "wb");
    if (!o) { perror("dump"); return 1; }
    const uint64_t vs = vocab_size, hs = hidden_size;
    fwrite(&vs, 8, 1, o);
    fwrite(&hs, 8, 1, o);
    for (uint64_t a = 0; a < vs; a++) {
        const uint32_t id = v_vocab[a].id;
        fwrite(&id, 4, 1, o);
    }
    fwrite(Wih, sizeof(real), vs * hs, o);
    fwrite(Woh, sizeof(real), vs * hs, o);
    const float a_final = alpha;
    fwrite(&a_final, 4, 1, o);
    fclose(o);
    fflush(stdout);
    _exit(0);
}
