/*
 * CPU baseline: the reference's UNMODIFIED walk engine followed by its dsgl SGNS
 * trainer (include/dsgl.hpp:1464, MKL branch), one process, chained the way the
 * commented-out tail of src/examples/huge_walk.cpp:79-133 chains them:
 * random_walk -> get_new_sort -> dsgl(vertex_cn, new_sort, graph).
 *
 * Test / baseline infrastructure only: built into oracle/_ref/ by
 * `make -C oracle ref` from the reference headers where they lie, with the
 * one-rank MPI and naive-GEMM stand-ins of oracle/ref_shim/.
 *
 * Bounded samples: the engine always runs 30 rounds (walk.hpp:740), so
 * --walk-rounds R stops after round R through the engine's own per-round
 * output hook (WalkConfig::set_output_consumer, walk.hpp:120-125, 757-759), and
 * --sgns-words N trains dsgl on the first walks of the corpus holding >= N
 * tokens.  Walk time excludes the engine's walk-file dump and path assembly
 * (its other_time, as huge_walk.cpp:110-111 reports it).
 *
 * Usage: ref_embed -g edges.bin -v V -w W --min_L L --min_R R --make-undirected
 *                  -t walk_threads [--walk-rounds R] [--sgns-words N]
 *                  [dsgl flags: -size -window -negative -sample -alpha -iter
 *                   -min-count -threads -eoutput ...]
 * Prints "ref_embed walk_s=... walks=... footprints=... sgns_s=... sgns_words=..."
 */
#define USE_MKL 1
#include "walk.hpp"
#include "dsgl.hpp"

#include <cstdlib>
#include <string>

int main(int argc, char **argv) {
    std::string graph_path, prefix = "/tmp/ref_embed_walks";
    vertex_id_t v_num = 0, walker_num = 0, min_len = 20, min_round = 5;
    bool undirected = false;
    int threads = 1, walk_rounds = 30;
    size_t sgns_words = 0;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto val = [&]() -> const char * { return i + 1 < argc ? argv[++i] : ""; };
        if (a == "-g") graph_path = val();
        else if (a == "-v") v_num = (vertex_id_t)strtoul(val(), nullptr, 10);
        else if (a == "-w") walker_num = (vertex_id_t)strtoul(val(), nullptr, 10);
        else if (a == "--min_L") min_len = (vertex_id_t)strtoul(val(), nullptr, 10);
        else if (a == "--min_R") min_round = (vertex_id_t)strtoul(val(), nullptr, 10);
        else if (a == "-o") prefix = val();
        else if (a == "--make-undirected") undirected = true;
        else if (a == "-t") threads = atoi(val());
        else if (a == "--walk-rounds") walk_rounds = atoi(val());
        else if (a == "--sgns-words") sgns_words = strtoull(val(), nullptr, 10);
    }
    if (graph_path.empty() || v_num == 0 || walker_num == 0) {
        fprintf(stderr, "usage: ref_embed -g edges.bin -v V -w W [--min_L L] [--min_R R] [-t T] [dsgl flags]\n");
        return 2;
    }
    MPI_Instance mpi_instance(&argc, &argv);
    WalkEngine<real_t, uint32_t> engine;
    engine.set_concurrency(threads);
    engine.set_init_round(min_round);
    engine.set_minLength(min_len);
    engine.load_graph(v_num, graph_path.c_str(), "", undirected);
    engine.vertex_cn.resize(engine.get_vertex_num());
    auto extension_comp = [&](Walker<uint32_t> &walker, vertex_id_t) { return walker.step >= 40 ? 0.0 : 1.0; };
    WalkerConfig<real_t, uint32_t> walker_conf(walker_num);
    TransitionConfig<real_t, uint32_t> tr_conf(extension_comp);
    WalkConfig walk_conf;
    walk_conf.set_output_file(prefix.c_str());
    Timer walk_timer;
    int rounds_done = 0;
    auto finish = [&]() {
        const double walk_s = walk_timer.duration() - engine.other_time;
        size_t walks = 0, footprints = 0;
        for (int x : engine.local_corpus) (x < 0 ? walks : footprints)++;
        if (sgns_words) {
            size_t keep = 0;
            while (keep < engine.local_corpus.size() && keep < sgns_words) keep++;
            while (keep < engine.local_corpus.size() && engine.local_corpus[keep - 1] != -1) keep++;
            engine.local_corpus.resize(keep);
        }
        size_t words = 0;
        for (int x : engine.local_corpus) words += x >= 0;
        engine.get_new_sort();
        Timer sgns_timer;
        dsgl(argc, argv, &engine.vertex_cn, &engine.new_sort, &engine);
        const double sgns_s = sgns_timer.duration();
        printf("\nref_embed walk_s=%.6f rounds=%d walks=%zu footprints=%zu sgns_s=%.6f sgns_words=%zu "
               "walk_threads=%d\n", walk_s, rounds_done, walks, footprints, sgns_s, words, threads);
        fflush(stdout);
        _exit(0);
    };
    double last_t = 0.0, last_other = 0.0;
    walk_conf.set_output_consumer([&](PathSet *paths) {
        // Per-round walk time: wall time since the previous round minus the
        // engine's own assemble + dump time of this round.
        size_t fp = 0, walks = 0;
        for (int s = 0; s < paths->seg_num; s++)
            for (walker_id_t w = 0; w < paths->path_num[s]; w++) { fp += paths->path_length[s][w]; walks++; }
        const double now = walk_timer.duration();
        printf("\nref_round r=%d walk_s=%.6f walks=%zu footprints=%zu\n", rounds_done + 1,
               (now - last_t) - (engine.other_time - last_other), walks, fp);
        fflush(stdout);
        last_t = now;
        last_other = engine.other_time;
        delete paths;
        if (++rounds_done >= walk_rounds) finish();
    });
    engine.random_walk(&walker_conf, &tr_conf, &walk_conf);
    finish();
}
