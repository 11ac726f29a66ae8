/*
 * CPU checker: drives the reference's UNMODIFIED walk engine
 * (include/walk.hpp WalkEngine::random_walk, walk.hpp:512) the way the walk
 * section of src/examples/huge_walk.cpp:79-113 would, one process, no MPI
 * (oracle/ref_shim/mpi.h stands in for a one-rank world).
 *
 * Test infrastructure only: built into oracle/_ref/ by oracle/Makefile from the
 * reference sources where they lie; never linked into the shipped library.
 *
 * Determinism for the pin test: with `-t 1` the engine runs one worker thread,
 * so walkers are advanced in ascending id order and both random streams are
 * consumed in a fixed order.  The candidate stream is the engine's own
 * mt19937 + uniform_int_distribution (util.hpp:22-47); its seed normally comes
 * from std::random_device, which this file pins to a constant (below).  The
 * acceptance stream is glibc rand() (walk.hpp:928), deterministic because the
 * walk path never calls srand().
 *
 * Usage: ref_walk -g edges.bin -v V -w W --min_L L --min_R R -o prefix
 *                 [--make-undirected] [-t threads] [--seed S]
 * Prints one line "ref_walk total_s=... dump_s=... walk_s=..." on stdout.
 */
#include "walk.hpp"

#include <cstdlib>
#include <cstring>
#include <string>

static unsigned int g_pinned_seed = 5489u;

// Every std::random_device draw returns the pinned seed, so each worker's
// mt19937 starts from a known state.  Interposes libstdc++'s out-of-line helper.
unsigned int std::random_device::_M_getval() { return g_pinned_seed; }

int main(int argc, char **argv) {
    std::string graph_path, out_prefix;
    vertex_id_t v_num = 0, walker_num = 0, min_len = 20, min_round = 5;
    bool undirected = false;
    int threads = 1;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&]() -> const char * {
            if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); exit(2); }
            return argv[++i];
        };
        if (a == "-g") graph_path = next();
        else if (a == "-v") v_num = (vertex_id_t)strtoul(next(), nullptr, 10);
        else if (a == "-w") walker_num = (vertex_id_t)strtoul(next(), nullptr, 10);
        else if (a == "--min_L") min_len = (vertex_id_t)strtoul(next(), nullptr, 10);
        else if (a == "--min_R") min_round = (vertex_id_t)strtoul(next(), nullptr, 10);
        else if (a == "-o") out_prefix = next();
        else if (a == "--make-undirected") undirected = true;
        else if (a == "-t") threads = atoi(next());
        else if (a == "--seed") g_pinned_seed = (unsigned int)strtoul(next(), nullptr, 10);
        else { fprintf(stderr, "unknown flag %s\n", a.c_str()); return 2; }
    }
    if (graph_path.empty() || v_num == 0 || walker_num == 0 || out_prefix.empty()) {
        fprintf(stderr, "usage: ref_walk -g edges.bin -v V -w W --min_L L --min_R R -o prefix [--make-undirected] [-t T]\n");
        return 2;
    }

    MPI_Instance mpi_instance(&argc, &argv);
    Timer total;
    WalkEngine<real_t, uint32_t> graph;
    graph.set_concurrency(threads);
    graph.set_init_round(min_round);
    graph.set_minLength(min_len);
    graph.load_graph(v_num, graph_path.c_str(), "", undirected);
    graph.vertex_cn.resize(graph.get_vertex_num());

    auto extension_comp = [&](Walker<uint32_t> &walker, vertex_id_t) { return walker.step >= 40 ? 0.0 : 1.0; };
    WalkerConfig<real_t, uint32_t> walker_conf(walker_num);
    TransitionConfig<real_t, uint32_t> tr_conf(extension_comp);
    WalkConfig walk_conf;
    walk_conf.set_output_file(out_prefix.c_str());

    Timer walk_timer;
    graph.random_walk(&walker_conf, &tr_conf, &walk_conf);
    double walk_total = walk_timer.duration();
    printf("ref_walk total_s=%.6f random_walk_s=%.6f dump_s=%.6f walk_s=%.6f threads=%d\n",
           total.duration(), walk_total, graph.other_time, walk_total - graph.other_time, threads);
    fflush(stdout);
    // Skip the engine's teardown: nothing after this point is measured or checked.
    _exit(0);
}
