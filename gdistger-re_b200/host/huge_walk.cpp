// huge_walk: the embedding job of the reference's src/examples/huge_walk.cpp on one
// GPU, over the distger C ABI (include/distger.h).
//
// Flow (huge_walk.cpp:19-62 + word2vec.cu TrainModel, word2vec.cu:1246-1297):
// load the edge file into a device CSR, build the SGNS vocabulary from the
// vertices' in+out degrees (huge_walk.cpp:40-44, word2vec.cu:791-809), then run
// the walk rounds of WalkEngine::random_walk (walk.hpp:609-782: round 1 with
// -w x --min_R walkers, then -w walkers per round, 30 rounds) and stream every
// trained round's walks straight into the trainer with the round's learning
// rate from the schedule.  The reference writes each round to
// ./out/tmp-0-<r>.txt and trains on files 3..30 (word2vec.cu:1285-1296), with
// alpha = ExponentialDecayLR(0.025, 0.1).get_lr() per file (word2vec.cu:1279-1290:
// the schedule overrides -alpha and the -cbow default of 0.05); here the walks
// stay in HBM and are written only when -o is given, and those are the defaults.
//
// Flags kept from the reference (option_helper.hpp:112-156, word2vec.cu:1546-1565,
// dsgl.hpp:1496-1535):
//   -g <edges.bin> -v <vertices> -w <walkers> [-o <walk prefix>] [--min_L n]
//   [--min_R n] [--make-undirected] [-r rate: accepted, unused as in walk.hpp:616]
//   -size -window -negative -batch-size -sample -alpha -iter -min-count
//   -emb_output <file> (word2vec.cu) or -eoutput <file> (dsgl)
//   -cbow 0|1 (default 1, word2vec.cu:59): cbow_kernel; -cbow 0 selects skip-gram,
//     with -reuse-neg 1 (default, word2vec.cu:59) __sgNegReuse's shared
//     negatives, with -reuse-neg 0 skip_gram_kernel (word2vec.cu:1073-1076, 912)
//   -threads / -debug / -sync-size / -sync-period ...: accepted, no effect on one GPU
//   -hs 0|1 (default 0, word2vec.cu:66): hierarchical softmax before negative sampling
//   -binary: only 0 is supported (text output)
// Added for the GPU build:
//   -mode plain|plain_bf16|minibatch|cbow|cbow_bf16|sg_shared   trainer form,
//                           overriding -cbow / -reuse-neg (plain = skip_gram_kernel on
//                           FP32 rows; plain_bf16 / cbow_bf16: the rule on BF16 rows;
//                           minibatch: dsgl)
//   -lr exp|fixed|cosine|step|custom   per-round schedule (default exp, decay 0.1)
//   -lr-start a             the schedule's first rate (default 0.025, word2vec.cu:1279;
//                           -alpha does not change it, as in the reference)
//   -rounds n               stop after round n (default 30)
//   -train-from n           first round whose walks are trained (default 3,
//                           word2vec.cu:1286)
//   -seed s  -device d  -master-rows n  -table-size n  -max-len n
//   -deterministic 0|1|2    0 Hogwild, 1 one worker in order, 2 adjoint gradient steps
//   -workers n              concurrent trainer workers (0 = automatic)
//   -autotune 0|1           time the kernels' launch shapes first (default 1)
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "distger.h"
#include "lr_scheduler.h"

namespace {

struct Options {
    std::string graph, walk_prefix, emb_output, mode, lr = "exp";
    uint32_t v_num = 0, walker_num = 0, min_len = 0, init_round = 0;
    bool undirected = false;
    int size = 100, window = 5, negative = 5, batch_size = 11, iter = 5, min_count = 5;
    float sample = 1e-3f, alpha = 0.025f, lr_start = 0.025f;
    bool alpha_set = false;
    int cbow = 1, reuse_neg = 1, hs = 0;  // word2vec.cu:59, 66
    int rounds = 30, train_from = 3, device = 0, deterministic = 0, max_len = 0;
    uint64_t seed = 1;
    uint32_t master_rows = 0, workers = 0;
    int autotune = 1;
    uint64_t table_size = 0;
};

[[noreturn]] void die(const char *what) {
    fprintf(stderr, "huge_walk: %s\n", what);
    exit(2);
}

void check(int rc, const char *call) {
    if (rc != DG_OK) {
        fprintf(stderr, "huge_walk: %s failed (%d): %s\n", call, rc, dg_last_error());
        exit(1);
    }
}

Options parse(int argc, char **argv) {
    Options o;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto val = [&]() -> const char * {
            if (i + 1 >= argc) die(("missing value for " + a).c_str());
            return argv[++i];
        };
        auto u32 = [&]() { return static_cast<uint32_t>(strtoul(val(), nullptr, 10)); };
        auto i32 = [&]() { return atoi(val()); };
        if (a == "-g" || a == "--graph") o.graph = val();
        else if (a == "-v" || a == "--vertex") o.v_num = u32();
        else if (a == "-w" || a == "--walker") o.walker_num = u32();
        else if (a == "-o" || a == "--output") o.walk_prefix = val();
        else if (a == "--min_L") o.min_len = u32();
        else if (a == "--min_R") o.init_round = u32();
        else if (a == "--make-undirected") o.undirected = true;
        else if (a == "-p" || a == "--partition") die("partition files split the graph across MPI ranks; one GPU holds it all");
        else if (a == "-r" || a == "--rate") val();
        else if (a == "-size") o.size = i32();
        else if (a == "-window") o.window = i32();
        else if (a == "-negative") o.negative = i32();
        else if (a == "-batch-size") o.batch_size = i32();
        else if (a == "-sample") o.sample = static_cast<float>(atof(val()));
        else if (a == "-alpha") { o.alpha = static_cast<float>(atof(val())); o.alpha_set = true; }
        else if (a == "-iter") o.iter = i32();
        else if (a == "-min-count") o.min_count = i32();
        else if (a == "-emb_output" || a == "-eoutput") o.emb_output = val();
        else if (a == "-threads" || a == "-debug" || a == "-train" || a == "-disk" || a == "-sync-size" ||
                 a == "-sync-period" || a == "-min-sync-words" || a == "-full-sync-times" || a == "-message-size" ||
                 a == "-save-vocab" || a == "-read-vocab" || a == "-classes")
            val();
        else if (a == "-cbow") o.cbow = i32();
        else if (a == "-reuse-neg") o.reuse_neg = i32();
        else if (a == "-hs") o.hs = i32();
        else if (a == "-binary") {
            if (atoi(val()) != 0) die("-binary 1 is not supported: the embedding is written as text");
        }
        else if (a == "-mode") o.mode = val();
        else if (a == "-lr") o.lr = val();
        else if (a == "-lr-start") o.lr_start = static_cast<float>(atof(val()));
        else if (a == "-rounds") o.rounds = i32();
        else if (a == "-train-from") o.train_from = i32();
        else if (a == "-seed") o.seed = strtoull(val(), nullptr, 10);
        else if (a == "-device") o.device = i32();
        else if (a == "-deterministic") o.deterministic = i32();
        else if (a == "-master-rows") o.master_rows = u32();
        else if (a == "-table-size") o.table_size = strtoull(val(), nullptr, 10);
        else if (a == "-max-len") o.max_len = i32();
        else if (a == "-workers") o.workers = u32();
        else if (a == "-autotune") o.autotune = i32();
        else die(("unknown flag " + a).c_str());
    }
    // option_helper.hpp asserts -v, -g, --min_L, --min_R and -w are present.
    if (o.graph.empty() || o.v_num == 0 || o.walker_num == 0)
        die("usage: huge_walk -g edges.bin -v V -w W [--min_L L] [--min_R R] [--make-undirected] [-o prefix] "
            "[-size d -window k -negative n -batch-size b -sample s -alpha a -iter i -min-count c "
            "-emb_output file] [-cbow 0|1 -reuse-neg 0|1] [-mode plain|plain_bf16|minibatch|cbow|cbow_bf16|sg_shared]");
    if (o.mode.empty()) o.mode = o.cbow ? "cbow" : o.reuse_neg ? "sg_shared" : "plain";
    // word2vec.cu:1554-1555: -cbow 1 sets alpha = 0.05 unless -alpha is given (the
    // per-round schedule then overrides it, word2vec.cu:1290).
    if ((o.mode == "cbow" || o.mode == "cbow_bf16") && !o.alpha_set) o.alpha = 0.05f;
    if (o.mode != "plain" && o.mode != "minibatch" && o.mode != "plain_bf16" && o.mode != "cbow" &&
        o.mode != "cbow_bf16" && o.mode != "sg_shared")
        die("-mode must be plain, plain_bf16, minibatch, cbow, cbow_bf16 or sg_shared");
    if (o.rounds < 1 || o.rounds > 30) die("-rounds must be 1..30 (walk.hpp:740 stops after round 30)");
    return o;
}

std::unique_ptr<dg_host::LR> make_lr(const Options &o) {
    // word2vec.cu:1279 hard-codes ExponentialDecayLR(0.025, 0.1); -lr-start moves its start.
    const float a0 = o.lr_start;
    if (o.lr == "exp") return std::make_unique<dg_host::ExponentialDecayLR>(a0, 0.1f);
    if (o.lr == "fixed") return std::make_unique<dg_host::FixedLR>(a0);
    if (o.lr == "cosine") return std::make_unique<dg_host::CosineAnnealingLR>(a0, a0 * 1e-4f, o.rounds);
    if (o.lr == "step") return std::make_unique<dg_host::StepDecayLR>(a0, 0.5f, 3);
    if (o.lr == "custom") return std::make_unique<dg_host::CustomLR>(a0);
    die("-lr must be exp, fixed, cosine, step or custom");
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

int main(int argc, char **argv) {
    const Options o = parse(argc, argv);
    const auto t_start = std::chrono::steady_clock::now();

    dg_graph *g = nullptr;
    check(dg_graph_create(o.graph.c_str(), o.v_num, o.undirected ? 1 : 0, o.device, &g), "dg_graph_create");
    dg_graph_info gi{};
    check(dg_graph_get_info(g, &gi), "dg_graph_get_info");
    const double load_s = seconds_since(t_start);
    printf("graph %s: %u vertices, %llu CSR entries, %.1f MB on device, load %.3f s\n", o.graph.c_str(), gi.v_num,
           static_cast<unsigned long long>(gi.m), gi.device_bytes / 1e6, load_s);

    // Vocabulary counts: in + out degree per vertex (huge_walk.cpp:40-44).
    std::vector<uint32_t> out_deg(o.v_num), in_deg(o.v_num), counts(o.v_num);
    check(dg_graph_copy_csr(g, nullptr, nullptr, nullptr, out_deg.data(), in_deg.data()), "dg_graph_copy_csr");
    for (uint32_t v = 0; v < o.v_num; v++) counts[v] = out_deg[v] + in_deg[v];

    dg_sgns_params sp{};
    sp.size = o.size;
    sp.window = o.window;
    sp.negative = o.negative;
    sp.batch_size = o.batch_size;
    sp.sample = o.sample;
    sp.alpha = o.alpha;
    sp.iter = o.iter;
    sp.min_count = o.min_count;
    sp.mode = o.mode == "plain"        ? DG_SGNS_PLAIN
              : o.mode == "plain_bf16" ? DG_SGNS_PLAIN_BF16
              : o.mode == "cbow"       ? DG_SGNS_CBOW
              : o.mode == "cbow_bf16"  ? DG_SGNS_CBOW_BF16
              : o.mode == "sg_shared"  ? DG_SGNS_SG_SHARED
                                       : DG_SGNS_MINIBATCH;
    sp.deterministic = o.deterministic;
    sp.seed = o.seed;
    sp.table_size = o.table_size;
    sp.master_rows = o.master_rows;
    sp.workers = o.workers;
    sp.hs = o.hs;
    dg_sgns *s = nullptr;
    check(dg_sgns_create(&sp, o.v_num, counts.data(), o.device, &s), "dg_sgns_create");
    dg_sgns_info si{};
    check(dg_sgns_get_info(s, &si), "dg_sgns_get_info");
    printf("vocab %u rows, d=%d, mode %s, %u FP32 master rows, table %llu\n", si.vocab_size, o.size, o.mode.c_str(),
           si.master_rows, static_cast<unsigned long long>(si.table_size));

    dg_walk_params wp{};
    wp.min_len = o.min_len ? o.min_len : 20;       // walk.hpp:404, set_minLength ignores 0
    wp.init_round = o.init_round ? o.init_round : 5;  // walk.hpp:405, set_init_round ignores 0
    wp.walker_num = o.walker_num;
    wp.max_len = static_cast<uint32_t>(o.max_len);
    wp.seed = o.seed;

    auto lr = make_lr(o);
    if (o.autotune) {
        // Launch shapes timed on this graph; walks do not depend on them and the
        // trial rounds' visit counts are rolled back.
        dg_tune_info ti{};
        check(dg_walk_autotune(g, &wp, 2, 0, &ti), "dg_walk_autotune");
        printf("autotune walk_kernel: shape %d of %d (%d walks per block, %d cached steps)\n", ti.chosen,
               ti.n_candidates, ti.shape[ti.chosen][0], ti.shape[ti.chosen][1]);
    }
    const auto t_embed = std::chrono::steady_clock::now();
    double walk_ms = 0, train_ms = 0, device_ms = 0;
    uint64_t steps = 0, footprints = 0, words = 0, pairs = 0;
    for (int r = 1; r <= o.rounds; r++) {
        dg_paths *keep = nullptr;
        dg_paths **keep_arg = o.walk_prefix.empty() ? nullptr : &keep;
        if (r >= o.train_from && o.autotune && r == o.train_from) {
            // The first trained round's walks also time the trainer's launch
            // shapes (rows are restored after every trial), then train.
            const float alpha = lr->get_lr();
            dg_paths *p = nullptr;
            check(dg_walk_run_round(g, &wp, static_cast<uint32_t>(r), 0, &p), "dg_walk_run_round");
            dg_tune_info ti{};
            check(dg_sgns_autotune(s, p, &ti), "dg_sgns_autotune");
            if (ti.n_candidates > 1)
                printf("autotune SGNS: shape %d of %d (%d threads per block, %d blocks per SM)\n", ti.chosen,
                       ti.n_candidates, ti.shape[ti.chosen][0], ti.shape[ti.chosen][1]);
            dg_round_info ri{};
            check(dg_paths_get_info(p, &ri), "dg_paths_get_info");
            dg_train_info tr{};
            check(dg_sgns_train_paths(s, p, alpha, &tr), "dg_sgns_train_paths");
            walk_ms += ri.walk_ms;
            train_ms += tr.train_ms;
            device_ms += ri.walk_ms + tr.train_ms;
            steps += ri.steps;
            footprints += ri.footprints;
            words += tr.words;
            pairs += tr.pairs;
            printf("round %d: walks %u steps %llu Delat RE %g alpha %.9g walk %.3f ms train %.3f ms (%llu words)\n", r,
                   ri.n_walks, static_cast<unsigned long long>(ri.steps), std::fabs(ri.delta_h), alpha, ri.walk_ms,
                   tr.train_ms, static_cast<unsigned long long>(tr.words));
            if (keep_arg) keep = p; else dg_paths_free(p);
        } else if (r >= o.train_from) {
            const float alpha = lr->get_lr();
            dg_pipeline_info pi{};
            check(dg_pipeline_round(g, s, &wp, static_cast<uint32_t>(r), 0, alpha, &pi, keep_arg), "dg_pipeline_round");
            walk_ms += pi.walk.walk_ms;
            train_ms += pi.train.train_ms;
            device_ms += pi.total_ms;
            steps += pi.walk.steps;
            footprints += pi.walk.footprints;
            words += pi.train.words;
            pairs += pi.train.pairs;
            printf("round %d: walks %u steps %llu Delat RE %g alpha %.9g walk %.3f ms train %.3f ms (%llu words)\n", r,
                   pi.walk.n_walks, static_cast<unsigned long long>(pi.walk.steps), std::fabs(pi.walk.delta_h), alpha,
                   pi.walk.walk_ms, pi.train.train_ms, static_cast<unsigned long long>(pi.train.words));
        } else {
            dg_paths *p = nullptr;
            check(dg_walk_run_round(g, &wp, static_cast<uint32_t>(r), 0, &p), "dg_walk_run_round");
            dg_round_info ri{};
            check(dg_paths_get_info(p, &ri), "dg_paths_get_info");
            walk_ms += ri.walk_ms;
            device_ms += ri.walk_ms;
            steps += ri.steps;
            footprints += ri.footprints;
            printf("round %d: walks %u steps %llu Delat RE %g (not trained) walk %.3f ms\n", r, ri.n_walks,
                   static_cast<unsigned long long>(ri.steps), std::fabs(ri.delta_h), ri.walk_ms);
            if (keep_arg) keep = p; else dg_paths_free(p);
        }
        if (keep) {
            // walk.hpp:686: <prefix>-<rank>-<round>.txt, rank 0 of 1.
            const std::string path = o.walk_prefix + "-0-" + std::to_string(r) + ".txt";
            check(dg_paths_write_text(keep, path.c_str()), "dg_paths_write_text");
            dg_paths_free(keep);
        }
    }
    const double embed_s = seconds_since(t_embed);
    if (!o.emb_output.empty()) check(dg_sgns_write_embedding(s, o.emb_output.c_str()), "dg_sgns_write_embedding");
    const double total_s = seconds_since(t_start);

    printf("walk-steps/s %.6e (walk kernels %.3f ms, %llu steps, %llu footprints)\n", steps / (walk_ms * 1e-3),
           walk_ms, static_cast<unsigned long long>(steps), static_cast<unsigned long long>(footprints));
    if (train_ms > 0)
        printf("SGNS words/s %.6e (train kernels %.3f ms, %llu words, %llu pairs)\n", words / (train_ms * 1e-3),
               train_ms, static_cast<unsigned long long>(words), static_cast<unsigned long long>(pairs));
    printf("embed: device %.3f s, rounds wall %.3f s, end-to-end %.3f s (graph load %.3f s)\n", device_ms * 1e-3,
           embed_s, total_s, load_s);
    dg_sgns_free(s);
    dg_graph_free(g);
    return 0;
}
