// gcn: common-neighbour counts of every edge, the reference's src/tools/gcn.cpp
// job over the distger C ABI (the counts are computed on the GPU by
// dg_common_neighbours).
//
// Flags kept from the tool (GcnOptionHelper, gcn.cpp:17-62):
//   -i <edges.txt>  -o <out.txt>  -v <vertices>  -t <threads: accepted, unused>
//   -s weighted|unweighted  [--make-undirected]
// Input is read as the tool reads it (gcn.cpp:93-103): "%u %u" pairs by fscanf
// until one fails -- the tool always reads the unweighted form, whatever -s
// says.  Output: "%u %u %d\n" per input edge, input order (gcn.cpp:357-366).
// Added: -b <edges.bin> also writes the 12-byte {u32 src, u32 dst, f32 cn}
// records that the reference's gconverter -s weighted would make of the output
// (gconverter.cpp:56-74), ready for dg_graph_create / huge_walk; -device d.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "distger.h"

namespace {

[[noreturn]] void die(const char *what) {
    fprintf(stderr, "gcn: %s\n", what);
    exit(2);
}

}  // namespace

int main(int argc, char **argv) {
    std::string in, out, bin, stat;
    uint32_t v_num = 0;
    bool undirected = false, have_t = false;
    int device = 0;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto val = [&]() -> const char * {
            if (i + 1 >= argc) die(("missing value for " + a).c_str());
            return argv[++i];
        };
        if (a == "-i" || a == "--input") in = val();
        else if (a == "-o" || a == "--output") out = val();
        else if (a == "-v" || a == "--vertex") v_num = static_cast<uint32_t>(strtoul(val(), nullptr, 10));
        else if (a == "-t" || a == "--thread") { val(); have_t = true; }
        else if (a == "-s" || a == "--static") stat = val();
        else if (a == "--make-undirected") undirected = true;
        else if (a == "-b") bin = val();
        else if (a == "-device") device = atoi(val());
        else die(("unknown flag " + a).c_str());
    }
    // gcn.cpp:42-61 asserts every one of these.
    if (in.empty() || out.empty() || v_num == 0 || !have_t || (stat != "weighted" && stat != "unweighted"))
        die("usage: gcn -i edges.txt -o out.txt -v V -t T -s weighted|unweighted [--make-undirected] [-b edges.bin]");
    FILE *f = fopen(in.c_str(), "r");
    if (!f) die(("cannot open " + in).c_str());
    std::vector<uint32_t> src, dst;
    unsigned s, d;
    while (2 == fscanf(f, "%u %u", &s, &d)) {
        src.push_back(s);
        dst.push_back(d);
    }
    fclose(f);
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<int32_t> cn(src.size());
    if (dg_common_neighbours(src.data(), dst.data(), src.size(), v_num, undirected ? 1 : 0, device, cn.data()) !=
        DG_OK) {
        fprintf(stderr, "gcn: %s\n", dg_last_error());
        return 1;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    FILE *o = fopen(out.c_str(), "w");
    if (!o) die(("cannot open " + out).c_str());
    for (size_t e = 0; e < src.size(); e++) fprintf(o, "%u %u %d\n", src[e], dst[e], cn[e]);
    fclose(o);
    if (!bin.empty()) {
        FILE *b = fopen(bin.c_str(), "wb");
        if (!b) die(("cannot open " + bin).c_str());
        for (size_t e = 0; e < src.size(); e++) {
            const float w = static_cast<float>(cn[e]);
            fwrite(&src[e], 4, 1, b);
            fwrite(&dst[e], 4, 1, b);
            fwrite(&w, 4, 1, b);
        }
        fclose(b);
    }
    printf("%zu common neighbours are calculated\n[get cn] time: %f \n", src.size(), secs);
    return 0;
}
