/*
 * The reference's own walk random streams, for the pin test only
 * (TEST INFRASTRUCTURE; see dg_oracle.h).  StdRandNumGenerator::gen draws
 * candidates with std::uniform_int_distribution<uint32_t>(0, degree - 1) over a
 * std::mt19937 (include/util.hpp:22-47); the acceptance draw is glibc rand()
 * (include/walk.hpp:928), used here from its default (srand(1)) state.
 */
#include "dg_oracle.h"

#include <cstdlib>
#include <random>

namespace {
struct Stream {
    std::mt19937 mt;
    explicit Stream(uint32_t seed) : mt(seed) {}
};
}  // namespace

extern "C" void *dgo_stream_new(uint32_t seed) {
    srand(1);
    return new Stream(seed);
}

extern "C" void dgo_stream_free(void *s) { delete static_cast<Stream *>(s); }

extern "C" uint32_t dgo_stream_cand(void *s, uint32_t degree) {
    std::uniform_int_distribution<uint32_t> dis(0, degree - 1);
    return dis(static_cast<Stream *>(s)->mt);
}

extern "C" uint32_t dgo_stream_acc(void *) { return (uint32_t)rand(); }
