/*
 * Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel
 * random numbers: as easy as 1, 2, 3", SC'11), restated for the CPU checker.
 * Test infrastructure only.
 *
 * The reference draws its walk randomness from per-thread mt19937 streams
 * seeded by std::random_device (include/util.hpp:22-47) and glibc rand()
 * (include/walk.hpp:928), so it cannot be replayed.  Seeded replay is defined
 * instead by one Philox block per transition attempt:
 *
 *   key     = (seed low 32 bits, seed high 32 bits)
 *   counter = (attempt index within the walk, walker id, round, DGO_WALK_TAG)
 *   x0..x3  = Philox4x32-10(counter, key)
 *   candidate slot = high 64 bits of ((x1:x0) * degree)       (replaces gen->gen(degree), walk.hpp:899)
 *   acceptance k   = x2 & 0x7fffffff, p = k / 2147483647.0    (replaces rand()/RAND_MAX, walk.hpp:928)
 */
#ifndef DGO_PHILOX_H
#define DGO_PHILOX_H

#include <stdint.h>

#define DGO_PHILOX_M0 0xD2511F53u
#define DGO_PHILOX_M1 0xCD9E8D57u
#define DGO_PHILOX_W0 0x9E3779B9u
#define DGO_PHILOX_W1 0xBB67AE85u
#define DGO_WALK_TAG 0x57414C4Bu /* "WALK" */

typedef struct { uint32_t v[4]; } dgo_u32x4;

static inline dgo_u32x4 dgo_philox4x32_10(dgo_u32x4 ctr, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += DGO_PHILOX_W0; k1 += DGO_PHILOX_W1; }
        uint64_t p0 = (uint64_t)DGO_PHILOX_M0 * ctr.v[0];
        uint64_t p1 = (uint64_t)DGO_PHILOX_M1 * ctr.v[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        dgo_u32x4 n;
        n.v[0] = hi1 ^ ctr.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ ctr.v[3] ^ k1;
        n.v[3] = lo0;
        ctr = n;
    }
    return ctr;
}

/* floor(x * n / 2^64) for a 64-bit uniform x: unbiased to within n / 2^64. */
static inline uint32_t dgo_scale64(uint64_t x, uint32_t n) {
    return (uint32_t)(((unsigned __int128)x * n) >> 64);
}

#endif
