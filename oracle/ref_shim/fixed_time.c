/* Stand-in for the C library's time(), loaded with LD_PRELOAD in front of the
 * reference's gtrain tool: it returns the value of DG_FIXED_TIME (0 when unset),
 * so that the tool's srand(time(0)) (src/tools/gtrain.cpp:302, 391) replays a
 * chosen seed and its split can be compared with the library's.  TEST
 * INFRASTRUCTURE ONLY. */
#include <stdlib.h>
#include <time.h>

time_t time(time_t *t) {
    const char *s = getenv("DG_FIXED_TIME");
    const time_t v = s ? (time_t)strtoll(s, NULL, 10) : (time_t)0;
    if (t) *t = v;
    return v;
}
