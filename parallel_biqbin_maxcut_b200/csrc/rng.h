// Random numbers for the heuristic and the separation.
//
// The reference draws everything from glibc rand() after srand(2020)
// (src/bab_functions.c:82).  The default engine does exactly that, so a
// single-threaded run consumes the reference's stream.  Extra engines (one
// per concurrent node) each own a stream of the same generator: glibc's
// random_r with the default 128-byte state is the algorithm behind rand(),
// so an engine seeded with s produces the sequence srand(s); rand(); ...
#pragma once
#include <stdlib.h>
#include <string.h>

namespace bqb {

struct Rng {
    bool glibc = true;   // true: the process-wide rand()
    struct random_data rd;
    char state[128];

    void seed(unsigned s)
    {
        glibc = false;
        memset(&rd, 0, sizeof rd);
        memset(state, 0, sizeof state);
        initstate_r(s, state, sizeof state, &rd);
        srandom_r(s, &rd);
    }
    int next()
    {
        if (glibc) return rand();
        int32_t r;
        random_r(&rd, &r);
        return (int)r;
    }
};

}  // namespace bqb
