/* Oracle (test infrastructure only): the k-gonal annealing chains of the
 * GPU separation, restated sequentially in plain C.
 *
 * One chain is the reference's qap_simulated_annealing
 * (src/qap_simulated_annealing.c:12-160) with its random numbers drawn from
 * the chain's own SplitMix64 stream instead of rand():
 *   - starting temperature k^2 (n + sum_{i<j} 2|X_ij|) / (n (n-1)), summed
 *     in the reference's loop order (:20-32),
 *   - random starting permutation by backward transpositions (:37-44),
 *   - starting value k + sum_{i<j} 2 H_ij X[p_i, p_j] (:54-57),
 *   - rounds of m1 transposition moves (i1 < k, i2 < n, swapped so that
 *     i1 <= i2), the move's cost change (:83-101), Metropolis acceptance
 *     unless delta / t > 5 (:103-115), best permutation kept (:117-143),
 *   - t *= 0.6, m1 = round(1.1 m1) per round, stop after a round without an
 *     accepted move of size > 0.001 (:61-66, :146-149).
 * The GPU kernel caps the rounds at max_rounds; so does this restatement.
 *
 * Compiled without -ffast-math: every sum is taken in the order written.
 *
 * Pinned against the reference: oracle_qap_sa_glibc draws from rand()
 * instead, and the same source built with the reference's flags
 * (-O3 -ffast-math, _port/libbqb_oracle_c_fm.so) returns the reference
 * build's qap_simulated_annealing value, permutation and rand() state.
 * Chain c of a call anneals type (c % types) + 1 with H = e e^T,
 * e_a = -1 for a < type - 1 (src/cutting_planes.c:239-244, 431-438), from
 * state seed + (c + 1) * 0xD1B54A32D192ED03. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#define ORACLE_RAND_MAX 2147483647

static uint32_t next31(uint64_t *state, int glibc)
{
    if (glibc) return (uint32_t)rand();
    uint64_t z = (*state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (uint32_t)(z >> 33);
}

/* One chain; returns its best value, best[0..k-1] its permutation head;
 * *capped = 1 if max_rounds ended it. */
static double chain(const double *X, int n, int k, int type, uint64_t state, int glibc, int max_rounds,
                    int *best, int *capped)
{
    int e[7];
    for (int a = 0; a < k; ++a) e[a] = (a < type - 1) ? -1 : 1;
    double sumX = n;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) sumX += 2.0 * fabs(X[j + (size_t)i * n]);
    double t = (double)(k * k);
    t *= sumX;
    t /= (double)(n * (n - 1));

    int *perm = (int *)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = n - 1; i > 0; --i) {
        const int r = (int)(next31(&state, glibc) % (uint32_t)i);
        const int tmp = perm[i];
        perm[i] = perm[r];
        perm[r] = tmp;
    }
    double t1 = t;
    int m1 = n;
    double sol = k;
    for (int i = 0; i < k; ++i)
        for (int j = i + 1; j < k; ++j) sol += (double)(2 * e[j] * e[i]) * X[perm[j] + (size_t)perm[i] * n];
    double cost = 1e9;
    for (int a = 0; a < k; ++a) best[a] = 0;
    int not_done = 1, round_ = 0;
    while (not_done > 0 && round_ < max_rounds) {
        not_done = 0;
        for (int it = 0; it < m1; ++it) {
            int i1 = (int)(next31(&state, glibc) % (uint32_t)k);
            int i2 = (int)(next31(&state, glibc) % (uint32_t)n);
            if (i2 < i1) {
                const int tmp = i1;
                i1 = i2;
                i2 = tmp;
            }
            double delta = 0.0;
            for (int i = 0; i < k; ++i)
                delta += (double)(e[i] * e[i1]) * (X[perm[i] + (size_t)n * perm[i2]] - X[perm[i] + (size_t)n * perm[i1]]);
            if (i2 < k)
                for (int i = 0; i < k; ++i)
                    delta += (double)(e[i] * e[i2]) *
                             (X[perm[i] + (size_t)n * perm[i1]] - X[perm[i] + (size_t)n * perm[i2]]);
            delta *= 2.0;
            const double tv1 = 2.0 - 2.0 * X[perm[i2] + (size_t)n * perm[i1]];
            double tv2 = 1.0;
            if (i2 < k) tv2 += (double)(-2 * e[i1] * e[i2]) + 1.0;
            delta += tv1 * tv2;
            const double sol_temp = sol + delta;
            int accept;
            if (delta > 0) {
                const double dt1 = delta / t1;
                if (dt1 > 5)
                    accept = 0;
                else
                    accept = ((double)next31(&state, glibc) / (double)ORACLE_RAND_MAX) < exp(-dt1) ? 1 : 0;
            } else {
                accept = 1;
            }
            if (accept) {
                if (fabs(delta) > 0.001) not_done = 1;
                const int tmp = perm[i1];
                perm[i1] = perm[i2];
                perm[i2] = tmp;
                sol = sol_temp;
                if (sol < cost) {
                    cost = sol;
                    for (int a = 0; a < k; ++a) best[a] = perm[a];
                }
            }
        }
        t1 *= 0.6;
        m1 = (int)round(m1 * 1.1);
        ++round_;
    }
    *capped = not_done > 0;
    free(perm);
    return cost;
}

/* All chains of one separation call: cost[c], perm[7c .. 7c+k-1]; returns
 * 1 if any chain hit max_rounds. */
int oracle_kgon_sa(const double *X, int n, int k, int types, int chains, unsigned long long seed, int max_rounds,
                   double *cost, int *perm)
{
    int any = 0;
    for (int c = 0; c < chains; ++c) {
        int capped = 0;
        int best[7] = {0, 0, 0, 0, 0, 0, 0};
        const uint64_t st = (uint64_t)seed + (uint64_t)(c + 1) * 0xD1B54A32D192ED03ull;
        cost[c] = chain(X, n, k, c % types + 1, st, 0, max_rounds, best, &capped);
        for (int a = 0; a < 7; ++a) perm[(size_t)c * 7 + a] = a < k ? best[a] : 0;
        any |= capped;
    }
    return any;
}

/* One chain of type `type` drawing from rand() (seed it with srand), with
 * no round limit: the reference's qap_simulated_annealing for H = e e^T. */
double oracle_qap_sa_glibc(const double *X, int n, int k, int type, int *ineq)
{
    int capped = 0;
    return chain(X, n, k, type, 0, 1, 1 << 30, ineq, &capped);
}
