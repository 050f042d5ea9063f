// Host-side pentagonal / heptagonal separation by simulated annealing
// (src/qap_simulated_annealing.c, src/cutting_planes.c:224-309, 416-503).
//
// This file is compiled with the reference's floating-point flags
// (-O3 -ffast-math, reference Makefile:17): the annealing's accept/reject
// decisions depend on sums the compiler reassociates under those flags, and
// the same flags make this restatement take the reference's decisions, so
// the separated cuts and the rand() stream after the call are the
// reference's for the same X.
#include <math.h>
#include <stdlib.h>

#include <vector>

#include "globals.h"
#include "rng.h"

namespace bqb {

// declared for the other translation units in separation.h
double pent_separate(const double* Xh, int N, Pentagonal_Inequality* list, int* size, Rng& rng);
double hept_separate(const double* Xh, int N, Heptagonal_Inequality* list, int* size, Rng& rng);
double pent_collect(const double* cost, const int* perm, int chains, Pentagonal_Inequality* list, int* size);
double hept_collect(const double* cost, const int* perm, int chains, Heptagonal_Inequality* list, int* size);

namespace {
constexpr double BIG_NUMBER = 1e9;   // src/biqbin.h:35
}
// k x k matrix H = e e^T for the sign vector of (kind, type); the tables of
// src/cutting_planes.c:239-244 (k = 5) and :431-438 (k = 7) are exactly these.
static void kgon_H(int k, int type, int* H)
{
    int e[7];
    for (int a = 0; a < k; ++a) e[a] = (a < type - 1) ? -1 : 1;
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) H[b + a * k] = e[a] * e[b];
}

}  // namespace bqb

using namespace bqb;

// Simulated annealing for min over permutations P of <(P X P^T)(1:k,1:k), H>
// (src/qap_simulated_annealing.c:12-190): temperature t = k^2 sum|X| /
// (n(n-1)), n inner steps at the start, t *= 0.6 and steps *= 1.1 per round,
// random transposition (i1 < k, i2 < n), Metropolis acceptance with
// exp(-delta/t) unless delta/t > 5; stops after a round with no accepted
// move of size > 0.001.  Random numbers are drawn in the reference's order.
namespace bqb {
double qap_sa(const int* H, int k, const double* Xm, int n, int* ineq, Rng& rng)
{
    // fewer than k vertices: no k-gonal inequality exists (the reference
    // reads past its permutation there); nothing is drawn or written
    if (n < k) return BIG_NUMBER;
    const int inner_iter = n;
    const double reduce_temp = 0.6;
    const double increase_iter = 1.1;
    double t = k * k;
    double sumX = n;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) sumX += 2 * fabs(Xm[j + i * n]);
    t *= sumX;
    t /= (n * (n - 1));
    double cost = BIG_NUMBER;
    std::vector<int> perm(n), best(n, 0);
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = n - 1; i > 0; --i) {
        const int r = rng.next() % i;
        const int tmp = perm[i];
        perm[i] = perm[r];
        perm[r] = tmp;
    }
    double t1 = t;
    int m1 = inner_iter;
    double sol = k;
    for (int i = 0; i < k; ++i)
        for (int j = i + 1; j < k; ++j) sol += 2 * H[j + i * k] * Xm[perm[j] + perm[i] * n];
    int not_done = 1;
    while (not_done > 0) {
        not_done = 0;
        for (int it = 0; it < m1; ++it) {
            int i1 = rng.next() % k;
            int i2 = rng.next() % n;
            if (i2 < i1) {
                const int tmp = i1;
                i1 = i2;
                i2 = tmp;
            }
            double delta = 0.0;
            for (int i = 0; i < k; ++i)
                delta += H[i + k * i1] * (Xm[perm[i] + n * perm[i2]] - Xm[perm[i] + n * perm[i1]]);
            if (i2 < k)
                for (int i = 0; i < k; ++i)
                    delta += H[i + k * i2] * (Xm[perm[i] + n * perm[i1]] - Xm[perm[i] + n * perm[i2]]);
            delta *= 2.0;
            const double tv1 = 2.0 - 2.0 * Xm[perm[i2] + n * perm[i1]];
            double tv2 = 1.0;
            if (i2 < k) tv2 += -2 * H[i1 + k * i2] + 1.0;
            delta += tv1 * tv2;
            const double sol_temp = sol + delta;
            int accept;
            if (delta > 0) {
                const double dt1 = delta / t1;
                if (dt1 > 5)
                    accept = 0;
                else
                    accept = ((double)rng.next() / ((double)RAND_MAX)) < exp(-dt1) ? 1 : 0;
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
                    best = perm;
                }
            }
        }
        t1 *= reduce_temp;
        m1 = (int)round(m1 * increase_iter);
    }
    for (int i = 0; i < k; ++i) ineq[i] = best[i];
    return cost;
}
}  // namespace bqb

BQB_API double qap_simulated_annealing(int* H, int k, double* Xm, int n, int* ineq)
{
    Rng glibc;
    return qap_sa(H, k, Xm, n, ineq, glibc);
}


namespace bqb {

// Streaming list of src/cutting_planes.c:247-304 (pentagonal) and :441-498
// (heptagonal), restated with its exact update rule, including the
// re-scan that starts from BIG_NUMBER and looks for a larger value.
template <int K, class Ineq>
struct KgonList {
    Ineq* list;
    int cap;
    int size = 0, least = 0;
    double least_val = -BIG_NUMBER;
    double min_all = BIG_NUMBER;
    KgonList(Ineq* l, int c) : list(l), cap(c) {}
    void offer(int type, double v, const int* perm)
    {
        min_all = v < min_all ? v : min_all;
        if (!(v < 1.0)) return;
        if (size < cap) {
            list[size].type = type;
            list[size].value = v;
            for (int a = 0; a < K; ++a) list[size].permutation[a] = perm[a];
            if (size == 0 || v > least_val) {
                least_val = v;
                least = size;
            }
            ++size;
        } else if (v < least_val) {
            list[least].type = type;
            list[least].value = v;
            for (int a = 0; a < K; ++a) list[least].permutation[a] = perm[a];
            least_val = BIG_NUMBER;
            for (int q = 0; q < size; ++q)
                if (list[q].value > least_val) {
                    least_val = list[q].value;
                    least = q;
                }
        }
    }
};

template <int K, class Ineq>
static double kgon_separate(const double* Xh, int N, Ineq* list, int* list_size, int trials, int types,
                            int cap, Rng& rng)
{
    KgonList<K, Ineq> L(list, cap);
    int H[49];
    int perm[7];
    for (int trial = 0; trial < trials; ++trial) {
        for (int type = 1; type <= types; ++type) {
            kgon_H(K, type, H);
            const double v = qap_sa(H, K, Xh, N, perm, rng);
            L.offer(type, v, perm);
        }
    }
    *list_size = L.size;
    return L.min_all;
}

// Chain results of the GPU annealing (chain c = (trial, type) pair
// c / types, c % types + 1) offered to the list in the reference's loop order.
template <int K, class Ineq>
static double kgon_collect(const double* cost, const int* perm, int chains, int types, Ineq* list,
                           int* list_size, int cap)
{
    KgonList<K, Ineq> L(list, cap);
    for (int c = 0; c < chains; ++c) L.offer(c % types + 1, cost[c], perm + (size_t)7 * c);
    *list_size = L.size;
    return L.min_all;
}

double pent_collect(const double* cost, const int* perm, int chains, Pentagonal_Inequality* list, int* size)
{
    return kgon_collect<5>(cost, perm, chains, 3, list, size, params.PentIneq);
}

double hept_collect(const double* cost, const int* perm, int chains, Heptagonal_Inequality* list, int* size)
{
    return kgon_collect<7>(cost, perm, chains, 4, list, size, params.HeptaIneq);
}

double pent_separate(const double* Xh, int N, Pentagonal_Inequality* list, int* size, Rng& rng)
{
    return kgon_separate<5>(Xh, N, list, size, params.Pent_Trials, 3, params.PentIneq, rng);
}

double hept_separate(const double* Xh, int N, Heptagonal_Inequality* list, int* size, Rng& rng)
{
    return kgon_separate<7>(Xh, N, list, size, params.Hepta_Trials, 4, params.HeptaIneq, rng);
}

}  // namespace bqb

