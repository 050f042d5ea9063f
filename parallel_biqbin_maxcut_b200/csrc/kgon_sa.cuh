// Pentagonal / heptagonal separation by simulated annealing on the GPU.
//
// The reference separates k-gonal inequalities (k = 5, 7) by running
// qap_simulated_annealing (src/qap_simulated_annealing.c:12-190) once per
// (trial, type) pair, one after another, all drawing from the process's
// rand() stream (src/cutting_planes.c:224-309, 416-503).  Here every
// (trial, type) pair is an independent annealing chain: one GPU thread runs
// one chain with the reference's schedule, move set, acceptance rule and
// stopping rule, drawing from its own counter-seeded SplitMix64 stream
// (Steele, Lea and Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014) in the reference's order of draws.  The chains' results are
// then merged into the cut list on the host in (trial, type) order with the
// reference's list rule, so only the random numbers differ from the
// reference's separation.
#pragma once
#include <math.h>
#include <stdint.h>

#include "bqb_common.cuh"

namespace bqb {

constexpr int SA_CHAINS_PER_CTA = 64;
// Rounds after which a chain is stopped even if it still moves (the
// reference has no limit).  Chains on IPM matrices of G(n, 0.5) instances,
// n = 30..128, end within 20-25 rounds (the temperature falls by 0.6 per
// round); 80 rounds bound a chain to n (1.1^80 - 1) / 0.1 < 20500 n moves
// and keep the round length m1 = n 1.1^r far inside int range.  A chain
// stopped here sets status[0].
constexpr int SA_MAX_ROUNDS = 80;
constexpr int SA_RAND_MAX = 2147483647;

// Chain c's random stream: state0 = seed + (c + 1) * SA_CHAIN_STRIDE,
// outputs SplitMix64(state) >> 33 (31-bit values, like rand()).
constexpr uint64_t SA_CHAIN_STRIDE = 0xD1B54A32D192ED03ull;

struct KgonSaState {
    DevBuf<double> cost;    // chains
    DevBuf<int> perm;       // chains x 7
    DevBuf<int> status;     // [0] round limit reached
    HostBuf<double> hcost;
    HostBuf<int> hperm;
    HostBuf<int> hstat;
};

__device__ __forceinline__ uint32_t sa_next(uint64_t& state)
{
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (uint32_t)(z >> 33);
}

// Starting temperature k^2 (n + sum_{i<j} 2|X_ij|) / (n (n-1)), summed by
// the calling thread in the reference's loop order.
__device__ inline double kgon_temperature(const double* Xs, int n, int K)
{
    double sumX = n;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) sumX = __dadd_rn(sumX, __dmul_rn(2.0, fabs(Xs[j + (size_t)i * n])));
    double t = (double)(K * K);
    t = __dmul_rn(t, sumX);
    return __ddiv_rn(t, (double)(n * (n - 1)));
}

// One annealing chain (chain index c, type (c % types) + 1) run by the
// calling thread.  Its permutation lives at P[i * pstride + lane].
// Writes cost_out[c], perm_out[7c .. 7c+6]; sets *status on the round limit.
__device__ inline void kgon_chain(const double* __restrict__ Xs, int n, int K, int types, int c,
                                  unsigned long long seed, double t0, unsigned short* P, int pstride, int lane,
                                  double* __restrict__ cost_out, int* __restrict__ perm_out, int* status)
{
    const int type = c % types + 1;
    // H(a, b) = e_a e_b with e_a = -1 for a < type - 1, else +1
    auto e = [&](int a) { return a < type - 1 ? -1 : 1; };
    auto PA = [&](int i) -> unsigned short& { return P[(size_t)i * pstride + lane]; };
    auto XA = [&](int a, int b) { return Xs[a + (size_t)n * b]; };

    uint64_t rs = seed + (uint64_t)(c + 1) * SA_CHAIN_STRIDE;
    for (int i = 0; i < n; ++i) PA(i) = (unsigned short)i;
    for (int i = n - 1; i > 0; --i) {
        const int r = (int)(sa_next(rs) % (uint32_t)i);
        const unsigned short tmp = PA(i);
        PA(i) = PA(r);
        PA(r) = tmp;
    }
    double t1 = t0;
    int m1 = n;
    double sol = K;
    for (int i = 0; i < K; ++i)
        for (int j = i + 1; j < K; ++j)
            sol = __dadd_rn(sol, __dmul_rn((double)(2 * e(j) * e(i)), XA(PA(j), PA(i))));
    double cost = 1e9;
    int best[7] = {0, 0, 0, 0, 0, 0, 0};
    int not_done = 1, rounds = 0;
    while (not_done > 0 && rounds < SA_MAX_ROUNDS) {
        not_done = 0;
        for (int it = 0; it < m1; ++it) {
            int i1 = (int)(sa_next(rs) % (uint32_t)K);
            int i2 = (int)(sa_next(rs) % (uint32_t)n);
            if (i2 < i1) {
                const int tmp = i1;
                i1 = i2;
                i2 = tmp;
            }
            const int p1 = PA(i1), p2 = PA(i2);
            double delta = 0.0;
            for (int i = 0; i < K; ++i) {
                const int pi = PA(i);
                const double d = __dsub_rn(XA(pi, p2), XA(pi, p1));
                delta = __dadd_rn(delta, e(i) * e(i1) > 0 ? d : -d);
            }
            if (i2 < K)
                for (int i = 0; i < K; ++i) {
                    const int pi = PA(i);
                    const double d = __dsub_rn(XA(pi, p1), XA(pi, p2));
                    delta = __dadd_rn(delta, e(i) * e(i2) > 0 ? d : -d);
                }
            delta = __dmul_rn(delta, 2.0);
            const double tv1 = __dsub_rn(2.0, __dmul_rn(2.0, XA(p2, p1)));
            double tv2 = 1.0;
            if (i2 < K) tv2 = __dadd_rn(tv2, __dadd_rn((double)(-2 * e(i1) * e(i2)), 1.0));
            delta = __dadd_rn(delta, __dmul_rn(tv1, tv2));
            const double sol_temp = __dadd_rn(sol, delta);
            int accept;
            if (delta > 0) {
                const double dt1 = __ddiv_rn(delta, t1);
                if (dt1 > 5)
                    accept = 0;
                else
                    accept = __ddiv_rn((double)sa_next(rs), (double)SA_RAND_MAX) < exp(-dt1) ? 1 : 0;
            } else {
                accept = 1;
            }
            if (accept) {
                if (fabs(delta) > 0.001) not_done = 1;
                PA(i1) = (unsigned short)p2;
                PA(i2) = (unsigned short)p1;
                sol = sol_temp;
                if (sol < cost) {
                    cost = sol;
#pragma unroll
                    for (int a = 0; a < 7; ++a)
                        if (a < K) best[a] = PA(a);
                }
            }
        }
        t1 = __dmul_rn(t1, 0.6);
        m1 = (int)round(__dmul_rn((double)m1, 1.1));
        ++rounds;
    }
    if (not_done > 0) atomicOr(status, 1);
    cost_out[c] = cost;
#pragma unroll
    for (int a = 0; a < 7; ++a) perm_out[(size_t)c * 7 + a] = a < K ? best[a] : 0;
}

// Draw j (0-based) of the stream that starts at state s0: sa_next adds the
// increment before mixing, so the state of draw j is s0 + (j + 1) gamma.
__device__ __forceinline__ uint32_t sa_draw(uint64_t s0, long long j)
{
    uint64_t st = s0 + (uint64_t)j * 0x9E3779B97F4A7C15ull;
    return sa_next(st);
}

// kgon_chain run by a whole warp, with the same result (cost, best
// permutation, stream position) as the one-thread form above.  A move
// draws i1 and i2, and a third number only when it goes uphill by at most
// 5 t; a rejected move changes nothing.  So, from stream position pos, lane
// q evaluates the move that would start at draw pos + q against the current
// permutation (its draws come straight from the counter-based stream), and
// the warp then follows the moves in order (the next one starts 2 or 3
// draws later) up to the first accepted one, which every lane applies; the
// next window starts after it.  Moves before it in the window were rejected,
// so they saw the same permutation as in the one-thread form, and every
// move's arithmetic is that form's.  P: this warp's permutation (n entries
// in shared memory).
__device__ inline void kgon_chain_warp(const double* __restrict__ Xs, int n, int K, int types, int c,
                                       unsigned long long seed, double t0, unsigned short* P,
                                       double* __restrict__ cost_out, int* __restrict__ perm_out, int* status)
{
    const int lane = threadIdx.x & 31;
    const int type = c % types + 1;
    auto e = [&](int a) { return a < type - 1 ? -1 : 1; };
    auto XA = [&](int a, int b) { return Xs[a + (size_t)n * b]; };
    const uint64_t s0 = seed + (uint64_t)(c + 1) * SA_CHAIN_STRIDE;

    double sol = K;
    if (lane == 0) {
        uint64_t rs = s0;
        for (int i = 0; i < n; ++i) P[i] = (unsigned short)i;
        for (int i = n - 1; i > 0; --i) {
            const int r = (int)(sa_next(rs) % (uint32_t)i);
            const unsigned short tmp = P[i];
            P[i] = P[r];
            P[r] = tmp;
        }
        for (int i = 0; i < K; ++i)
            for (int j = i + 1; j < K; ++j)
                sol = __dadd_rn(sol, __dmul_rn((double)(2 * e(j) * e(i)), XA(P[j], P[i])));
    }
    sol = __shfl_sync(0xffffffffu, sol, 0);
    __syncwarp();
    long long pos = n - 1;   // draws used by the shuffle
    double t1 = t0;
    int m1 = n;
    double cost = 1e9;
    int best[7] = {0, 0, 0, 0, 0, 0, 0};
    int not_done = 1, rounds = 0;
    while (not_done > 0 && rounds < SA_MAX_ROUNDS) {
        not_done = 0;
        int it = 0;
        while (it < m1) {
            // the move that would start at draw pos + lane
            const long long q = pos + lane;
            int i1 = (int)(sa_draw(s0, q) % (uint32_t)K);
            int i2 = (int)(sa_draw(s0, q + 1) % (uint32_t)n);
            if (i2 < i1) {
                const int tmp = i1;
                i1 = i2;
                i2 = tmp;
            }
            const int p1 = P[i1], p2 = P[i2];
            double delta = 0.0;
            for (int i = 0; i < K; ++i) {
                const int pi = P[i];
                const double d = __dsub_rn(XA(pi, p2), XA(pi, p1));
                delta = __dadd_rn(delta, e(i) * e(i1) > 0 ? d : -d);
            }
            if (i2 < K)
                for (int i = 0; i < K; ++i) {
                    const int pi = P[i];
                    const double d = __dsub_rn(XA(pi, p1), XA(pi, p2));
                    delta = __dadd_rn(delta, e(i) * e(i2) > 0 ? d : -d);
                }
            delta = __dmul_rn(delta, 2.0);
            const double tv1 = __dsub_rn(2.0, __dmul_rn(2.0, XA(p2, p1)));
            double tv2 = 1.0;
            if (i2 < K) tv2 = __dadd_rn(tv2, __dadd_rn((double)(-2 * e(i1) * e(i2)), 1.0));
            delta = __dadd_rn(delta, __dmul_rn(tv1, tv2));
            int accept, draws = 2;
            if (delta > 0) {
                const double dt1 = __ddiv_rn(delta, t1);
                if (dt1 > 5) {
                    accept = 0;
                } else {
                    draws = 3;
                    accept = __ddiv_rn((double)sa_draw(s0, q + 2), (double)SA_RAND_MAX) < exp(-dt1) ? 1 : 0;
                }
            } else {
                accept = 1;
            }
            const int packed = draws | (accept << 2);
            // follow the moves in order from offset 0
            int off = 0, hit = -1;
            while (off < 32 && it < m1) {
                const int v = __shfl_sync(0xffffffffu, packed, off);
                ++it;
                if (v >> 2) {
                    hit = off;
                    break;
                }
                off += v & 3;
            }
            if (hit < 0) {
                pos += off;   // window used up (or the round ended): nothing moved
                continue;
            }
            const double dh = __shfl_sync(0xffffffffu, delta, hit);
            const int a1 = __shfl_sync(0xffffffffu, i1, hit), a2 = __shfl_sync(0xffffffffu, i2, hit);
            const int q1 = __shfl_sync(0xffffffffu, p1, hit), q2 = __shfl_sync(0xffffffffu, p2, hit);
            const int dr = __shfl_sync(0xffffffffu, packed, hit) & 3;
            pos += hit + dr;
            if (fabs(dh) > 0.001) not_done = 1;
            __syncwarp();
            if (lane == 0) {
                P[a1] = (unsigned short)q2;
                P[a2] = (unsigned short)q1;
            }
            __syncwarp();
            sol = __dadd_rn(sol, dh);
            if (sol < cost) {
                cost = sol;
#pragma unroll
                for (int a = 0; a < 7; ++a)
                    if (a < K) best[a] = P[a];
            }
            __syncwarp();
        }
        t1 = __dmul_rn(t1, 0.6);
        m1 = (int)round(__dmul_rn((double)m1, 1.1));
        ++rounds;
    }
    if (lane == 0) {
        if (not_done > 0) atomicOr(status, 1);
        cost_out[c] = cost;
#pragma unroll
        for (int a = 0; a < 7; ++a) perm_out[(size_t)c * 7 + a] = a < K ? best[a] : 0;
    }
}

// Run `chains` chains of the k-gonal annealing on the n x n matrix dX
// (device, column-major).  Chain c anneals type (c % types) + 1, i.e. the
// chains are the reference's (trial, type) loop flattened.  Results (host,
// valid after the call): st.hcost[c], st.hperm[7c .. 7c+k-1], st.hstat[0].
void kgon_sa_device(KgonSaState& st, const double* dX, int n, int k, int types, int chains, uint64_t seed,
                    cudaStream_t s);

}  // namespace bqb
