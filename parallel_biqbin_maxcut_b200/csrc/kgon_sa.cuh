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

// Run `chains` chains of the k-gonal annealing on the n x n matrix dX
// (device, column-major).  Chain c anneals type (c % types) + 1, i.e. the
// chains are the reference's (trial, type) loop flattened.  Results (host,
// valid after the call): st.hcost[c], st.hperm[7c .. 7c+k-1], st.hstat[0].
void kgon_sa_device(KgonSaState& st, const double* dX, int n, int k, int types, int chains, uint64_t seed,
                    cudaStream_t s);

}  // namespace bqb
