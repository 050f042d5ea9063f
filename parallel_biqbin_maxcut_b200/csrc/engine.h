// A bounding engine: everything one node's bound needs, so that several
// nodes can be bounded at the same time, each on its own stream.
//
// The default engine is what the drop-in entry points use: the library
// stream, glibc rand(), and the reference's process globals (Cuts, X,
// dual_gamma, ...; re-read on every call because the host program owns and
// may re-point them).  Extra engines own private copies of that host state,
// their own stream and their own random stream (rng.h).
#pragma once
#include <atomic>
#include <vector>

#include "bundle.cuh"
#include "cuts.cuh"
#include "globals.h"
#include "heur.cuh"
#include "kgon_sa.cuh"
#include "rng.h"
#include "trisep.cuh"
#include "warm.h"

namespace bqb {

// Device-resident state of the node being bounded.
struct NodeDev {
    int n = 0;
    DevBuf<double> L;      // PP->L (n x n)
    DevBuf<double> L0;     // L - B^T(gamma) scratch
    DevBuf<double> X;      // the reference's global X (current primal matrix)
    DevBuf<double> out;    // IPM output words
    DevBuf<double> P0L;    // SP->L (N0 x N0)
    int P0N = 0;
    const double* P0L_src = nullptr;
    unsigned P0L_gen = 0;
    DevCuts cuts;
    BundleDev b;
    HostBuf<double> hs;    // pinned scratch for small reads
    HostBuf<int> hi;
};

// The host-side arrays the bound reads and writes (the reference's globals
// src/global_var.h:21-47, or an engine's private copies).
struct HostState {
    Triangle_Inequality* cuts;
    Pentagonal_Inequality* pcuts;
    Pentagonal_Inequality* plist;
    Heptagonal_Inequality* hcuts;
    Heptagonal_Inequality* hlist;
    double* dual_gamma;
    double* X;
    double* f;
};

struct Engine {
    cudaStream_t stream = nullptr;
    bool is_default = false;
    Rng rng;
    NodeDev nd;
    HeurState heur;
    TriSepState tri;
    KgonSaState sa;          // GPU k-gonal separation (extra engines)
    uint64_t sa_seed = 0;    // its chains' seed base ...
    uint64_t sa_calls = 0;   // ... and the separation calls made so far
    DevBuf<double> ipm_ws;
    DevBuf<double> cert_ws, cert_v;   // the bound certificate's factor (n x n) and vectors
    WarmDev warm;            // learned warm start of the bundle multipliers
    // set by a B&B driver before sdp_bound: the parent node's final cuts
    // (null: none); sdp_bound leaves the node's own final cuts in
    // final_cuts when the warm start or the recorder is on
    const ParentCuts* parent = nullptr;
    std::shared_ptr<ParentCuts> final_cuts;
    // private host state (extra engines only)
    std::vector<Triangle_Inequality> cuts_v;
    std::vector<Pentagonal_Inequality> pcuts_v, plist_v;
    std::vector<Heptagonal_Inequality> hcuts_v, hlist_v;
    std::vector<double> dual_v, X_v;
    double f_v = 0.0;
    Problem PP{};
    std::vector<double> PPL;

    HostState host();
    void ensure_private(int N);   // size the private arrays for problems up to N x N
};

// Bumped whenever this library's process_adj_matrix builds a new SP->L, so
// engines re-upload it even when the allocator returns the same address.
extern std::atomic<unsigned> g_sp_generation;

Engine& default_engine();
Engine* engine_create(unsigned seed);
void engine_destroy(Engine* e);

// SDPbound (src/bounding.c:24-342) in engine E.
double sdp_bound(Engine& E, BabNode* node, Problem* SP_, Problem* PP_, int rank);

// Launch the fused submissions still waiting on the host (capi_fused.cu).
void fused_launch_pending();
// Best-first B&B with the open-node pool on the device (capi_fused.cu).
int fused_pool_bab(const std::vector<BabNode>& open, int cap, double budget_s, long long* created,
                   long long* evaluated, int* stopped);

}  // namespace bqb
