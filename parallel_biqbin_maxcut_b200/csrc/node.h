// The device-resident bounding driver (SDPbound) and its pieces.
#pragma once
#include <atomic>

#include "engine.h"

// A host heuristic with runHeuristic_unpacked's contract
// (src/heuristic.c:19): P0_L, P0_N, P_L, P_N, node xfixed, node sol.X, x.
typedef double (*bqb_heuristic_fn)(double*, int, double*, int, int*, int*, int*);

namespace bqb {

extern std::atomic<bqb_heuristic_fn> g_heuristic_hook;
extern std::atomic<long long> g_heuristic_runs;

// bdl_iter iterations of src/bundle.c:47-235 on the engine's device-resident
// bundle; t in/out on the host.  Synchronises once at the end; returns f.
double bundle_iterations(Engine& E, int bdl_iter, double* t);

// Pack the cut lists of H (counts from P) and upload them with their pair
// CSR; resize the bundle's m-vectors.
void upload_cuts(Engine& E, const HostState& H, const Problem* P);

// updateTriangleInequalities (src/cutting_planes.c:132-214) with the
// separation run on the engine's device-resident X.
double tri_update_dev(Engine& E, HostState& H, Problem* P, const double* y, int* added, int* subtracted);

// update{Pentagonal,Heptagonal}Inequalities (src/cutting_planes.c:316-406,
// 509-602) on host state H with random stream rng; H.X holds X.
double pent_update(HostState& H, Problem* P, const double* y, int* added, int* subtracted, int triag, Rng& rng);
// The same updates with the separation run by the GPU annealing chains on
// the engine's device X (extra engines).
double pent_update_dev(Engine& E, HostState& H, Problem* P, const double* y, int* added, int* subtracted,
                       int triag);
double hept_update_dev(Engine& E, HostState& H, Problem* P, const double* y, int* added, int* subtracted,
                       int hept_index);
double hept_update(HostState& H, Problem* P, const double* y, int* added, int* subtracted, int hept_index,
                   Rng& rng);

}  // namespace bqb
