// Cut-list management shared by the drop-in entry points and the device-
// resident bounding driver.
#pragma once
#include "globals.h"
#include "rng.h"
#include "trisep.cuh"

namespace bqb {

// src/cutting_planes.c:144-166: store y into the cuts, drop those with
// y < 1e-5 keeping order; returns the number kept.
int tri_purge(Triangle_Inequality* cuts, int n_ineq, const double* y);
// src/cutting_planes.c:172-206: append the separated cuts not already among
// the first `kept` cuts, in list order, with y = 0, until MaxTriIneqAdded.
// Membership is a hash lookup (the reference scans linearly); the result is
// the same list.  Returns the number added.
int tri_append(Triangle_Inequality* cuts, int kept, const TriCand* list, int list_size);

int pent_purge(Pentagonal_Inequality* cuts, int n_ineq, const double* y);
int pent_append(Pentagonal_Inequality* cuts, int kept, const Pentagonal_Inequality* list, int size);
int hept_purge(Heptagonal_Inequality* cuts, int n_ineq, const double* y);
int hept_append(Heptagonal_Inequality* cuts, int kept, const Heptagonal_Inequality* list, int size);

// Host simulated-annealing separation of pentagonal / heptagonal cuts
// (src/cutting_planes.c:224-309, 416-503), drawing from rng in the
// reference's order (the default engine's rng is rand() itself).  X: host, N x N column-major.  Returns the minimum
// value found.
double pent_separate(const double* Xh, int N, Pentagonal_Inequality* list, int* size, Rng& rng);
double hept_separate(const double* Xh, int N, Heptagonal_Inequality* list, int* size, Rng& rng);

// The same lists from the GPU annealing chains (kgon_sa.cuh): chain c's
// value cost[c] and permutation perm[7c ..] offered in chain order.
double pent_collect(const double* cost, const int* perm, int chains, Pentagonal_Inequality* list, int* size);
double hept_collect(const double* cost, const int* perm, int chains, Heptagonal_Inequality* list, int* size);

TriSepState& trisep_state();

}  // namespace bqb
