// Separation entry points: triangle separation on the GPU (trisep.cu) with
// host cut-list management; the pentagonal / heptagonal separation by
// simulated annealing runs on the host (host_sep.cpp).
#include <math.h>
#include <string.h>

#include <array>
#include <unordered_set>
#include <vector>

#include "engine.h"
#include "node.h"
#include "separation.h"

namespace bqb {

namespace {
constexpr double BIG_NUMBER = 1e9;   // src/biqbin.h:35

struct Key8Hash {
    size_t operator()(const std::array<int, 8>& a) const
    {
        uint64_t h = 1469598103934665603ull;
        for (int v : a) h = (h ^ (uint64_t)(uint32_t)v) * 1099511628211ull;
        return (size_t)h;
    }
};
}  // namespace

TriSepState& trisep_state() { return default_engine().tri; }

int tri_purge(Triangle_Inequality* cuts, int n_ineq, const double* y)
{
    int next = 0;
    for (int c = 0; c < n_ineq; ++c) {
        cuts[c].y = y[c];
        if (cuts[c].y < 1e-5) continue;
        cuts[next].type = cuts[c].type;
        cuts[next].i = cuts[c].i;
        cuts[next].j = cuts[c].j;
        cuts[next].k = cuts[c].k;
        cuts[next].y = cuts[c].y;
        ++next;
    }
    return next;
}

int tri_append(Triangle_Inequality* cuts, int kept, const TriCand* list, int list_size)
{
    std::unordered_set<uint32_t> have;
    have.reserve((size_t)kept * 2 + 16);
    for (int c = 0; c < kept; ++c) have.insert(tri_code(cuts[c].type, cuts[c].i, cuts[c].j, cuts[c].k));
    int next = kept, added = 0;
    for (int q = 0; q < list_size; ++q) {
        if (next == BQB_MAX_TRI_INEQ) break;
        if (have.count(list[q].code)) continue;
        int t, i, j, k;
        tri_decode(list[q].code, &t, &i, &j, &k);
        cuts[next].type = t;
        cuts[next].i = i;
        cuts[next].j = j;
        cuts[next].k = k;
        cuts[next].value = list[q].value;
        cuts[next].y = 0.0;
        ++next;
        ++added;
    }
    return added;
}

template <int K, class Ineq>
static int kgon_purge(Ineq* cuts, int n_ineq, const double* y)
{
    int next = 0;
    for (int c = 0; c < n_ineq; ++c) {
        cuts[c].y = y[c];
        if (cuts[c].y < 1e-5) continue;
        cuts[next].type = cuts[c].type;
        cuts[next].y = cuts[c].y;
        for (int a = 0; a < K; ++a) cuts[next].permutation[a] = cuts[c].permutation[a];
        ++next;
    }
    return next;
}

template <int K, class Ineq, int MAXADD>
static int kgon_append(Ineq* cuts, int kept, const Ineq* list, int size)
{
    auto key = [](const Ineq& q) {
        std::array<int, 8> a{};
        a[0] = q.type;
        for (int i = 0; i < K; ++i) a[i + 1] = q.permutation[i];
        return a;
    };
    std::unordered_set<std::array<int, 8>, Key8Hash> have;
    have.reserve((size_t)kept * 2 + 16);
    for (int c = 0; c < kept; ++c) have.insert(key(cuts[c]));
    int next = kept, added = 0;
    for (int q = 0; q < size; ++q) {
        if (next == MAXADD) break;
        if (have.count(key(list[q]))) continue;
        cuts[next].type = list[q].type;
        for (int a = 0; a < K; ++a) cuts[next].permutation[a] = list[q].permutation[a];
        cuts[next].value = list[q].value;
        cuts[next].y = 0.0;
        ++next;
        ++added;
    }
    return added;
}

int pent_purge(Pentagonal_Inequality* c, int n, const double* y) { return kgon_purge<5>(c, n, y); }
int hept_purge(Heptagonal_Inequality* c, int n, const double* y) { return kgon_purge<7>(c, n, y); }
int pent_append(Pentagonal_Inequality* c, int kept, const Pentagonal_Inequality* l, int s)
{
    return kgon_append<5, Pentagonal_Inequality, BQB_MAX_PENT_INEQ>(c, kept, l, s);
}
int hept_append(Heptagonal_Inequality* c, int kept, const Heptagonal_Inequality* l, int s)
{
    return kgon_append<7, Heptagonal_Inequality, BQB_MAX_HEPTA_INEQ>(c, kept, l, s);
}

}  // namespace bqb

using namespace bqb;

// ---- drop-in entry points ----------------------------------------------

BQB_API double evaluateTriangleInequality(double* XX, int N, int type, int ii, int jj, int kk)
{
    double v[4];
    tri_values(XX[ii + jj * N], XX[ii + kk * N], XX[jj + kk * N], v);
    return (type >= 1 && type <= 3) ? v[type - 1] : v[3];
}

namespace {
DevBuf<double>& sep_x()
{
    static DevBuf<double> b;
    return b;
}
}  // namespace

BQB_API double getViolated_TriangleInequalities(double* Xm, int N, Triangle_Inequality* Lst, int* ListSize)
{
    Runtime& R = rt();
    TriSepState& st = trisep_state();
    double* dX = sep_x().ensure((size_t)N * N);
    BQB_CUDA(cudaMemcpyAsync(dX, Xm, (size_t)N * N * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    int size = 0;
    const double mx = trisep_device(st, dX, N, params.TriIneq, params.violated_TriIneq, &size, R.stream);
    for (int q = 0; q < size; ++q) {
        int t, i, j, k;
        tri_decode(st.hlist.p[q].code, &t, &i, &j, &k);
        Lst[q].type = t;
        Lst[q].i = i;
        Lst[q].j = j;
        Lst[q].k = k;
        Lst[q].value = st.hlist.p[q].value;
    }
    *ListSize = size;
    return mx;
}

BQB_API double updateTriangleInequalities(Problem* P, double* y, int* NumAdded, int* NumSubtracted)
{
    const int kept = tri_purge(Cuts, P->NIneq, y);
    const int subtracted = P->NIneq - kept;
    P->NIneq = kept;
    Runtime& R = rt();
    TriSepState& st = trisep_state();
    const int N = P->n;
    double* dX = sep_x().ensure((size_t)N * N);
    BQB_CUDA(cudaMemcpyAsync(dX, X, (size_t)N * N * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    int size = 0;
    const double mx = trisep_device(st, dX, N, params.TriIneq, params.violated_TriIneq, &size, R.stream);
    const int added = tri_append(Cuts, kept, st.hlist.p, size);
    P->NIneq += added;
    *NumAdded = added;
    *NumSubtracted = subtracted;
    return mx;
}

BQB_API double getViolated_PentagonalInequalities(double* Xm, int N, Pentagonal_Inequality* Lst, int* ListSize)
{
    return pent_separate(Xm, N, Lst, ListSize, default_engine().rng);
}

BQB_API double getViolated_HeptagonalInequalities(double* Xm, int N, Heptagonal_Inequality* Lst, int* ListSize)
{
    return hept_separate(Xm, N, Lst, ListSize, default_engine().rng);
}

namespace bqb {

double pent_update(HostState& H, Problem* P, const double* y, int* NumAdded, int* NumSubtracted, int triag, Rng& rng)
{
    const int kept = pent_purge(H.pcuts, P->NPentIneq, y + triag);
    const int subtracted = P->NPentIneq - kept;
    P->NPentIneq = kept;
    int size = 0;
    const double mn = pent_separate(H.X, P->n, H.plist, &size, rng);
    const int added = pent_append(H.pcuts, kept, H.plist, size);
    P->NPentIneq += added;
    *NumAdded = added;
    *NumSubtracted = subtracted;
    return mn;
}

double hept_update(HostState& H, Problem* P, const double* y, int* NumAdded, int* NumSubtracted, int hept_index,
                   Rng& rng)
{
    const int kept = hept_purge(H.hcuts, P->NHeptaIneq, y + hept_index);
    const int subtracted = P->NHeptaIneq - kept;
    P->NHeptaIneq = kept;
    int size = 0;
    const double mn = hept_separate(H.X, P->n, H.hlist, &size, rng);
    const int added = hept_append(H.hcuts, kept, H.hlist, size);
    P->NHeptaIneq += added;
    *NumAdded = added;
    *NumSubtracted = subtracted;
    return mn;
}

namespace {

template <int K>
double kgon_separate_dev(Engine& E, int n, int types, int trials, int* chains_out)
{
    const int chains = trials > 0 ? trials * types : 0;
    *chains_out = chains;
    if (chains == 0 || n < K) return BIG_NUMBER;
    const uint64_t seed = E.sa_seed + E.sa_calls++;
    kgon_sa_device(E.sa, E.nd.X.p, n, K, types, chains, seed, E.stream);
    return 0.0;
}

}  // namespace

double pent_update_dev(Engine& E, HostState& H, Problem* P, const double* y, int* NumAdded, int* NumSubtracted,
                       int triag)
{
    const int kept = pent_purge(H.pcuts, P->NPentIneq, y + triag);
    const int subtracted = P->NPentIneq - kept;
    P->NPentIneq = kept;
    int size = 0, chains = 0;
    double mn = kgon_separate_dev<5>(E, P->n, 3, params.Pent_Trials, &chains);
    if (chains > 0 && P->n >= 5) mn = pent_collect(E.sa.hcost.p, E.sa.hperm.p, chains, H.plist, &size);
    const int added = pent_append(H.pcuts, kept, H.plist, size);
    P->NPentIneq += added;
    *NumAdded = added;
    *NumSubtracted = subtracted;
    return mn;
}

double hept_update_dev(Engine& E, HostState& H, Problem* P, const double* y, int* NumAdded, int* NumSubtracted,
                       int hept_index)
{
    const int kept = hept_purge(H.hcuts, P->NHeptaIneq, y + hept_index);
    const int subtracted = P->NHeptaIneq - kept;
    P->NHeptaIneq = kept;
    int size = 0, chains = 0;
    double mn = kgon_separate_dev<7>(E, P->n, 4, params.Hepta_Trials, &chains);
    if (chains > 0 && P->n >= 7) mn = hept_collect(E.sa.hcost.p, E.sa.hperm.p, chains, H.hlist, &size);
    const int added = hept_append(H.hcuts, kept, H.hlist, size);
    P->NHeptaIneq += added;
    *NumAdded = added;
    *NumSubtracted = subtracted;
    return mn;
}

}  // namespace bqb

// GPU annealing chains on a host matrix (test and inspection entry point).
BQB_API int bqb_kgon_sa(const double* Xm, int n, int k, int types, int chains, unsigned long long seed,
                        double* cost, int* perm)
{
    if (n < k || (k != 5 && k != 7) || types < 1 || chains < 0) return 2;
    if (chains == 0) return 0;
    Runtime& R = rt();
    static KgonSaState st;
    static DevBuf<double> dX;
    double* d = dX.ensure((size_t)n * n);
    BQB_CUDA(cudaMemcpyAsync(d, Xm, (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    kgon_sa_device(st, d, n, k, types, chains, seed, R.stream);
    memcpy(cost, st.hcost.p, (size_t)chains * sizeof(double));
    memcpy(perm, st.hperm.p, (size_t)chains * 7 * sizeof(int));
    return st.hstat.p[0] ? 1 : 0;
}

BQB_API double updatePentagonalInequalities(Problem* P, double* y, int* NumAdded, int* NumSubtracted, int triag)
{
    Engine& E = default_engine();
    HostState H = E.host();
    return pent_update(H, P, y, NumAdded, NumSubtracted, triag, E.rng);
}

BQB_API double updateHeptagonalInequalities(Problem* P, double* y, int* NumAdded, int* NumSubtracted,
                                            int hept_index)
{
    Engine& E = default_engine();
    HostState H = E.host();
    return hept_update(H, P, y, NumAdded, NumSubtracted, hept_index, E.rng);
}
