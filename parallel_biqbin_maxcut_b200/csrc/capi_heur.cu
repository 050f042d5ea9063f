// Heuristic entry points: runHeuristic, runHeuristic_unpacked, GW_heuristic,
// mc_1opt, update_best.  The GPU does the factorisation, projection, 1-opt
// and evaluation; the host keeps the reference's control flow and draws
// every random number from the engine's stream in the reference's order
// (src/heuristic.c:38-39, 103, 142-143), so for the same rand() state and
// the same X the heuristic values and cuts are the reference's.
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <vector>

#include "engine.h"
#include "globals.h"
#include "heur.cuh"
#include "internal.h"

extern "C" double evaluateSolution(int* sol);

namespace bqb {

namespace {
constexpr double BIG_NUMBER = 1e9;

// Upload the node's fixed variables in the eval_kernel layout.
void upload_fixed(HeurState& st, const int* xfixed, const int* sol, int N, cudaStream_t s)
{
    std::vector<int> h(3 * (size_t)N);
    int rank = 0;
    for (int i = 0; i < N; ++i) {
        h[i] = xfixed[i] ? 1 : 0;
        h[N + i] = sol[i];
        h[2 * N + i] = xfixed[i] ? 0 : rank++;
    }
    int* d = st.fixed.ensure(3 * (size_t)N);
    BQB_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaStreamSynchronize(s));
}

void ensure_round_buffers(HeurState& st, int n, int N0, int num)
{
    st.Z.ensure((size_t)n * n);
    st.V.ensure((size_t)num * n);
    st.x.ensure((size_t)num * n);
    st.sols.ensure((size_t)num * (N0 - 1 > 0 ? N0 - 1 : 1));
    st.vals.ensure(num > 1 ? num : 1);
    st.best.ensure((size_t)N0 + 1);
    st.bestval.ensure(1);
    st.status.ensure(2);
    st.hbest.ensure((size_t)N0 + 1);
    st.hval.ensure(2);
    st.hstat.ensure(2);
}

// Hyperplanes v_i = rand()/RAND_MAX - 0.5, count-major (src/heuristic.c:142-143).
void draw_hyperplanes(HeurState& st, Rng& rng, int n, int num, cudaStream_t s)
{
    double* hv = st.hV.ensure((size_t)num * n);
    for (int c = 0; c < num; ++c)
        for (int i = 0; i < n; ++i) hv[(size_t)c * n + i] = ((double)rng.next() / (double)(RAND_MAX)) - 0.5;
    BQB_CUDA(cudaMemcpyAsync(st.V.p, hv, (size_t)num * n * sizeof(double), cudaMemcpyHostToDevice, s));
}

// Run one GW round on the factor already in st.Z; copy the best cut to x.
double gw_round_host(HeurState& st, Rng& rng, const double* dPL, int n, const double* dP0L, int N0, int num,
                     int* x, cudaStream_t s)
{
    draw_hyperplanes(st, rng, n, num, s);
    BQB_CUDA(cudaMemsetAsync(st.status.p, 0, 2 * sizeof(int), s));
    gw_round_device(st, dPL, n, dP0L, N0, num, s);
    BQB_CUDA(cudaMemcpyAsync(st.hbest.p, st.best.p, (size_t)N0 * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(st.hval.p, st.bestval.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(st.hstat.p, st.status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    if (st.hstat.p[1]) fatal("GW_heuristic", "1-opt did not terminate");
    if (num > 0) memcpy(x, st.hbest.p + 1, (size_t)(N0 - 1) * sizeof(int));
    return num > 0 ? st.hval.p[0] : -BIG_NUMBER;
}

// A GW round of H hyperplanes at once: the hyperplanes are drawn on the
// device from a seed taken from the engine's stream (two draws), projected
// on the tensor cores with the sign in the epilogue (gw_project_tf32), then
// 1-opt, lifting, exact evaluation and the first best as in every round.
double gw_round_batched(HeurState& st, Rng& rng, const double* dPL, int n, const double* dP0L, int N0, int H,
                        int* x, cudaStream_t s)
{
    const unsigned long long seed =
        ((unsigned long long)(unsigned)rng.next() << 31) ^ (unsigned long long)(unsigned)rng.next();
    BQB_CUDA(cudaMemsetAsync(st.status.p, 0, 2 * sizeof(int), s));
    const cudaError_t e = gw_project_tf32(st.Z.p, n, H, seed, st.x.p, st.Vf, st.tcerr, s);
    if (e != cudaSuccess) fatal("GW_heuristic (batched projection)", cudaGetErrorString(e));
    gw_round_finish(st, dPL, n, dP0L, N0, H, s);
    int terr = 0;
    BQB_CUDA(cudaMemcpyAsync(st.hbest.p, st.best.p, (size_t)N0 * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(st.hval.p, st.bestval.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(st.hstat.p, st.status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(&terr, st.tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    if (terr) fatal("GW_heuristic", "a bounded wait in the tensor-core projection ran out");
    if (st.hstat.p[1]) fatal("GW_heuristic", "1-opt did not terminate");
    memcpy(x, st.hbest.p + 1, (size_t)(N0 - 1) * sizeof(int));
    return st.hval.p[0];
}

std::atomic<int> g_gw_hyperplanes{0};

}  // namespace

int gw_hyperplanes() { return g_gw_hyperplanes.load(); }

// runHeuristic_unpacked (src/heuristic.c:19-115) with device-resident X, P_L
// and P0_L.  x: host, length N0 - 1.  hyperplanes > 0: every GW round
// projects that many device-drawn hyperplanes at once on the tensor cores
// (gw_round_batched) instead of N0 host-drawn ones in rand() order.
double heuristic_device(HeurState& st, Rng& rng, const double* dX, const double* dPL, int n, const double* dP0L,
                        int N0, const int* xfixed, const int* sol, int* x, cudaStream_t s, int hyperplanes)
{
    const int N = N0 - 1;
    const int num = hyperplanes > 0 ? hyperplanes : N0;
    ensure_round_buffers(st, n, N0, num);
    upload_fixed(st, xfixed, sol, N, s);

    std::vector<double> xh(n);
    for (int i = 0; i < n; ++i) xh[i] = 2 * (rng.next() % 2) - 1;
    // fh = value of the random cut lifted with the fixed variables
    {
        std::vector<int> tx(N);
        int idx = 0;
        for (int i = 0; i < N; ++i) {
            if (xfixed[i])
                tx[i] = sol[i];
            else
                tx[i] = (int)((xh[idx++] + 1) / 2.0);
        }
        BQB_CUDA(cudaMemcpyAsync(st.sols.p, tx.data(), (size_t)N * sizeof(int), cudaMemcpyHostToDevice, s));
        evaluate_device(st, dP0L, N0, 1, s);
    }
    double fh;
    BQB_CUDA(cudaMemcpyAsync(&st.hval.p[1], st.vals.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    fh = st.hval.p[1];

    DevBuf<double>& dxh = st.Xs;   // reuse as the xh staging vector
    dxh.ensure((size_t)n);
    BQB_CUDA(cudaMemcpyAsync(st.Z.p, dX, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    int done = 0;
    double heur_val = -BIG_NUMBER;
    while (done < 2) {
        ++done;
        potrf_device(st.Z.p, n, st.status.p, s);
        BQB_CUDA(cudaMemcpyAsync(st.hstat.p, st.status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaStreamSynchronize(s));
        if (st.hstat.p[0]) {
            fatal("runHeuristic_unpacked", "Problem with Cholesky factorization");
            return heur_val;
        }
        heur_val = hyperplanes > 0 ? gw_round_batched(st, rng, dPL, n, dP0L, N0, num, x, s)
                                   : gw_round_host(st, rng, dPL, n, dP0L, N0, num, x, s);
        if (heur_val > fh) {
            done = 0;
            fh = heur_val;
            int idx = 0;
            for (int i = 0; i < N; ++i)
                if (!xfixed[i]) xh[idx++] = 2 * x[i] - 1;
            xh[n - 1] = -1.0;
        }
        const double c = 0.3 + 0.6 * ((double)rng.next() / (double)(RAND_MAX));
        BQB_CUDA(cudaMemcpyAsync(dxh.p, xh.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
        remix_device(st.Z.p, dX, dxh.p, c, n, s);
        BQB_CUDA(cudaStreamSynchronize(s));   // xh is reused on the host
    }
    return heur_val;
}

}  // namespace bqb

using namespace bqb;

namespace {
struct HeurStage {
    DevBuf<double> X, PL, P0L;
};
HeurStage& hstage()
{
    static HeurStage s;
    return s;
}
}  // namespace

BQB_API double runHeuristic_unpacked(double* P0_L, int P0_N, double* P_L, int P_N, int* node_xfixed,
                                     int* node_sol_X, int* x)
{
    Runtime& R = rt();
    HeurStage& h = hstage();
    const size_t nn = (size_t)P_N * P_N, NN = (size_t)P0_N * P0_N;
    double* dX = h.X.ensure(nn);
    double* dPL = h.PL.ensure(nn);
    double* dP0L = h.P0L.ensure(NN);
    BQB_CUDA(cudaMemcpyAsync(dX, X, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    BQB_CUDA(cudaMemcpyAsync(dPL, P_L, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    BQB_CUDA(cudaMemcpyAsync(dP0L, P0_L, NN * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    Engine& E = default_engine();
    return heuristic_device(E.heur, E.rng, dX, dPL, P_N, dP0L, P0_N, node_xfixed, node_sol_X, x, R.stream);
}

BQB_API double runHeuristic(Problem* P0, Problem* P, BabNode* node, int* x)
{
    return runHeuristic_unpacked(P0->L, P0->n, P->L, P->n, node->xfixed, node->sol.X, x);
}

// GW_heuristic (src/heuristic.c:119-186): the factor is the global Z (lower
// triangle), as the reference reads it.
BQB_API double GW_heuristic(double* P0_L, int P0_N, double* P_L, int P_N, int* node_xfixed, int* node_sol_X,
                            int* x, int num)
{
    Runtime& R = rt();
    HeurState& st = default_engine().heur;
    HeurStage& h = hstage();
    const size_t nn = (size_t)P_N * P_N, NN = (size_t)P0_N * P0_N;
    ensure_round_buffers(st, P_N, P0_N, num > 0 ? num : 1);
    double* dPL = h.PL.ensure(nn);
    double* dP0L = h.P0L.ensure(NN);
    BQB_CUDA(cudaMemcpyAsync(st.Z.p, Z, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    BQB_CUDA(cudaMemcpyAsync(dPL, P_L, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    BQB_CUDA(cudaMemcpyAsync(dP0L, P0_L, NN * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    upload_fixed(st, node_xfixed, node_sol_X, P0_N - 1, R.stream);
    if (num <= 0) return -BIG_NUMBER;
    return gw_round_host(st, default_engine().rng, dPL, P_N, dP0L, P0_N, num, x, R.stream);
}

// mc_1opt (src/heuristic.c:195-296): x in +-1 form, improved in place;
// returns x'Lx after the local search.
BQB_API double mc_1opt(int* x, double* P_L, int P_N)
{
    Runtime& R = rt();
    HeurState& st = default_engine().heur;
    HeurStage& h = hstage();
    const size_t nn = (size_t)P_N * P_N;
    st.x.ensure((size_t)P_N);
    st.vals.ensure(1);
    st.status.ensure(2);
    st.hval.ensure(2);
    st.hstat.ensure(2);
    double* dPL = h.PL.ensure(nn);
    BQB_CUDA(cudaMemcpyAsync(dPL, P_L, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    BQB_CUDA(cudaMemcpyAsync(st.x.p, x, (size_t)P_N * sizeof(int), cudaMemcpyHostToDevice, R.stream));
    BQB_CUDA(cudaMemsetAsync(st.status.p, 0, 2 * sizeof(int), R.stream));
    one_opt_device(st, dPL, P_N, 1, R.stream);
    BQB_CUDA(cudaMemcpyAsync(x, st.x.p, (size_t)P_N * sizeof(int), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaMemcpyAsync(st.hval.p, st.vals.p, sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaMemcpyAsync(st.hstat.p, st.status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaStreamSynchronize(R.stream));
    if (st.hstat.p[1]) fatal("mc_1opt", "local search did not terminate");
    return st.hval.p[0];
}

// update_best (src/heuristic.c:304-318).
BQB_API int update_best(int* xbest, int* xnew, double* best, int P0_N)
{
    const double v = evaluateSolution(xnew);
    if (*best < v) {
        memcpy(xbest, xnew, sizeof(int) * (size_t)(P0_N - 1));
        *best = v;
        return 1;
    }
    return 0;
}

// Hyperplanes per GW round for the concurrent engines and the solvers built
// on them (0, the default: the reference's P0_N hyperplanes drawn on the host
// in rand() order; H > 0: H hyperplanes drawn on the device and projected at
// once on the tensor cores).  The drop-in entry points always follow the
// reference.  Values above 65536 are clamped.
BQB_API void bqb_set_gw_hyperplanes(int H)
{
    g_gw_hyperplanes.store(H < 0 ? 0 : (H > 65536 ? 65536 : H));
}
