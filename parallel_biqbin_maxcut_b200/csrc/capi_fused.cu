// Host side of the fused node kernel (nodek.cu): bqb_bound_nodes_fused.
//
// One call bounds a batch of nodes of the problem set up by
// process_adj_matrix: the nodes' fixings go to the device, one persistent
// kernel bounds them all (one CTA per SM, nodes pulled from a counter),
// bounds, fractional solutions and the best heuristic solution of every
// node come back.  The incumbent enters as Bab_LBGet() and every improvement
// found on the device is passed to Bab_LBUpd in node order afterwards.
// Nodes the kernel flags (slot capacities, numerical failures) are bounded
// again by an engine (bqb_bound_nodes), which follows the reference's code
// path exactly.
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "engine.h"
#include "globals.h"
#include "ipm.cuh"
#include "nodek.h"

extern "C" {
double Bab_LBGet(void);
int Bab_LBUpd(double new_lb, BabSolution* bs);
int bqb_bound_nodes(BabNode* nodes, int count, int rank, int threads, const double* const* L_dev, double* bounds);
extern double diff;
}

namespace bqb {
namespace {

struct FusedState {
    std::mutex mu;
    cudaStream_t stream = nullptr;
    DevBuf<unsigned char> arena;
    DevBuf<double> P0L, bound, fracsol, hval;
    DevBuf<int> xf, sx, hsol, status, next, order;
    DevBuf<unsigned long long> node_ns;
    std::vector<double> last_node_ms;
    DevBuf<unsigned long long> lb, prof;
    HostBuf<int> hfix;
    HostBuf<double> hb, hfs, hhv;
    HostBuf<int> hhs, hst, hord;
    HostBuf<unsigned long long> hns;
    const double* P0L_src = nullptr;
    int P0N = 0;
    unsigned P0L_gen = 0;
    unsigned long long seed = 0x5eed0f0cb200ull;
    unsigned long long calls = 0;
    long long fallbacks = 0;
    // timing of the fused kernel (CUDA events on its stream)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double st_calls = 0, st_nodes = 0, st_kernel_ms = 0, st_fallback_nodes = 0, st_fallback_ms = 0;
};

FusedState& fstate()
{
    static FusedState s;
    return s;
}

unsigned long long host_ordered(double x)
{
    unsigned long long u;
    memcpy(&u, &x, sizeof u);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

int next_pow2(int v)
{
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

}  // namespace
}  // namespace bqb

using namespace bqb;

// Fused bounding of `count` nodes (see include/bqb_gpu.h).
BQB_API int bqb_bound_nodes_fused(BabNode* nodes, int count, int rank, double* bounds)
{
    if (count <= 0) return 0;
    if (!SP || !SP->L) return 1;
    Runtime& R = rt();
    const int N0 = SP->n;
    if (N0 > NK_NMAX || N0 < 3) return bqb_bound_nodes(nodes, count, rank, 16, nullptr, bounds);
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    if (!F.stream) BQB_CUDA(cudaStreamCreateWithFlags(&F.stream, cudaStreamNonBlocking));
    cudaStream_t s = F.stream;
    const int N = N0 - 1;

    FusedCfg c;
    memset(&c, 0, sizeof c);
    c.N0 = N0;
    c.count = count;
    c.rank = rank;
    c.diff = diff;
    c.init_bundle_iter = params.init_bundle_iter;
    c.max_bundle_iter = params.max_bundle_iter;
    c.triag_iter = params.triag_iter;
    c.pent_iter = params.pent_iter;
    c.hept_iter = params.hept_iter;
    c.max_outer_iter = params.max_outer_iter;
    c.extra_iter = params.extra_iter;
    c.violated_TriIneq = params.violated_TriIneq;
    c.TriIneq = params.TriIneq;
    c.PentIneq = params.PentIneq;
    c.HeptaIneq = params.HeptaIneq;
    c.Pent_Trials = params.Pent_Trials;
    c.Hepta_Trials = params.Hepta_Trials;
    c.include_Pent = params.include_Pent;
    c.include_Hepta = params.include_Hepta;
    c.use_diff = params.use_diff;
    c.seed = F.seed + 0x9E3779B97F4A7C15ull * (++F.calls);
    c.bcap = 64;
    int mt = 8 * (params.TriIneq > 0 ? params.TriIneq : 1);
    if (mt < 8192) mt = 8192;
    if (mt > BQB_MAX_TRI_INEQ) mt = BQB_MAX_TRI_INEQ;
    c.mt_cap = mt;
    c.mp_cap = 4096;
    c.mh_cap = 4096;
    c.hash_size = next_pow2(2 * mt);
    const int pc = params.Pent_Trials > 0 ? 3 * params.Pent_Trials : 0;
    const int hc = params.Hepta_Trials > 0 ? 4 * params.Hepta_Trials : 0;
    c.sa_chains = pc > hc ? pc : hc;
    c.smem_bytes = nk_smem_bytes(N0, params.TriIneq, c.bcap, R.smem_optin);
    if (c.smem_bytes > R.smem_optin) return bqb_bound_nodes(nodes, count, rank, 16, nullptr, bounds);
    const size_t slot_bytes = nk_layout(c);
    int slots = R.num_sms;
    if (slots > count) slots = count;

    // problem and node data
    const unsigned gen = g_sp_generation.load();
    if (F.P0L_src != SP->L || F.P0N != N0 || F.P0L_gen != gen) {
        F.P0L.ensure((size_t)N0 * N0);
        BQB_CUDA(cudaMemcpyAsync(F.P0L.p, SP->L, (size_t)N0 * N0 * sizeof(double), cudaMemcpyHostToDevice, s));
        F.P0L_src = SP->L;
        F.P0N = N0;
        F.P0L_gen = gen;
    }
    const size_t cN = (size_t)count * N;
    int* hf = F.hfix.ensure(2 * cN);
    for (int i = 0; i < count; ++i) {
        memcpy(hf + (size_t)i * N, nodes[i].xfixed, N * sizeof(int));
        memcpy(hf + cN + (size_t)i * N, nodes[i].sol.X, N * sizeof(int));
    }
    // heaviest nodes first (longest-processing-time order): a node's work
    // grows with its subproblem size, so free vertices decide the order
    {
        std::vector<int> ord(count);
        std::vector<int> nfree(count);
        for (int i = 0; i < count; ++i) {
            ord[i] = i;
            int nf = 0;
            for (int j = 0; j < N; ++j) nf += nodes[i].xfixed[j] ? 0 : 1;
            nfree[i] = nf;
        }
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return nfree[a] > nfree[b]; });
        int* ho = F.hord.ensure(count);
        memcpy(ho, ord.data(), count * sizeof(int));
        F.order.ensure(count);
        BQB_CUDA(cudaMemcpyAsync(F.order.p, ho, count * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    F.xf.ensure(cN);
    F.sx.ensure(cN);
    BQB_CUDA(cudaMemcpyAsync(F.xf.p, hf, cN * sizeof(int), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemcpyAsync(F.sx.p, hf + cN, cN * sizeof(int), cudaMemcpyHostToDevice, s));
    F.bound.ensure(count);
    F.fracsol.ensure(cN);
    F.hval.ensure(count);
    F.hsol.ensure(cN);
    F.status.ensure(count);
    F.node_ns.ensure(count);
    F.next.ensure(1);
    F.lb.ensure(1);
    F.arena.ensure(slot_bytes * slots);
    BQB_CUDA(cudaMemsetAsync(F.next.p, 0, sizeof(int), s));
    const unsigned long long lb0 = host_ordered(Bab_LBGet());
    BQB_CUDA(cudaMemcpyAsync(F.lb.p, &lb0, sizeof lb0, cudaMemcpyHostToDevice, s));
    c.P0L = F.P0L.p;
    c.xfixed = F.xf.p;
    c.solx = F.sx.p;
    c.bound = F.bound.p;
    c.fracsol = F.fracsol.p;
    c.hval = F.hval.p;
    c.hsol = F.hsol.p;
    c.status = F.status.p;
    c.node_ns = F.node_ns.p;
    c.order = F.order.p;
    c.next = F.next.p;
    c.lb = F.lb.p;
    c.ipm_stats = ipm_stats_device();
    if (!F.prof.p) {
        F.prof.ensure(NKP_COUNT);
        BQB_CUDA(cudaMemsetAsync(F.prof.p, 0, NKP_COUNT * sizeof(unsigned long long), s));
    }
    c.prof = F.prof.p;
    c.arena = F.arena.p;
    if (!F.ev0) {
        BQB_CUDA(cudaEventCreate(&F.ev0));
        BQB_CUDA(cudaEventCreate(&F.ev1));
    }
    BQB_CUDA(cudaEventRecord(F.ev0, s));
    nk_launch(c, slots, s);
    BQB_CUDA(cudaEventRecord(F.ev1, s));

    double* hb = F.hb.ensure(count);
    double* hfs = F.hfs.ensure(cN);
    double* hhv = F.hhv.ensure(count);
    int* hhs = F.hhs.ensure(cN);
    int* hst = F.hst.ensure(count);
    BQB_CUDA(cudaMemcpyAsync(hb, F.bound.p, count * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(hfs, F.fracsol.p, cN * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(hhv, F.hval.p, count * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(hhs, F.hsol.p, cN * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(hst, F.status.p, count * sizeof(int), cudaMemcpyDeviceToHost, s));
    unsigned long long* hns = F.hns.ensure(count);
    BQB_CUDA(cudaMemcpyAsync(hns, F.node_ns.p, count * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    F.last_node_ms.assign(count, 0.0);
    for (int i = 0; i < count; ++i) F.last_node_ms[i] = 1e-6 * (double)hns[i];
    float kms = 0.f;
    BQB_CUDA(cudaEventElapsedTime(&kms, F.ev0, F.ev1));
    F.st_calls += 1;
    F.st_nodes += count;
    F.st_kernel_ms += kms;

    std::vector<int> redo;
    for (int i = 0; i < count; ++i) {
        if (hst[i]) {
            redo.push_back(i);
            continue;
        }
        bounds[i] = hb[i];
        memcpy(nodes[i].fracsol, hfs + (size_t)i * N, N * sizeof(double));
    }
    // incumbent updates in node order (updateSolution's test and update)
    for (int i = 0; i < count; ++i) {
        if (!(hhv[i] > Bab_LBGet())) continue;
        BabSolution bs;
        memset(&bs, 0, sizeof bs);
        memcpy(bs.X, hhs + (size_t)i * N, N * sizeof(int));
        Bab_LBUpd(hhv[i], &bs);
    }
    if (!redo.empty()) {
        F.fallbacks += (long long)redo.size();
        std::vector<BabNode> sub(redo.size());
        std::vector<double> sb(redo.size());
        for (size_t q = 0; q < redo.size(); ++q) sub[q] = nodes[redo[q]];
        const int th = redo.size() < 16 ? (int)redo.size() : 16;
        BQB_CUDA(cudaEventRecord(F.ev0, s));
        const int rc = bqb_bound_nodes(sub.data(), (int)sub.size(), rank, th, nullptr, sb.data());
        BQB_CUDA(cudaEventRecord(F.ev1, s));
        BQB_CUDA(cudaEventSynchronize(F.ev1));
        float fms = 0.f;
        BQB_CUDA(cudaEventElapsedTime(&fms, F.ev0, F.ev1));
        F.st_fallback_nodes += (double)redo.size();
        F.st_fallback_ms += fms;
        if (rc) return rc;
        for (size_t q = 0; q < redo.size(); ++q) {
            nodes[redo[q]] = sub[q];
            bounds[redo[q]] = sb[q];
        }
    }
    return 0;
}

// Nodes the fused kernel handed back to an engine since the process started.
BQB_API long long bqb_fused_fallbacks(void) { return fstate().fallbacks; }

// out[5] = {calls, nodes, fused kernel ms, nodes bounded again by engines,
// their ms} since the last reset (CUDA events on the fused stream; the
// fallback interval brackets the engines' work from that stream, which the
// engines synchronise before returning).
BQB_API void bqb_fused_stats(double* out)
{
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    out[0] = F.st_calls;
    out[1] = F.st_nodes;
    out[2] = F.st_kernel_ms;
    out[3] = F.st_fallback_nodes;
    out[4] = F.st_fallback_ms;
}

// Device milliseconds of every node of the last bqb_bound_nodes_fused call
// (as many as that call had, at most `count`); returns how many were written.
BQB_API int bqb_fused_node_times(double* out, int count)
{
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    const int m = (int)F.last_node_ms.size() < count ? (int)F.last_node_ms.size() : count;
    for (int i = 0; i < m; ++i) out[i] = F.last_node_ms[i];
    return m;
}

BQB_API void bqb_fused_stats_reset(void)
{
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    F.st_calls = F.st_nodes = F.st_kernel_ms = F.st_fallback_nodes = F.st_fallback_ms = 0;
    if (F.prof.p) BQB_CUDA(cudaMemset(F.prof.p, 0, NKP_COUNT * sizeof(unsigned long long)));
}

// Time per phase of the fused kernel (seconds, summed over its CTAs) since
// the last reset: out[11] = {subproblem, IPM, heuristic, triangle scan,
// triangle list update, k-gonal separation, cut upload, B^T, B, lambda_eta,
// bundle step}.
BQB_API void bqb_fused_profile(double* out)
{
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    unsigned long long h[NKP_COUNT] = {};
    if (F.prof.p) BQB_CUDA(cudaMemcpy(h, F.prof.p, sizeof h, cudaMemcpyDeviceToHost));
    for (int i = 0; i < NKP_COUNT; ++i) out[i] = 1e-9 * (double)h[i];
}
