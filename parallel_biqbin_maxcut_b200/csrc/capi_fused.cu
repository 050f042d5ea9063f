// Host side of the fused node kernel (nodek.cu).
//
// One submission bounds a batch of nodes of the problem set up by
// process_adj_matrix: the nodes' fixings go to the device, one persistent
// kernel bounds them all (one CTA per SM, heaviest nodes first, nodes pulled
// from a counter), and bounds, fractional solutions and the best heuristic
// solution of every node come back.  The incumbent enters as Bab_LBGet()
// and every improvement found on the device is passed to Bab_LBUpd in node
// order when the batch is collected.  Nodes the kernel flags (slot
// capacities, numerical failures) are bounded again by engines
// (bqb_bound_nodes), which follow the reference's code path exactly.
//
// A submission takes one of NK_SUBS submission slots (its fixings, its
// ticket) until it is collected; a launch takes one of NK_LAUNCHES launch
// records (stream, events, device arena, node buffers, pinned result
// buffers) until every submission it carries has been collected.  The two
// are separate so that a launch carrying several submissions never holds a
// submission slot: a slot frees when its own submission is collected.
// Every busy launch record carries at least one uncollected submission, so
// with NK_LAUNCHES >= NK_SUBS a launch record is free whenever staged
// submissions are launched.  Several launches are in flight at once: when
// the last, heaviest nodes of one batch hold a few SMs, the next batch's
// CTAs take the rest.  A submission made while a launch is running waits
// on the host; the next collect (or the next submission that finds the GPU
// idle) launches every waiting submission as one kernel, whose node order
// is heaviest-first over all of them, so the heavy nodes of later batches
// start early instead of forming the tail of the last launch.  Each
// submission is still collected on its own, in any order.
// bqb_bound_nodes_fused is a submission collected at once.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <vector>

#include "engine.h"
#include "globals.h"
#include "internal.h"
#include "ipm.cuh"
#include "nodek.h"

extern "C" {
double Bab_LBGet(void);
int Bab_LBUpd(double new_lb, BabSolution* bs);
int bqb_bound_nodes(BabNode* nodes, int count, int rank, int threads, const double* const* L_dev, double* bounds);
int getBranchingVariable(BabNode* node);
extern double diff;
}

namespace bqb {
namespace {

constexpr int NK_SUBS = 8;
constexpr int NK_LAUNCHES = NK_SUBS;
static_assert(NK_LAUNCHES >= NK_SUBS, "a staged submission must always find a free launch record");

// One uncollected submission.
struct FusedSub {
    bool busy = false;       // holds an uncollected submission
    bool launched = false;   // its nodes are in a launch
    int launch = -1;         // the launch record carrying its nodes
    int offset = 0;          // its first node in that launch's arrays
    int count = 0, rank = 0, N = 0;
    unsigned long long ticket = 0;
    HostBuf<int> hfix;       // xfixed rows then sol.X rows, count x N each
};

// One launch of the fused kernel and its buffers.
struct FusedLaunch {
    int refs = 0;            // uncollected submissions it carries (0: free)
    bool counted = false;    // launch time added to the statistics
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevBuf<unsigned char> arena;
    DevBuf<double> bound, fracsol, hval;
    DevBuf<int> xf, sx, hsol, status, next, order;
    DevBuf<unsigned long long> lb, node_ns;
    HostBuf<int> gfix, hhs, hst, hord;
    HostBuf<double> hb, hfs, hhv;
    HostBuf<unsigned long long> hns, hlb;
};

struct FusedState {
    std::mutex mu;
    FusedSub sub[NK_SUBS];
    FusedLaunch run[NK_LAUNCHES];
    unsigned long long next_ticket = 0;
    DevBuf<double> P0L;
    DevBuf<unsigned long long> prof;
    const double* P0L_src = nullptr;
    int P0N = 0;
    unsigned P0L_gen = 0;
    unsigned long long seed = 0x5eed0f0cb200ull;
    long long fallbacks = 0;
    std::vector<double> last_node_ms;
    double st_calls = 0, st_nodes = 0, st_kernel_ms = 0, st_fallback_nodes = 0, st_fallback_ms = 0;
    long long st_launches = 0;
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

// The reference parameters and slot capacities of a launch.
void fill_cfg(FusedCfg& c, int N0, int count, int rank, unsigned long long seed, size_t smem_optin)
{
    memset(&c, 0, sizeof c);
    c.le_prof = le_prof_device();
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
    c.seed = seed;
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
    c.smem_bytes = nk_smem_bytes(N0, params.TriIneq, c.bcap, smem_optin);
}

bool fused_supported(int N0, size_t smem_optin)
{
    if (N0 > NK_NMAX || N0 < 3) return false;
    FusedCfg c;
    fill_cfg(c, N0, 1, 1, 0, smem_optin);
    return c.smem_bytes <= smem_optin;
}

// Stage a submission in slot S: its fixings go to S's pinned buffer (the
// caller holds F.mu).
void stage(FusedState& F, FusedSub& S, const BabNode* nodes, int count, int rank)
{
    const int N = SP->n - 1;
    const size_t cN = (size_t)count * N;
    int* hf = S.hfix.ensure(2 * cN);
    for (int i = 0; i < count; ++i) {
        memcpy(hf + (size_t)i * N, nodes[i].xfixed, N * sizeof(int));
        memcpy(hf + cN + (size_t)i * N, nodes[i].sol.X, N * sizeof(int));
    }
    S.busy = true;
    S.launched = false;
    S.launch = -1;
    S.offset = 0;
    S.count = count;
    S.rank = rank;
    S.N = N;
    S.ticket = F.next_ticket++;
}

// A free launch record, its stream and events created on first use; -1 when
// every record still carries an uncollected submission (the caller holds
// F.mu).
int free_launch(FusedState& F)
{
    for (int q = 0; q < NK_LAUNCHES; ++q) {
        FusedLaunch& L = F.run[q];
        if (L.refs > 0) continue;
        if (!L.stream) {
            BQB_CUDA(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
            BQB_CUDA(cudaEventCreate(&L.ev0));
            BQB_CUDA(cudaEventCreate(&L.ev1));
        }
        return q;
    }
    return -1;
}

// One launch for the staged submissions `members` (slot indices in ticket
// order, same rank) on a free launch record (the caller holds F.mu).
// Returns false when no launch record is free.
bool launch(FusedState& F, const std::vector<int>& members)
{
    Runtime& R = rt();
    const int li = free_launch(F);
    if (li < 0) return false;
    FusedLaunch& P = F.run[li];
    const int N0 = SP->n;
    const int N = N0 - 1;
    const FusedSub& S0 = F.sub[members[0]];
    const int rank = S0.rank;
    int count = 0;
    for (int q : members) count += F.sub[q].count;
    cudaStream_t s = P.stream;
    FusedCfg c;
    fill_cfg(c, N0, count, rank, F.seed + 0x9E3779B97F4A7C15ull * (S0.ticket + 1), R.smem_optin);
    const size_t slot_bytes = nk_layout(c);
    int slots = R.num_sms;
    if (slots > count) slots = count;

    const unsigned gen = g_sp_generation.load();
    if (F.P0L_src != SP->L || F.P0N != N0 || F.P0L_gen != gen) {
        // every launch reads P0L: let the launches in flight finish first
        for (int q = 0; q < NK_LAUNCHES; ++q)
            if (F.run[q].refs > 0) BQB_CUDA(cudaStreamSynchronize(F.run[q].stream));
        F.P0L.ensure((size_t)N0 * N0);
        BQB_CUDA(cudaMemcpy(F.P0L.p, SP->L, (size_t)N0 * N0 * sizeof(double), cudaMemcpyHostToDevice));
        F.P0L_src = SP->L;
        F.P0N = N0;
        F.P0L_gen = gen;
    }
    if (!F.prof.p) {
        F.prof.ensure(2 * NKP_COUNT);
        BQB_CUDA(cudaMemset(F.prof.p, 0, 2 * NKP_COUNT * sizeof(unsigned long long)));
    }
    const size_t cN = (size_t)count * N;
    int* hf = P.gfix.ensure(2 * cN);
    int off = 0;
    for (int q : members) {
        FusedSub& M = F.sub[q];
        const size_t mN = (size_t)M.count * N;
        memcpy(hf + (size_t)off * N, M.hfix.p, mN * sizeof(int));
        memcpy(hf + cN + (size_t)off * N, M.hfix.p + mN, mN * sizeof(int));
        M.launched = true;
        M.launch = li;
        M.offset = off;
        off += M.count;
    }
    std::vector<int> ord(count), nfree(count);
    for (int i = 0; i < count; ++i) {
        int nf = 0;
        for (int j = 0; j < N; ++j) nf += hf[(size_t)i * N + j] ? 0 : 1;
        nfree[i] = nf;
        ord[i] = i;
    }
    // heaviest nodes first (longest-processing-time order): a node's work
    // grows with its subproblem size
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return nfree[a] > nfree[b]; });
    int* ho = P.hord.ensure(count);
    memcpy(ho, ord.data(), count * sizeof(int));
    P.xf.ensure(cN);
    P.sx.ensure(cN);
    P.order.ensure(count);
    P.bound.ensure(count);
    P.fracsol.ensure(cN);
    P.hval.ensure(count);
    P.hsol.ensure(cN);
    P.status.ensure(count);
    P.node_ns.ensure(count);
    P.next.ensure(1);
    P.lb.ensure(1);
    P.arena.ensure(slot_bytes * slots);
    unsigned long long* hlb = P.hlb.ensure(1);
    hlb[0] = host_ordered(Bab_LBGet());
    BQB_CUDA(cudaMemcpyAsync(P.xf.p, hf, cN * sizeof(int), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemcpyAsync(P.sx.p, hf + cN, cN * sizeof(int), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemcpyAsync(P.order.p, ho, count * sizeof(int), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemcpyAsync(P.lb.p, hlb, sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemsetAsync(P.next.p, 0, sizeof(int), s));
    c.P0L = F.P0L.p;
    c.xfixed = P.xf.p;
    c.solx = P.sx.p;
    c.bound = P.bound.p;
    c.fracsol = P.fracsol.p;
    c.hval = P.hval.p;
    c.hsol = P.hsol.p;
    c.status = P.status.p;
    c.node_ns = P.node_ns.p;
    c.order = P.order.p;
    c.next = P.next.p;
    c.lb = P.lb.p;
    c.ipm_stats = ipm_stats_device();
    c.prof = F.prof.p;
    c.warm_p = warm_device_params();
    c.warm_stats = c.warm_p ? warm_device_stats() : nullptr;
    c.arena = P.arena.p;
    BQB_CUDA(cudaEventRecord(P.ev0, s));
    nk_launch(c, slots, s);
    BQB_CUDA(cudaEventRecord(P.ev1, s));
    BQB_CUDA(cudaMemcpyAsync(P.hb.ensure(count), P.bound.p, count * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(P.hfs.ensure(cN), P.fracsol.p, cN * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(P.hhv.ensure(count), P.hval.p, count * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(P.hhs.ensure(cN), P.hsol.p, cN * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(P.hst.ensure(count), P.status.p, count * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(P.hns.ensure(count), P.node_ns.p, count * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, s));
    P.refs = (int)members.size();
    P.counted = false;
    ++F.st_launches;
    return true;
}

// Launch the staged submissions: one launch per run of equal rank, in
// ticket order (the caller holds F.mu).  Returns false when a launch found
// no free record (which the slot count rules out; the submissions stay
// staged and the caller reports the error).
bool launch_staged(FusedState& F)
{
    std::vector<int> st;
    for (int q = 0; q < NK_SUBS; ++q)
        if (F.sub[q].busy && !F.sub[q].launched) st.push_back(q);
    std::sort(st.begin(), st.end(), [&](int a, int b) { return F.sub[a].ticket < F.sub[b].ticket; });
    size_t i = 0;
    while (i < st.size()) {
        std::vector<int> group{st[i]};
        size_t j = i + 1;
        while (j < st.size() && F.sub[st[j]].rank == F.sub[st[i]].rank) group.push_back(st[j++]);
        if (!launch(F, group)) return false;
        i = j;
    }
    return true;
}

// Is a launch still running on the GPU?
bool any_running(FusedState& F)
{
    for (int q = 0; q < NK_LAUNCHES; ++q) {
        FusedLaunch& L = F.run[q];
        if (L.refs <= 0) continue;
        const cudaError_t e = cudaEventQuery(L.ev1);
        if (e == cudaErrorNotReady) return true;
        if (e != cudaSuccess) BQB_CUDA(e);
    }
    return false;
}

// Wait for submission S and hand its results to the caller's nodes (the
// caller holds F.mu).  S's slot is free when this returns; its launch record
// frees when the last submission it carries has been collected.
int collect(FusedState& F, FusedSub& S, BabNode* nodes, double* bounds)
{
    // submissions still waiting on the host start now, behind the launches
    // in flight, so they run while this one is waited for
    if (!launch_staged(F)) {
        set_error("bqb_fused_collect", "no free launch record");
        return 1;
    }
    FusedLaunch& L = F.run[S.launch];
    BQB_CUDA(cudaStreamSynchronize(L.stream));
    const int count = S.count, N = S.N, o = S.offset, rank = S.rank;
    S.busy = false;
    S.launched = false;
    S.launch = -1;
    if (!L.counted) {
        float kms = 0.f;
        BQB_CUDA(cudaEventElapsedTime(&kms, L.ev0, L.ev1));
        F.st_kernel_ms += kms;
        L.counted = true;
    }
    F.st_calls += 1;
    F.st_nodes += count;
    F.last_node_ms.assign(count, 0.0);
    for (int i = 0; i < count; ++i) F.last_node_ms[i] = 1e-6 * (double)L.hns.p[o + i];

    std::vector<int> redo;
    for (int i = 0; i < count; ++i) {
        if (L.hst.p[o + i]) {
            redo.push_back(i);
            continue;
        }
        bounds[i] = L.hb.p[o + i];
        memcpy(nodes[i].fracsol, L.hfs.p + (size_t)(o + i) * N, N * sizeof(double));
    }
    // incumbent updates in node order (updateSolution's test and update)
    for (int i = 0; i < count; ++i) {
        if (!(L.hhv.p[o + i] > Bab_LBGet())) continue;
        BabSolution bs;
        memset(&bs, 0, sizeof bs);
        memcpy(bs.X, L.hhs.p + (size_t)(o + i) * N, N * sizeof(int));
        Bab_LBUpd(L.hhv.p[o + i], &bs);
    }
    // every result of this submission has been read from L's host buffers
    --L.refs;
    if (!redo.empty()) {
        F.fallbacks += (long long)redo.size();
        std::vector<BabNode> sub(redo.size());
        std::vector<double> sb(redo.size());
        for (size_t q = 0; q < redo.size(); ++q) sub[q] = nodes[redo[q]];
        const int th = redo.size() < 16 ? (int)redo.size() : 16;
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = bqb_bound_nodes(sub.data(), (int)sub.size(), rank, th, nullptr, sb.data());
        const auto t1 = std::chrono::steady_clock::now();
        F.st_fallback_nodes += (double)redo.size();
        F.st_fallback_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
        if (rc) return rc;
        for (size_t q = 0; q < redo.size(); ++q) {
            nodes[redo[q]] = sub[q];
            bounds[redo[q]] = sb[q];
        }
    }
    return 0;
}

// The device-resident node pool's buffers (one pool per process).
struct PoolState {
    int cap = 0;
    cudaStream_t stream = nullptr;
    DevBuf<int> xf, sx, heap, pstate, host_list, status, hsol;
    DevBuf<double> ub, bound, fracsol, hval;
    DevBuf<unsigned long long> lb, node_ns, deadline;
    DevBuf<unsigned char> arena;
    HostBuf<int> hst;
    HostBuf<unsigned long long> hlb;
};

PoolState& pstate_host()
{
    static PoolState s;
    return s;
}

}  // namespace

// Best-first B&B over the open nodes `open` (priority: their upper_bound)
// with the node pool on the device (nodek_kernel in pool mode): CTAs pop,
// bound, branch and push until no node is open.  Nodes the kernel flags go
// to the host, are bounded by engines, branched there and pushed back, and
// the kernel runs again.  Returns 0, 1 when the pool is full or a lock wait
// ran out, 2 on an engine error; *created counts the node records (open
// nodes included), *evaluated the nodes bounded.
int fused_pool_bab(const std::vector<BabNode>& open, int cap, double budget_s, long long* created,
                   long long* evaluated, int* stopped)
{
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    PoolState& Q = pstate_host();
    Runtime& R = rt();
    const int N0 = SP->n, N = N0 - 1;
    if (!Q.stream) BQB_CUDA(cudaStreamCreateWithFlags(&Q.stream, cudaStreamNonBlocking));
    cudaStream_t s = Q.stream;
    if (cap < (int)open.size() + 2) cap = (int)open.size() + 2;
    Q.cap = cap;
    const size_t cN = (size_t)cap * N;
    Q.xf.ensure(cN);
    Q.sx.ensure(cN);
    Q.heap.ensure(cap);
    Q.pstate.ensure(NKQ_WORDS);
    Q.host_list.ensure(cap);
    Q.status.ensure(cap);
    Q.hsol.ensure(cN);
    Q.ub.ensure(cap);
    Q.bound.ensure(cap);
    Q.fracsol.ensure(cN);
    Q.hval.ensure(cap);
    Q.lb.ensure(1);
    Q.node_ns.ensure(cap);
    Q.deadline.ensure(1);
    int* hst = Q.hst.ensure(NKQ_WORDS);

    // the open nodes, highest priority first (a sorted array is a heap)
    std::vector<int> order(open.size());
    for (size_t i = 0; i < open.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return open[a].upper_bound > open[b].upper_bound; });
    std::vector<int> hx((size_t)open.size() * N), hs((size_t)open.size() * N), hheap(open.size());
    std::vector<double> hub(open.size()), hhv(open.size(), -1e300);
    for (size_t q = 0; q < open.size(); ++q) {
        memcpy(&hx[q * N], open[q].xfixed, N * sizeof(int));
        memcpy(&hs[q * N], open[q].sol.X, N * sizeof(int));
        hub[q] = open[q].upper_bound;
        hheap[q] = order[q];
    }
    const int m = (int)open.size();
    if (m > 0) {
        BQB_CUDA(cudaMemcpyAsync(Q.xf.p, hx.data(), hx.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        BQB_CUDA(cudaMemcpyAsync(Q.sx.p, hs.data(), hs.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        BQB_CUDA(cudaMemcpyAsync(Q.ub.p, hub.data(), m * sizeof(double), cudaMemcpyHostToDevice, s));
        BQB_CUDA(cudaMemcpyAsync(Q.hval.p, hhv.data(), m * sizeof(double), cudaMemcpyHostToDevice, s));
        BQB_CUDA(cudaMemcpyAsync(Q.heap.p, hheap.data(), m * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    for (int w = 0; w < NKQ_WORDS; ++w) hst[w] = 0;
    hst[NKQ_SIZE] = m;
    hst[NKQ_CREATED] = m;
    BQB_CUDA(cudaMemcpyAsync(Q.pstate.p, hst, NKQ_WORDS * sizeof(int), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    if (budget_s > 0) nk_deadline(Q.deadline.p, (unsigned long long)(budget_s * 1e9), s);

    // P0L on the device (the same copy the fused launches use)
    const unsigned gen = g_sp_generation.load();
    if (F.P0L_src != SP->L || F.P0N != N0 || F.P0L_gen != gen) {
        for (int q = 0; q < NK_LAUNCHES; ++q)
            if (F.run[q].refs > 0) BQB_CUDA(cudaStreamSynchronize(F.run[q].stream));
        F.P0L.ensure((size_t)N0 * N0);
        BQB_CUDA(cudaMemcpy(F.P0L.p, SP->L, (size_t)N0 * N0 * sizeof(double), cudaMemcpyHostToDevice));
        F.P0L_src = SP->L;
        F.P0N = N0;
        F.P0L_gen = gen;
    }
    if (!F.prof.p) {
        F.prof.ensure(2 * NKP_COUNT);
        BQB_CUDA(cudaMemset(F.prof.p, 0, 2 * NKP_COUNT * sizeof(unsigned long long)));
    }
    *evaluated = 0;
    *stopped = 0;
    int rc = 0;
    int made_total = m;
    while (true) {
        FusedCfg c;
        fill_cfg(c, N0, 0, 1, F.seed + 0x632BE59BD9B4E019ull * (unsigned long long)(*evaluated + 1), R.smem_optin);
        const size_t slot_bytes = nk_layout(c);
        const int slots = R.num_sms;
        Q.arena.ensure(slot_bytes * slots);
        unsigned long long* hlb = Q.hlb.ensure(1);
        hlb[0] = host_ordered(Bab_LBGet());
        BQB_CUDA(cudaMemcpyAsync(Q.lb.p, hlb, sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
        c.P0L = F.P0L.p;
        c.xfixed = Q.xf.p;
        c.solx = Q.sx.p;
        c.bound = Q.bound.p;
        c.fracsol = Q.fracsol.p;
        c.hval = Q.hval.p;
        c.hsol = Q.hsol.p;
        c.status = Q.status.p;
        c.node_ns = Q.node_ns.p;
        c.lb = Q.lb.p;
        c.ipm_stats = ipm_stats_device();
        c.prof = F.prof.p;
        c.warm_p = warm_device_params();
        c.warm_stats = c.warm_p ? warm_device_stats() : nullptr;
        c.pool = 1;
        c.pool_cap = cap;
        c.branching = params.branchingStrategy;
        c.heap = Q.heap.p;
        c.ub = Q.ub.p;
        c.pstate = Q.pstate.p;
        c.host_list = Q.host_list.p;
        c.deadline = budget_s > 0 ? Q.deadline.p : nullptr;
        c.arena = Q.arena.p;
        nk_launch(c, slots, s);
        BQB_CUDA(cudaMemcpyAsync(hst, Q.pstate.p, NKQ_WORDS * sizeof(int), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaStreamSynchronize(s));
        ++F.st_launches;
        const int made = hst[NKQ_CREATED] < cap ? hst[NKQ_CREATED] : cap;
        made_total = made;
        // heuristic improvements: the best value any node reported
        std::vector<double> hv(made);
        BQB_CUDA(cudaMemcpy(hv.data(), Q.hval.p, made * sizeof(double), cudaMemcpyDeviceToHost));
        int bi = -1;
        for (int q = 0; q < made; ++q)
            if (hv[q] > Bab_LBGet() && (bi < 0 || hv[q] > hv[bi])) bi = q;
        if (bi >= 0) {
            BabSolution bs;
            memset(&bs, 0, sizeof bs);
            BQB_CUDA(cudaMemcpy(bs.X, Q.hsol.p + (size_t)bi * N, N * sizeof(int), cudaMemcpyDeviceToHost));
            Bab_LBUpd(hv[bi], &bs);
        }
        *evaluated += hst[NKQ_EVALUATED];
        if (hst[NKQ_ERROR]) {
            set_error("bqb_solve_device", (hst[NKQ_ERROR] & 2) ? "the device node pool is full"
                                                             : "a lock wait in the node pool ran out");
            rc = 1;
            break;
        }
        if (hst[NKQ_STOPPED]) {
            *stopped = 1;
            break;
        }
        // nodes the kernel flagged: engines bound them, the host branches
        const int h = hst[NKQ_HOST];
        std::vector<int> hl(h);
        if (h > 0)
            BQB_CUDA(cudaMemcpy(hl.data(), Q.host_list.p, h * sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<BabNode> hn(h);
        std::vector<double> hb(h, 0.0);
        for (int q = 0; q < h; ++q) {
            memset(&hn[q], 0, sizeof(BabNode));
            BQB_CUDA(cudaMemcpy(hn[q].xfixed, Q.xf.p + (size_t)hl[q] * N, N * sizeof(int), cudaMemcpyDeviceToHost));
            BQB_CUDA(cudaMemcpy(hn[q].sol.X, Q.sx.p + (size_t)hl[q] * N, N * sizeof(int), cudaMemcpyDeviceToHost));
        }
        if (h > 0) {
            F.fallbacks += h;
            const int e = bqb_bound_nodes(hn.data(), h, 1, h < 16 ? h : 16, nullptr, hb.data());
            if (e) {
                rc = 2;
                break;
            }
        }
        // their children, then the open nodes left on the device
        int size = hst[NKQ_SIZE], made2 = made;
        std::vector<int> heap(size);
        std::vector<double> ubh(made2);
        if (size > 0) BQB_CUDA(cudaMemcpy(heap.data(), Q.heap.p, size * sizeof(int), cudaMemcpyDeviceToHost));
        BQB_CUDA(cudaMemcpy(ubh.data(), Q.ub.p, made2 * sizeof(double), cudaMemcpyDeviceToHost));
        bool added = false;
        for (int q = 0; q < h; ++q) {
            if (!(Bab_LBGet() + 1.0 < hb[q])) continue;
            hn[q].upper_bound = hb[q];
            const int ic = getBranchingVariable(&hn[q]);
            if (ic < 0) continue;
            for (int xic = 0; xic <= 1; ++xic) {
                if (made2 >= cap) {
                    set_error("bqb_solve_device", "the device node pool is full");
                    rc = 1;
                    break;
                }
                std::vector<int> cx(hn[q].xfixed, hn[q].xfixed + N), cs(hn[q].sol.X, hn[q].sol.X + N);
                cx[ic] = 1;
                cs[ic] = xic;
                const double nb = -1e300;
                BQB_CUDA(cudaMemcpy(Q.xf.p + (size_t)made2 * N, cx.data(), N * sizeof(int), cudaMemcpyHostToDevice));
                BQB_CUDA(cudaMemcpy(Q.sx.p + (size_t)made2 * N, cs.data(), N * sizeof(int), cudaMemcpyHostToDevice));
                BQB_CUDA(cudaMemcpy(Q.ub.p + made2, &hb[q], sizeof(double), cudaMemcpyHostToDevice));
                BQB_CUDA(cudaMemcpy(Q.hval.p + made2, &nb, sizeof(double), cudaMemcpyHostToDevice));
                ubh.push_back(hb[q]);
                // sift up in the host copy of the heap
                heap.push_back(made2);
                int i = (int)heap.size() - 1;
                while (i > 0) {
                    const int pi = (i - 1) / 2;
                    if (!(ubh[heap[pi]] < ubh[heap[i]])) break;
                    std::swap(heap[pi], heap[i]);
                    i = pi;
                }
                ++made2;
                added = true;
            }
            if (rc) break;
        }
        made_total = made2;
        if (rc) break;
        if (heap.empty()) break;
        if (added || h > 0) {
            size = (int)heap.size();
            BQB_CUDA(cudaMemcpy(Q.heap.p, heap.data(), size * sizeof(int), cudaMemcpyHostToDevice));
            for (int w = 0; w < NKQ_WORDS; ++w) hst[w] = 0;
            hst[NKQ_SIZE] = size;
            hst[NKQ_CREATED] = made2;
            BQB_CUDA(cudaMemcpy(Q.pstate.p, hst, NKQ_WORDS * sizeof(int), cudaMemcpyHostToDevice));
        } else {
            // open nodes left without a flagged node: CTAs that waited too
            // long for work left; run again
            hst[NKQ_HOST] = 0;
            hst[NKQ_EVALUATED] = 0;
            hst[NKQ_ACTIVE] = 0;
            BQB_CUDA(cudaMemcpy(Q.pstate.p, hst, NKQ_WORDS * sizeof(int), cudaMemcpyHostToDevice));
        }
    }
    *created = made_total;
    return rc;
}

// Launch every submission still waiting on the host: process_adj_matrix
// calls this before it replaces the problem they were made for.
void fused_launch_pending()
{
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    if (!launch_staged(F)) fatal("fused_launch_pending", "no free launch record");
}

}  // namespace bqb

using namespace bqb;

// Start bounding `count` nodes (see include/bqb_gpu.h).
BQB_API long long bqb_fused_submit(const BabNode* nodes, int count, int rank)
{
    if (count <= 0) return -4;
    if (!SP || !SP->L) return -2;
    Runtime& R = rt();
    if (!fused_supported(SP->n, R.smem_optin)) return -3;
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    for (int q = 0; q < NK_SUBS; ++q) {
        FusedSub& S = F.sub[(F.next_ticket + q) % NK_SUBS];
        if (S.busy) continue;
        stage(F, S, nodes, count, rank);
        // an idle GPU starts at once; otherwise the submission waits to be
        // launched together with the others submitted meanwhile
        if (!any_running(F) && !launch_staged(F)) {
            set_error("bqb_fused_submit", "no free launch record");
            S.busy = false;
            return -1;
        }
        return (long long)S.ticket;
    }
    set_error("bqb_fused_submit", "eight submissions are uncollected");
    return -1;
}

// Wait for a submission and fill bounds[i] and nodes[i].fracsol.
BQB_API int bqb_fused_collect(long long ticket, BabNode* nodes, double* bounds)
{
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    for (int q = 0; q < NK_SUBS; ++q) {
        FusedSub& S = F.sub[q];
        if (S.busy && (long long)S.ticket == ticket) return collect(F, S, nodes, bounds);
    }
    set_error("bqb_fused_collect", "unknown or already collected ticket");
    return 1;
}

// Fused bounding of `count` nodes, collected before returning.
BQB_API int bqb_bound_nodes_fused(BabNode* nodes, int count, int rank, double* bounds)
{
    if (count <= 0) return 0;
    if (!SP || !SP->L) return 1;
    if (!fused_supported(SP->n, rt().smem_optin)) return bqb_bound_nodes(nodes, count, rank, 16, nullptr, bounds);
    const long long t = bqb_fused_submit(nodes, count, rank);
    if (t < 0) return t == -1 ? 2 : 1;
    return bqb_fused_collect(t, nodes, bounds);
}

// Nodes the fused kernel handed back to an engine since the process started.
BQB_API long long bqb_fused_fallbacks(void) { return fstate().fallbacks; }

// out[5] = {collected submissions, nodes, fused kernel ms (summed over
// submissions; overlapping launches each count their own time), nodes
// bounded again by engines, their ms} since the last reset.
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

// Fused-kernel launches since the last bqb_fused_stats_reset (a launch
// carries one submission or several that waited for it).
BQB_API long long bqb_fused_launches(void)
{
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    return F.st_launches;
}

// Device milliseconds of every node of the last collected submission (as
// many as it had, at most `count`); returns how many were written.
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
    F.st_launches = 0;
    if (F.prof.p) BQB_CUDA(cudaMemset(F.prof.p, 0, 2 * NKP_COUNT * sizeof(unsigned long long)));
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

// Calls per phase of the fused kernel since the last reset (out[11], the
// phases of bqb_fused_profile; out[2] counts the heuristic runs).
BQB_API void bqb_fused_phase_calls(long long* out)
{
    FusedState& F = fstate();
    std::lock_guard<std::mutex> lock(F.mu);
    unsigned long long h[NKP_COUNT] = {};
    if (F.prof.p)
        BQB_CUDA(cudaMemcpy(h, F.prof.p + NKP_COUNT, sizeof h, cudaMemcpyDeviceToHost));
    for (int i = 0; i < NKP_COUNT; ++i) out[i] = (long long)h[i];
}
