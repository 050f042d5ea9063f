// Bounding of one B&B node with all matrices resident in HBM, in an engine.
//
// sdp_bound restates src/bounding.c:24-342 line for line in its control flow
// (the same tests, constants and parameter use); every matrix operation runs
// on the device: the basic IPM, the heuristic, the triangle separation, the
// bundle iterations (lambda_eta, fct_eval, step bookkeeping) and the
// subgradient rebuild after the cuts change.  The host keeps the cut lists
// (the reference's global arrays, or the engine's private copies) and reads
// back only scalars, the separated triangle list, X's last column
// (fracsol) and, when pentagonal / heptagonal separation runs, X itself.
// Everything runs on the engine's stream, so engines bound nodes
// concurrently.
#include <math.h>
#include <string.h>

#include <chrono>
#include <mutex>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "internal.h"
#include "ipm.cuh"
#include "node.h"
#include "separation.h"

extern "C" {
double Bab_LBGet(void);
int updateSolution(int* x);
double getFixedValue(BabNode* node, Problem* SP_);
extern double diff;
}

namespace bqb {

std::atomic<bqb_heuristic_fn> g_heuristic_hook{nullptr};
std::atomic<long long> g_heuristic_runs{0};
std::atomic<long long> g_bundle_iters{0};

// Root effort: with it on, a node bounded with rank 0 (the root) runs the
// outer loop of SDPbound to max_outer_iter + extra_iter rounds unless it is
// pruned, skipping the two early give-up tests of src/bounding.c:203-214.
// The bound stays a valid bound (the loop only runs longer); the reference
// has no such switch, so it is off unless the caller turns it on.
std::atomic<int> g_root_effort{0};

// Parent start: with it on, every node exports its final cuts (triangle,
// pentagonal, heptagonal; original vertex numbers) and multipliers, and a
// node bounded with its parent's cuts (a B&B driver sets Engine::parent)
// starts from them: the parent's cuts that avoid the child's fixed vertices
// join the child's first cut list with the parent's multipliers, and that
// start is evaluated once (one IPM) and kept when its dual value is below the
// plain start's, as the learned warm start's proposal is.  Every cut of the
// parent that avoids the fixed vertices is valid for the child, and any
// multipliers >= 0 give a valid bound.  Off unless the caller turns it on; a
// loaded warm-start model takes precedence.
std::atomic<int> g_parent_start{0};

// Bound certificates (off by default): with them on, every node's final
// bound B = F(gamma) + fixed value is certified in FP64 -- one more IPM at
// the final multipliers gamma gives y, and sdp_certificate an upper bound
// on the basic SDP value of L - B^T(gamma) from it -- and the excess of the
// certified bound over B is recorded (B itself is what the node returns).
std::atomic<int> g_cert_on{0};
std::mutex g_cert_mu;
struct CertStats {
    long long nodes = 0, failed = 0;
    double max_rel = 0.0, sum_rel = 0.0, max_mismatch = 0.0, max_shift = 0.0;
} g_cert;

// Trace of SDPbound's outer loop: one row of BQB_TRACE_COLS values per
// round while tracing is on (inspection only).
constexpr int BQB_TRACE_COLS = 9;
std::atomic<int> g_trace_on{0};
std::mutex g_trace_mu;
std::vector<double> g_trace;
std::atomic<long long> g_trace_node{0};

// Time by phase of sdp_bound on every engine (off by default; for
// profiling).  With it on, each phase boundary synchronises the engine's
// stream and adds the host time since the previous boundary to the phase
// that ended, so the parts sum to the bounding time (the synchronisations
// make it a little slower than without).
enum EngPhase : int {
    EP_IPM,          // the IPM calls (basic bound, fct_eval's, proposals)
    EP_LAMBDA,       // lambda_eta
    EP_OPBT,         // L0 = L - B^T(gamma)
    EP_BUNDLE,       // op_B of the new element, the bundle step and X combination
    EP_HEUR,         // the heuristic
    EP_TRI,          // triangle separation and cut-list update
    EP_KGON,         // pentagonal and heptagonal separation (X copy included)
    EP_REBUILD,      // cut upload, subgradient rebuild, state reads
    EP_TOTAL,        // whole sdp_bound calls
    EP_UPLOAD,       // (part of the rest) cut upload: records, op_B^T index, buffer sizes
    EP_FRAC,         // (part of the rest) X's last column for fracsol
    EP_ALLOC,        // (part of the rest) bundle capacity growth
    EP_WORDS
};
std::atomic<int> g_eprof_on{0};
std::atomic<long long> g_eprof_ns[EP_WORDS];

struct PhaseClock {
    cudaStream_t s;
    bool on;
    std::chrono::steady_clock::time_point t;
    explicit PhaseClock(cudaStream_t st) : s(st), on(g_eprof_on.load() != 0), t(std::chrono::steady_clock::now()) {}
    void mark(int phase)
    {
        if (!on) return;
        BQB_CUDA(cudaStreamSynchronize(s));
        const auto now = std::chrono::steady_clock::now();
        g_eprof_ns[phase].fetch_add(std::chrono::duration_cast<std::chrono::nanoseconds>(now - t).count());
        t = now;
    }
    // restart the clock without charging the time since the last boundary
    void skip()
    {
        if (on) t = std::chrono::steady_clock::now();
    }
};

// Adds a whole call's time on return (with profiling on).
struct CallClock {
    bool on;
    std::chrono::steady_clock::time_point t0;
    CallClock() : on(g_eprof_on.load() != 0), t0(std::chrono::steady_clock::now()) {}
    ~CallClock()
    {
        if (on)
            g_eprof_ns[EP_TOTAL].fetch_add(
                std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count());
    }
};

void upload_cuts(Engine& E, const HostState& H, const Problem* P)
{
    std::vector<CutRec> rec = pack_cuts(H.cuts, P->NIneq, H.pcuts, P->NPentIneq, H.hcuts, P->NHeptaIneq);
    E.nd.cuts.upload(rec, P->NIneq, P->NPentIneq, P->NHeptaIneq, E.stream);
    E.nd.b.ensure_m(E.nd.cuts.m, E.stream);
}

double tri_update_dev(Engine& E, HostState& H, Problem* P, const double* y, int* added, int* subtracted)
{
    const int kept = tri_purge(H.cuts, P->NIneq, y);
    *subtracted = P->NIneq - kept;
    P->NIneq = kept;
    int size = 0;
    const double mx =
        trisep_device(E.tri, E.nd.X.p, P->n, params.TriIneq, params.violated_TriIneq, &size, E.stream);
    *added = tri_append(H.cuts, kept, E.tri.hlist.p, size);
    P->NIneq += *added;
    return mx;
}

static void fetch_state(NodeDev& nd, cudaStream_t s)
{
    BQB_CUDA(cudaMemcpyAsync(nd.hs.p, nd.b.dstate.p, BD_WORDS * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(nd.hi.p, nd.b.istate.p, BI_WORDS * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    const int err = nd.hi.p[BI_ERR];
    if (err & 1) fatal("bundle_method", "Bundle size too large! Adjust MaxBundle");
    if (err & 2) fatal("solve_lambda", "Problem in solving linear system");
    if (err & 4) fatal("ipm_mc_pk", "Problem with Cholesky factorization or linear system");
    if (err & 8) fatal("bundle_method", "no free bundle slot");
}

double bundle_iterations(Engine& E, int bdl_iter, double* t)
{
    NodeDev& nd = E.nd;
    BundleDev& b = nd.b;
    cudaStream_t s = E.stream;
    const int n = nd.n;
    const size_t nn = (size_t)n * n;
    PhaseClock pc(s);
    nd.hs.ensure(8);
    nd.hi.ensure(8);
    // k grows by at most one per iteration
    BQB_CUDA(cudaMemcpyAsync(nd.hi.p, b.istate.p, BI_WORDS * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    const int k = nd.hi.p[BI_K];
    pc.mark(EP_REBUILD);
    b.ensure_cap(k + bdl_iter + 2, n, s);
    pc.mark(EP_ALLOC);
    nd.hi.p[BI_CAP] = b.cap;
    BQB_CUDA(cudaMemcpyAsync(b.istate.p + BI_CAP, nd.hi.p + BI_CAP, sizeof(int), cudaMemcpyHostToDevice, s));
    nd.hs.p[0] = *t;
    BQB_CUDA(cudaMemcpyAsync(b.dstate.p + BD_T, nd.hs.p, sizeof(double), cudaMemcpyHostToDevice, s));
    g_bundle_iters.fetch_add(bdl_iter);
    pc.mark(EP_REBUILD);
    for (int it = 0; it < bdl_iter; ++it) {
        lambda_eta_launch(b, nullptr, s);
        pc.mark(EP_LAMBDA);
        BQB_CUDA(cudaMemcpyAsync(nd.L0.p, nd.L.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
        if (nd.cuts.m > 0) opBt_launch(nd.cuts, nd.L0.p, n, b.gtest.p, s);
        pc.mark(EP_OPBT);
        ipm_device(E.ipm_ws, nd.L0.p, b.Xb.p, n, nd.out.p, s, b.istate.p + BI_NEXT);
        pc.mark(EP_IPM);
        if (nd.cuts.m > 0)
            opB_launch(nd.cuts, b.Xb.p, nn, b.istate.p + BI_NEXT, 1, n, b.G.p, b.ldg, true, s);
        bundle_step_launch(b, nd.out.p, nd.L.p, s);
        bundle_xcomb_launch(b, nd.X.p, s);
        pc.mark(EP_BUNDLE);
    }
    fetch_state(nd, s);
    pc.mark(EP_REBUILD);
    *t = nd.hs.p[BD_T];
    return nd.hs.p[BD_F];
}

// SDPbound (src/bounding.c:24-342) in engine E.
double sdp_bound(Engine& E, BabNode* node, Problem* SP_, Problem* PP_, int rank)
{
    cudaStream_t s = E.stream;
    NodeDev& nd = E.nd;
    HostState H = E.host();
    const int n = PP_->n;
    CallClock call_clock;
    PhaseClock pc(s);
    // (counted while it runs: concurrent large nodes share the GPU's CTAs)
    struct LargeShare {
        bool on;
        explicit LargeShare(bool o) : on(o)
        {
            if (on) g_large_share.fetch_add(1);
        }
        ~LargeShare()
        {
            if (on) g_large_share.fetch_sub(1);
        }
    } large_share(n > IPM_REG_NMAX);
    E.final_cuts.reset();
    const int N0 = SP_->n;
    const int NB = N0 - 1;   // BabPbSize
    const size_t nn = (size_t)n * n;
    nd.n = n;
    nd.hs.ensure(8);
    nd.hi.ensure(8);

    double* dL = nd.L.ensure(nn);
    nd.L0.ensure(nn);
    double* dX = nd.X.ensure(nn);
    double* dout = nd.out.ensure(4);
    // PP->L may be host or device memory (unified addressing decides)
    BQB_CUDA(cudaMemcpyAsync(dL, PP_->L, nn * sizeof(double), cudaMemcpyDefault, s));
    const unsigned gen = g_sp_generation.load();
    if (nd.P0L_src != SP_->L || nd.P0N != N0 || nd.P0L_gen != gen) {
        nd.P0L.ensure((size_t)N0 * N0);
        BQB_CUDA(cudaMemcpyAsync(nd.P0L.p, SP_->L, (size_t)N0 * N0 * sizeof(double), cudaMemcpyHostToDevice, s));
        nd.P0L_src = SP_->L;
        nd.P0N = N0;
        nd.P0L_gen = gen;
    }
    auto upload = [&]() {
        pc.mark(EP_REBUILD);
        upload_cuts(E, H, PP_);
        pc.mark(EP_UPLOAD);
    };
    // A node that branches without running its bundle (the use_diff rule, or
    // no violated triangle) has no final cuts of its own: its children get
    // its parent's (original vertex numbers, so they stay valid for every
    // descendant that keeps their vertices; the child's mapping drops the
    // others), so parent-informed starts and recorded parent features reach
    // past it.
    auto pass_parent_cuts = [&]() {
        if ((warm_active() || warm_recording() || g_parent_start.load() != 0) && E.parent)
            E.final_cuts = std::make_shared<ParentCuts>(*E.parent);
    };
    // the certificate of the bound B = fval + fixed value at the current
    // multipliers (none: the basic bound)
    auto certify = [&](bool with_cuts, double fval, double fixed) {
        if (!g_cert_on.load()) return;
        const int m = with_cuts ? nd.cuts.m : 0;
        double* L0 = nd.L0.ensure(nn);
        BQB_CUDA(cudaMemcpyAsync(L0, dL, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
        std::vector<double> g(m > 0 ? m : 1);
        if (m > 0) {
            opBt_launch(nd.cuts, L0, n, nd.b.gam.p, s);
            BQB_CUDA(cudaMemcpyAsync(g.data(), nd.b.gam.p, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        double* v = E.cert_v.ensure((size_t)n + 8);
        ipm_device(E.ipm_ws, L0, E.warm.X.ensure(nn), n, v + n, s, nullptr, v);
        sdp_certificate(E.cert_ws, L0, v, n, v + n + 4, s);
        double h[8];
        BQB_CUDA(cudaMemcpyAsync(h, v + n, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaStreamSynchronize(s));
        // sum of the multipliers, with its rounding bounded
        double sg = 0.0, sa = 0.0;
        for (int i = 0; i < m; ++i) {
            sg += g[i];
            sa += fabs(g[i]);
        }
        const double sg_hi = sg + (m + 1) * 0x1p-53 * sa;
        const double B = fval + fixed;
        const double Bc = h[4] + sg_hi + fixed;
        const double scale = fabs(B) > 1.0 ? fabs(B) : 1.0;
        std::lock_guard<std::mutex> lk(g_cert_mu);
        ++g_cert.nodes;
        if ((int)h[7] != 0 || (int)h[2] != IPM_OK) {
            ++g_cert.failed;
            return;
        }
        const double rel = (Bc - B) / scale;
        g_cert.max_rel = rel > g_cert.max_rel ? rel : g_cert.max_rel;
        g_cert.sum_rel += rel;
        const double mis = fabs(h[0] - (fval - sg)) / scale;   // the rerun's phi against F - sum(gamma)
        g_cert.max_mismatch = mis > g_cert.max_mismatch ? mis : g_cert.max_mismatch;
        g_cert.max_shift = h[6] > g_cert.max_shift ? h[6] : g_cert.max_shift;
    };
    std::vector<int> x(NB > 0 ? NB : 1);
    std::vector<double> col(n);
    auto store_fracsol = [&]() {
        pc.mark(EP_REBUILD);
        BQB_CUDA(cudaMemcpyAsync(col.data(), dX + (size_t)(n - 1) * n, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaStreamSynchronize(s));
        int index = 0;
        for (int i = 0; i < NB; ++i) {
            if (node->xfixed[i])
                node->fracsol[i] = (double)node->sol.X[i];
            else
                node->fracsol[i] = 0.5 * (col[index++] + 1.0);
        }
        pc.mark(EP_FRAC);
    };
    std::vector<double> hostL;
    auto heuristic = [&]() {
        pc.mark(EP_REBUILD);
        for (int i = 0; i < NB; ++i) x[i] = node->xfixed[i] ? node->sol.X[i] : 0;
        g_heuristic_runs.fetch_add(1);
        bqb_heuristic_fn hook = g_heuristic_hook.load();
        if (hook && E.is_default) {
            // runHeuristic's plug-in point (src/heuristic.c:11-17): the caller's
            // function gets host P0_L, P_L and the node's arrays, and the
            // global X holds the node's X (runHeuristic_unpacked reads it)
            hostL.resize(nn);
            BQB_CUDA(cudaMemcpyAsync(H.X, dX, nn * sizeof(double), cudaMemcpyDeviceToHost, s));
            BQB_CUDA(cudaMemcpyAsync(hostL.data(), dL, nn * sizeof(double), cudaMemcpyDeviceToHost, s));
            BQB_CUDA(cudaStreamSynchronize(s));
            hook(SP_->L, N0, hostL.data(), n, node->xfixed, node->sol.X, x.data());
        } else {
            heuristic_device(E.heur, E.rng, dX, dL, n, nd.P0L.p, N0, node->xfixed, node->sol.X, x.data(), s,
                             E.is_default ? 0 : gw_hyperplanes());
        }
        updateSolution(x.data());
        pc.mark(EP_HEUR);
    };

    int bdl_iter = params.init_bundle_iter;
    const double fixedvalue = getFixedValue(node, SP_);
    PP_->NIneq = 0;
    PP_->NPentIneq = 0;
    PP_->NHeptaIneq = 0;
    int tri_add = 0, tri_sub = 0, pent_add = 0, pent_sub = 0, hept_add = 0, hept_sub = 0;
    double viol3 = 0.0, viol5 = 0.0;
    double& f = *H.f;

    // basic SDP relaxation
    pc.mark(EP_REBUILD);
    ipm_device(E.ipm_ws, dL, dX, n, dout, s);
    BQB_CUDA(cudaMemcpyAsync(nd.hs.p, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    pc.mark(EP_IPM);
    check_ipm_status_host(nd.hs.p);
    f = nd.hs.p[0];
    const double basic_bound = f + fixedvalue;
    store_fracsol();
    heuristic();

    double bound = f + fixedvalue;
    if (bound < Bab_LBGet() + 1.0) {
        certify(false, f, fixedvalue);
        return bound;
    }
    if (params.use_diff && rank != 0 && bound > Bab_LBGet() + diff + 1.0) {
        certify(false, f, fixedvalue);
        pass_parent_cuts();
        return bound;
    }

    pc.mark(EP_REBUILD);
    viol3 = tri_update_dev(E, H, PP_, H.dual_gamma, &tri_add, &tri_sub);
    pc.mark(EP_TRI);
    // No violated triangle inequality (X is a cut matrix up to the
    // tolerance): the bundle would start from t = .../0 with no cuts, where
    // the reference's BLAS calls reject m = 0 (src/bounding.c:122-131,
    // src/bundle.c:63, 315) and its result is undefined.  The basic bound is
    // the node's bound, returned as the reference's early exits return it.
    if (PP_->NIneq == 0) {
        certify(false, f, fixedvalue);
        pass_parent_cuts();
        return bound;
    }
    for (int i = 0; i < PP_->NIneq; ++i) H.dual_gamma[i] = H.cuts[i].y;
    double t = 0.5 * (bound - Bab_LBGet()) / (PP_->NIneq * viol3 * viol3);

    // bundle init: X_bundle(0) = X, G(:,0) = 1 - B(X), F(0) = <L,X>, bundle = 1
    upload();

    // Learned warm start (off unless a model is loaded and switched on):
    // evaluate the proposed multipliers once (L0 = L - B^T(gamma_w), one
    // IPM) and start the bundle there when their dual value is below the
    // plain start's (gamma = 0, where the dual value is the basic bound f).
    // Any gamma >= 0 gives a valid bound; the bundle then runs to its own
    // stopping rules.  With the parent's final cuts (a B&B driver sets
    // E.parent), every cut gets the parent's multiplier as a feature, and
    // the parent's cuts that the child's separation did not find are
    // candidates: those whose predicted multiplier reaches
    // WARM_SHORTLIST_MIN join the first cut list (the shortlist); when the
    // proposal is rejected the list goes back to the child's own cuts.
    // Recording keeps the first cut list's features and, at the end, the
    // multipliers those cuts finish with (training pairs); while recording
    // without a model every parent candidate joins the list, so the pairs
    // say which of them the bundle keeps.
    const bool warm_on = warm_active();
    const bool warm_rec = warm_recording();
    const bool pstart_on = g_parent_start.load() != 0;
    const bool pstart = pstart_on && !warm_on && !warm_rec && E.parent != nullptr;
    bool inherited = false;   // this node's list holds its parent's k-gonal cuts
    std::vector<float> warm_feats;
    std::vector<Triangle_Inequality> warm_first;
    double warm_scale = 1.0;
    std::vector<int> orig;   // subproblem vertex -> original vertex
    const int n_own = PP_->NIneq;
    if (warm_on || warm_rec || pstart_on) {
        orig.resize(n);
        int idx = 0;
        for (int i = 0; i < NB && idx < n - 1; ++i)
            if (!node->xfixed[i]) orig[idx++] = i;
        orig[n - 1] = NB;
    }
    std::vector<double> pg;
    if ((warm_on || warm_rec) && E.parent) {
        const ParentCuts& PC = *E.parent;
        pg.assign(n_own, -1.0);
        std::unordered_map<uint64_t, int> have;
        have.reserve((size_t)n_own * 2 + 16);
        for (int c = 0; c < n_own; ++c) {
            const Triangle_Inequality& t = H.cuts[c];
            const uint64_t key = orig_cut_key(t.type, orig[t.i], orig[t.j], orig[t.k]);
            have[key] = c;
            auto it = PC.index.find(key);
            if (it != PC.index.end()) pg[c] = it->second;
        }
        std::vector<int> cidx(NB + 1, -1);
        for (int q = 0; q < n; ++q) cidx[orig[q]] = q;
        int m = n_own;
        for (size_t c = 0; c < PC.key.size() && m < BQB_MAX_TRI_INEQ; ++c) {
            if (!(PC.gam[c] > 0.0) || have.count(PC.key[c])) continue;
            const int type = (int)(PC.key[c] >> 48);
            const int a = cidx[(PC.key[c] >> 32) & 0xFFFF], bb = cidx[(PC.key[c] >> 16) & 0xFFFF],
                      cc = cidx[PC.key[c] & 0xFFFF];
            if (a < 0 || bb < 0 || cc < 0) continue;   // a vertex the child fixed
            Triangle_Inequality& t = H.cuts[m++];
            t.type = type;
            t.i = a;
            t.j = bb;
            t.k = cc;
            t.value = NAN;   // evaluated at X by the feature kernel
            t.y = 0.0;
            pg.push_back(PC.gam[c]);
        }
        PP_->NIneq = m;
    }
    std::vector<float> feats_all;   // (recording) the features of every candidate of the first list
    std::vector<int> rows;          // (recording) first list -> row of feats_all
    if (warm_on || warm_rec) {
        warm_features(E.warm, H.cuts, PP_->NIneq, dX, dL, n, viol3, bound - Bab_LBGet(), s,
                      pg.empty() ? nullptr : pg.data());
        if (warm_rec) warm_scale = warm_fetch_features(E.warm, PP_->NIneq, feats_all, s);
        for (int c = 0; c < PP_->NIneq; ++c) rows.push_back(c);
    }
    for (int c = n_own; c < PP_->NIneq; ++c) H.cuts[c].value = 0.0;
    if (warm_on) {
        const int mall = PP_->NIneq;
        warm_infer(E.warm, mall, s);
        double* hg = E.warm.hgam.ensure(mall);
        BQB_CUDA(cudaMemcpyAsync(hg, E.warm.gam.p, (size_t)mall * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaMemcpyAsync(E.warm.hscale.ensure(1), E.warm.scale.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaStreamSynchronize(s));
        const double sc = E.warm.hscale.p[0];
        // the shortlist: candidates whose predicted multiplier is large enough
        std::vector<double> prop(hg, hg + n_own);
        rows.resize(n_own);
        int m = n_own;
        for (int c = n_own; c < mall; ++c)
            if (hg[c] >= WARM_SHORTLIST_MIN * sc) {
                H.cuts[m] = H.cuts[c];
                prop.push_back(hg[c]);
                rows.push_back(c);
                ++m;
            }
        PP_->NIneq = m;
        upload();
        BQB_CUDA(cudaMemcpyAsync(E.warm.gam.p, prop.data(), (size_t)m * sizeof(double), cudaMemcpyHostToDevice, s));
        BQB_CUDA(cudaMemcpyAsync(nd.L0.p, dL, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
        opBt_launch(nd.cuts, nd.L0.p, n, E.warm.gam.p, s);
        double* Xw = E.warm.X.ensure(nn);
        pc.mark(EP_REBUILD);
        ipm_device(E.ipm_ws, nd.L0.p, Xw, n, dout, s);
        BQB_CUDA(cudaMemcpyAsync(nd.hs.p, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaStreamSynchronize(s));
        pc.mark(EP_IPM);
        double fw = nd.hs.p[0];
        for (int i = 0; i < m; ++i) fw += prop[i];
        const bool keep = (int)nd.hs.p[2] == IPM_OK && fw < f;
        warm_count(keep);
        if (keep) {
            for (int i = 0; i < m; ++i) H.dual_gamma[i] = prop[i];
            BQB_CUDA(cudaMemcpyAsync(dX, Xw, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
            f = fw;
        } else if (m != n_own) {
            PP_->NIneq = n_own;   // back to the child's own cuts
            rows.resize(n_own);
            upload();
        }
        if (!keep)
            for (int i = 0; i < PP_->NIneq; ++i) H.dual_gamma[i] = 0.0;
    } else {
        if (PP_->NIneq != n_own) {
            for (int i = n_own; i < PP_->NIneq; ++i) H.dual_gamma[i] = 0.0;
            upload();
        }
    }
    if (pstart) {
        const ParentCuts& PC = *E.parent;
        std::vector<int> cidx(NB + 1, -1);
        for (int q = 0; q < n; ++q) cidx[orig[q]] = q;
        std::unordered_set<uint64_t> have;
        have.reserve((size_t)n_own * 2 + 16);
        std::vector<double> prop;
        prop.reserve((size_t)n_own + PC.key.size() + PC.pent.size() + PC.hept.size());
        for (int c = 0; c < n_own; ++c) {
            const Triangle_Inequality& t = H.cuts[c];
            have.insert(orig_cut_key(t.type, orig[t.i], orig[t.j], orig[t.k]));
            prop.push_back(H.cuts[c].y);
        }
        int m = n_own;
        for (size_t c = 0; c < PC.key.size() && m < BQB_MAX_TRI_INEQ; ++c) {
            if (!(PC.gam[c] > 0.0) || have.count(PC.key[c])) continue;
            const int a = cidx[(PC.key[c] >> 32) & 0xFFFF], bb = cidx[(PC.key[c] >> 16) & 0xFFFF],
                      cc = cidx[PC.key[c] & 0xFFFF];
            if (a < 0 || bb < 0 || cc < 0) continue;   // a vertex the child fixed
            Triangle_Inequality& t = H.cuts[m++];
            t.type = (int)(PC.key[c] >> 48);
            t.i = a;
            t.j = bb;
            t.k = cc;
            t.value = 0.0;
            t.y = PC.gam[c];
            prop.push_back(PC.gam[c]);
        }
        // k-gonal cuts: every vertex must survive in the child
        auto map_kgon = [&](const ParentKgon& q, int k, int* perm) {
            for (int a = 0; a < k; ++a) {
                perm[a] = cidx[q.v[a]];
                if (perm[a] < 0) return false;
            }
            return true;
        };
        int np = 0, nh = 0;
        for (const ParentKgon& q : PC.pent) {
            if (np >= BQB_MAX_PENT_INEQ) break;
            Pentagonal_Inequality& c = H.pcuts[np];
            if (!(q.gam > 0.0) || !map_kgon(q, 5, c.permutation)) continue;
            c.type = q.type;
            c.value = 0.0;
            c.y = q.gam;
            ++np;
        }
        for (const ParentKgon& q : PC.hept) {
            if (nh >= BQB_MAX_HEPTA_INEQ) break;
            Heptagonal_Inequality& c = H.hcuts[nh];
            if (!(q.gam > 0.0) || !map_kgon(q, 7, c.permutation)) continue;
            c.type = q.type;
            c.value = 0.0;
            c.y = q.gam;
            ++nh;
        }
        for (int i = 0; i < np; ++i) prop.push_back(H.pcuts[i].y);
        for (int i = 0; i < nh; ++i) prop.push_back(H.hcuts[i].y);
        if (m > n_own || np > 0 || nh > 0) {
            PP_->NIneq = m;
            PP_->NPentIneq = np;
            PP_->NHeptaIneq = nh;
            upload();
            const int mt = nd.cuts.m;
            double* gp = nd.b.gam.p;
            BQB_CUDA(cudaMemcpyAsync(gp, prop.data(), (size_t)mt * sizeof(double), cudaMemcpyHostToDevice, s));
            BQB_CUDA(cudaMemcpyAsync(nd.L0.p, dL, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
            opBt_launch(nd.cuts, nd.L0.p, n, gp, s);
            double* Xw = E.warm.X.ensure(nn);
            pc.mark(EP_REBUILD);
            ipm_device(E.ipm_ws, nd.L0.p, Xw, n, dout, s);
            BQB_CUDA(cudaMemcpyAsync(nd.hs.p, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
            BQB_CUDA(cudaStreamSynchronize(s));
            pc.mark(EP_IPM);
            double fw = nd.hs.p[0];
            for (int i = 0; i < mt; ++i) fw += prop[i];
            const bool keep = (int)nd.hs.p[2] == IPM_OK && fw < f;
            warm_count(keep);
            if (keep) {
                for (int i = 0; i < mt; ++i) H.dual_gamma[i] = prop[i];
                BQB_CUDA(cudaMemcpyAsync(dX, Xw, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
                f = fw;
                inherited = true;
            } else {
                PP_->NIneq = n_own;   // back to the child's own cuts
                PP_->NPentIneq = 0;
                PP_->NHeptaIneq = 0;
                upload();
            }
        }
    }
    if (warm_rec) {
        // the features of the first list as it stands (own cuts, then the
        // shortlisted or, without a model, all parent candidates)
        warm_feats.resize(rows.size() * WARM_F);
        for (size_t r = 0; r < rows.size(); ++r)
            memcpy(&warm_feats[r * WARM_F], &feats_all[(size_t)rows[r] * WARM_F], WARM_F * sizeof(float));
        warm_first.assign(H.cuts, H.cuts + PP_->NIneq);
    }
    BundleDev& b = nd.b;
    pc.mark(EP_REBUILD);
    b.ensure_cap(1 + bdl_iter + 2, n, s);
    pc.mark(EP_ALLOC);
    const int m0 = nd.cuts.m;
    BQB_CUDA(cudaMemcpyAsync(b.gam.p, H.dual_gamma, (size_t)m0 * sizeof(double), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemcpyAsync(b.Xb.p, dX, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
    opB_launch(nd.cuts, b.Xb.p, nn, nullptr, 1, n, b.G.p, b.ldg, true, s);
    {
        int* hi = nd.hi.p;
        for (int q = 0; q < 8; ++q) hi[q] = 0;
        hi[BI_K] = 0;        // F(0) is written at position 0 below, then K = 1
        hi[BI_NEXT] = 0;
        hi[BI_CAP] = b.cap;
        BQB_CUDA(cudaMemcpyAsync(b.istate.p, hi, BI_WORDS * sizeof(int), cudaMemcpyHostToDevice, s));
        bundle_fval_launch(b, dL, b.istate.p + BI_NEXT, b.istate.p + BI_K, s);
        bundle_append_launch(b, s);
        nd.hs.p[BD_F] = f;
        nd.hs.p[BD_T] = t;
        nd.hs.p[BD_FTEST] = 0.0;
        nd.hs.p[BD_DEL] = 0.0;
        BQB_CUDA(cudaMemcpyAsync(b.dstate.p, nd.hs.p, BD_WORDS * sizeof(double), cudaMemcpyHostToDevice, s));
        BQB_CUDA(cudaStreamSynchronize(s));
    }

    int count = 0;
    bool done = false, prune = false, giveup = false;
    const bool root_effort = rank == 0 && g_root_effort.load() != 0;
    const long long trace_id = g_trace_on.load() ? g_trace_node.fetch_add(1) : -1;
    const auto trace_t0 = std::chrono::steady_clock::now();
    while (!done) {
        ++count;
        const double oldf = f;
        pc.mark(EP_REBUILD);
        f = bundle_iterations(E, bdl_iter, &t);
        pc.skip();
        bound = f + fixedvalue;
        prune = bound < Bab_LBGet() + 1.0;
        if (!prune) {
            heuristic();
            prune = bound < Bab_LBGet() + 1.0;
        }
        const double gap = bound - Bab_LBGet();
        if (!root_effort) {
            if (count == params.triag_iter + params.pent_iter + params.hept_iter)
                if (gap - 1.0 > (oldf - f) * (params.max_outer_iter - count)) giveup = true;
            if (count == params.max_outer_iter)
                if (gap - 1.0 > (oldf - f) * params.extra_iter) giveup = true;
        }
        if (count == params.max_outer_iter + params.extra_iter) giveup = true;

        if (!prune && !giveup) {
            const int triag = PP_->NIneq;
            const int penta = PP_->NPentIneq;
            const int m = PP_->NIneq + PP_->NPentIneq + PP_->NHeptaIneq;
            BQB_CUDA(cudaMemcpyAsync(H.dual_gamma, b.gam.p, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, s));
            BQB_CUDA(cudaStreamSynchronize(s));
            pc.mark(EP_REBUILD);
            viol3 = tri_update_dev(E, H, PP_, H.dual_gamma, &tri_add, &tri_sub);
            pc.mark(EP_TRI);
            const bool do_pent = params.include_Pent && (count > params.triag_iter || viol3 < 0.2);
            const bool do_hept = params.include_Hepta && ((count > params.triag_iter + params.pent_iter) ||
                                                          (viol3 < 0.2 && (1 - viol5 < 0.4)));
            if (inherited) {
                // inherited k-gonal cuts carry the bundle's current
                // multipliers into rounds that do not separate them
                if (!do_pent)
                    for (int i = 0; i < penta; ++i) H.pcuts[i].y = H.dual_gamma[triag + i];
                if (!do_hept)
                    for (int i = 0; i < PP_->NHeptaIneq; ++i) H.hcuts[i].y = H.dual_gamma[triag + penta + i];
            }
            // the default engine anneals on the host from the rand() stream
            // (the reference's cuts); extra engines run the chains on the GPU
            if ((do_pent || params.include_Hepta) && E.is_default) {
                BQB_CUDA(cudaMemcpyAsync(H.X, dX, nn * sizeof(double), cudaMemcpyDeviceToHost, s));
                BQB_CUDA(cudaStreamSynchronize(s));
            }
            if (do_pent)
                viol5 = E.is_default ? pent_update(H, PP_, H.dual_gamma, &pent_add, &pent_sub, triag, E.rng)
                                     : pent_update_dev(E, H, PP_, H.dual_gamma, &pent_add, &pent_sub, triag);
            if (do_hept) {
                if (E.is_default)
                    hept_update(H, PP_, H.dual_gamma, &hept_add, &hept_sub, triag + penta, E.rng);
                else
                    hept_update_dev(E, H, PP_, H.dual_gamma, &hept_add, &hept_sub, triag + penta);
            }
            pc.mark(EP_KGON);
        } else {
            tri_add = tri_sub = pent_add = pent_sub = hept_add = hept_sub = 0;
        }
        // no cuts left: the bundle cannot move (the reference's bundle
        // calls BLAS with m = 0 there, which is undefined); stop here
        done = prune || giveup || PP_->NIneq + PP_->NPentIneq + PP_->NHeptaIneq == 0;
        store_fracsol();
        if (trace_id >= 0) {
            const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - trace_t0).count();
            const double row[BQB_TRACE_COLS] = {(double)trace_id, (double)rank,  (double)count,
                                                bound,            Bab_LBGet(),   (double)PP_->NIneq,
                                                (double)PP_->NPentIneq, (double)PP_->NHeptaIneq, secs};
            std::lock_guard<std::mutex> g(g_trace_mu);
            g_trace.insert(g_trace.end(), row, row + BQB_TRACE_COLS);
        }

        if (!done) {
            for (int i = 0; i < PP_->NIneq; ++i) H.dual_gamma[i] = H.cuts[i].y;
            for (int i = 0; i < PP_->NPentIneq; ++i) H.dual_gamma[i + PP_->NIneq] = H.pcuts[i].y;
            for (int i = 0; i < PP_->NHeptaIneq; ++i)
                H.dual_gamma[i + PP_->NIneq + PP_->NPentIneq] = H.hcuts[i].y;
            upload();
            const int m = nd.cuts.m;
            BQB_CUDA(cudaMemcpyAsync(b.gam.p, H.dual_gamma, (size_t)m * sizeof(double), cudaMemcpyHostToDevice, s));
            // current bundle size (host copy) for capacity and the G rebuild
            BQB_CUDA(cudaMemcpyAsync(nd.hi.p, b.istate.p, BI_WORDS * sizeof(int), cudaMemcpyDeviceToHost, s));
            BQB_CUDA(cudaStreamSynchronize(s));
            const int k = nd.hi.p[BI_K];
            pc.mark(EP_REBUILD);
            b.ensure_cap(k + 2 + bdl_iter + 2, n, s);
            pc.mark(EP_ALLOC);
            nd.hi.p[BI_CAP] = b.cap;
            BQB_CUDA(cudaMemcpyAsync(b.istate.p + BI_CAP, nd.hi.p + BI_CAP, sizeof(int), cudaMemcpyHostToDevice, s));
            // fct_eval(PP, dual_gamma, X_test, g) into the free slot
            BQB_CUDA(cudaMemcpyAsync(nd.L0.p, dL, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
            if (m > 0) opBt_launch(nd.cuts, nd.L0.p, n, b.gam.p, s);
            pc.mark(EP_REBUILD);
            ipm_device(E.ipm_ws, nd.L0.p, b.Xb.p, n, dout, s, b.istate.p + BI_NEXT);
            pc.mark(EP_IPM);
            // G(:, i) = 1 - B(X_bundle(i)) for the bundle, then g for the new element
            opB_launch(nd.cuts, b.Xb.p, nn, b.slot.p, k, n, b.G.p, b.ldg, true, s);
            opB_launch(nd.cuts, b.Xb.p, nn, b.istate.p + BI_NEXT, 1, n, b.G.p, b.ldg, true, s);
            bundle_fval_launch(b, dL, b.istate.p + BI_NEXT, b.istate.p + BI_K, s);
            bundle_append_launch(b, s);
            BQB_CUDA(cudaMemcpyAsync(nd.hs.p, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
            BQB_CUDA(cudaMemcpyAsync(nd.hi.p, b.istate.p, BI_WORDS * sizeof(int), cudaMemcpyDeviceToHost, s));
            BQB_CUDA(cudaStreamSynchronize(s));
            check_ipm_status_host(nd.hs.p);
            if (nd.hi.p[BI_ERR] & 1) fatal("SDPbound", "Bundle size too large! Adjust MaxBundle");
            t *= 1.05;
        }
        bdl_iter += count % 2;
        bdl_iter = (bdl_iter < params.max_bundle_iter) ? bdl_iter : params.max_bundle_iter;
    }
    if (warm_on || warm_rec || pstart_on) {
        const int mall = PP_->NIneq + PP_->NPentIneq + PP_->NHeptaIneq;
        std::vector<double> fg(mall > 0 ? mall : 1);
        if (mall > 0) {
            BQB_CUDA(cudaMemcpyAsync(fg.data(), b.gam.p, (size_t)mall * sizeof(double), cudaMemcpyDeviceToHost, s));
            BQB_CUDA(cudaStreamSynchronize(s));
        }
        if (warm_rec && !warm_first.empty())
            warm_record(warm_feats, warm_scale, warm_first.data(), (int)warm_first.size(), H.cuts, fg.data(),
                        PP_->NIneq);
        // the node's final triangle cuts, for its children
        auto fc = std::make_shared<ParentCuts>();
        fc->key.reserve(PP_->NIneq);
        fc->gam.reserve(PP_->NIneq);
        for (int c = 0; c < PP_->NIneq; ++c) {
            const Triangle_Inequality& t = H.cuts[c];
            const uint64_t key = orig_cut_key(t.type, orig[t.i], orig[t.j], orig[t.k]);
            fc->key.push_back(key);
            fc->gam.push_back(fg[c]);
            fc->index[key] = fg[c];
        }
        if (pstart_on) {
            for (int i = 0; i < PP_->NPentIneq; ++i) {
                ParentKgon q{H.pcuts[i].type, {0, 0, 0, 0, 0, 0, 0}, fg[PP_->NIneq + i]};
                for (int a = 0; a < 5; ++a) q.v[a] = orig[H.pcuts[i].permutation[a]];
                fc->pent.push_back(q);
            }
            for (int i = 0; i < PP_->NHeptaIneq; ++i) {
                ParentKgon q{H.hcuts[i].type, {0, 0, 0, 0, 0, 0, 0}, fg[PP_->NIneq + PP_->NPentIneq + i]};
                for (int a = 0; a < 7; ++a) q.v[a] = orig[H.hcuts[i].permutation[a]];
                fc->hept.push_back(q);
            }
        }
        E.final_cuts = std::move(fc);
    }
    bound = f + fixedvalue;
    if (rank == 0) diff = basic_bound - bound;
    pc.mark(EP_REBUILD);
    certify(true, f, fixedvalue);
    return bound;
}

}  // namespace bqb

using namespace bqb;

// Replace the default engine's GW heuristic by a host function with
// runHeuristic_unpacked's contract (NULL: back to the GPU heuristic).
BQB_API void bqb_set_heuristic_hook(bqb_heuristic_fn fn) { g_heuristic_hook.store(fn); }

// Heuristic calls made by SDPbound / sdp_bound since the last reset.
BQB_API long long bqb_heuristic_runs(int reset)
{
    return reset ? g_heuristic_runs.exchange(0) : g_heuristic_runs.load();
}

// Bundle iterations (src/bundle.c:9-239, one fct_eval each) run by SDPbound
// on the default engine and on engines since the last reset.
BQB_API long long bqb_bundle_iterations(int reset)
{
    return reset ? g_bundle_iters.exchange(0) : g_bundle_iters.load();
}

// Time by phase of the engines' SDPbound (seconds, summed over engines and
// calls): out[12] = {IPM, lambda_eta, L - B^T(gamma), op_B + bundle step,
// heuristic, triangle separation, pentagonal / heptagonal separation, the
// rest, whole calls, cut upload, fracsol, bundle growth}.  Profiling only: with it on, every
// phase boundary synchronises the engine's stream.  reset != 0 zeroes the
// sums after reading.  No reference counterpart.
BQB_API void bqb_engine_profile_enable(int on) { g_eprof_on.store(on ? 1 : 0); }
BQB_API void bqb_engine_profile(double* out, int reset)
{
    for (int i = 0; i < EP_WORDS; ++i) {
        const long long v = reset ? g_eprof_ns[i].exchange(0) : g_eprof_ns[i].load();
        if (out) out[i] = 1e-9 * (double)v;
    }
}

// FP64 certificates of the engines' node bounds on (1) / off (0): each node
// costs one more IPM and a Cholesky factorisation.  bqb_certify_stats:
// out[6] = {nodes certified, the largest and the mean excess of the
// certified bound over the node's bound (relative to max(1, |bound|)),
// nodes whose certificate failed, the largest diagonal shift a certificate
// needed, the largest difference between the rerun IPM's value and the
// bundle's F - sum(gamma) (relative)}; reset != 0 zeroes the statistics.
// No reference counterpart.
BQB_API void bqb_certify_enable(int on) { g_cert_on.store(on ? 1 : 0); }
BQB_API void bqb_certify_stats(double* out, int reset)
{
    std::lock_guard<std::mutex> lk(g_cert_mu);
    if (out) {
        out[0] = (double)g_cert.nodes;
        out[1] = g_cert.max_rel;
        out[2] = g_cert.nodes > g_cert.failed ? g_cert.sum_rel / (double)(g_cert.nodes - g_cert.failed) : 0.0;
        out[3] = (double)g_cert.failed;
        out[4] = g_cert.max_shift;
        out[5] = g_cert.max_mismatch;
    }
    if (reset) g_cert = CertStats{};
}

// Parent start on (1) or off (0, the reference's start at every node).
BQB_API void bqb_set_parent_start(int on) { g_parent_start.store(on ? 1 : 0); }

// Root effort on (1) or off (0, the reference's give-up rule at every node).
BQB_API void bqb_set_root_effort(int full) { g_root_effort.store(full ? 1 : 0); }

// Tracing of SDPbound's outer loop on (1) / off (0); switching it on clears
// the trace and restarts the node numbering.
BQB_API void bqb_bound_trace_enable(int on)
{
    std::lock_guard<std::mutex> g(g_trace_mu);
    g_trace.clear();
    g_trace_node.store(0);
    g_trace_on.store(on ? 1 : 0);
}

// Copies up to max_rows trace rows (node, rank, round, bound, incumbent,
// triangle / pentagonal / heptagonal cuts after the round's separation,
// seconds since the node's loop started) into out and returns the number
// of rows recorded so far.
BQB_API int bqb_bound_trace(double* out, int max_rows)
{
    std::lock_guard<std::mutex> g(g_trace_mu);
    const int rows = (int)(g_trace.size() / BQB_TRACE_COLS);
    const int k = rows < max_rows ? rows : max_rows;
    if (out && k > 0) memcpy(out, g_trace.data(), (size_t)k * BQB_TRACE_COLS * sizeof(double));
    return rows;
}

// SDPbound (src/bounding.c:24-342) in the default engine: the reference's
// globals and rand() stream.
BQB_API double SDPbound(BabNode* node, Problem* SP_, Problem* PP_, int rank)
{
    rt();
    return sdp_bound(default_engine(), node, SP_, PP_, rank);
}
