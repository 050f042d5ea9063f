// Engines: the default one (drop-in, process globals) and private ones.
#include "engine.h"

namespace bqb {

std::atomic<unsigned> g_sp_generation{0};

Engine& default_engine()
{
    static Engine* e = [] {
        Engine* d = new Engine();
        d->stream = rt().stream;
        d->is_default = true;
        return d;
    }();
    return *e;
}

HostState Engine::host()
{
    if (is_default)
        return HostState{Cuts, Pent_Cuts, Pent_List, Hepta_Cuts, Hepta_List, dual_gamma, X, &f};
    return HostState{cuts_v.data(), pcuts_v.data(), plist_v.data(), hcuts_v.data(), hlist_v.data(),
                     dual_v.data(), X_v.data(), &f_v};
}

void Engine::ensure_private(int N)
{
    const size_t mmax = (size_t)BQB_MAX_TRI_INEQ + BQB_MAX_PENT_INEQ + BQB_MAX_HEPTA_INEQ;
    if (cuts_v.size() < (size_t)BQB_MAX_TRI_INEQ) cuts_v.resize(BQB_MAX_TRI_INEQ);
    if (pcuts_v.size() < (size_t)BQB_MAX_PENT_INEQ) pcuts_v.resize(BQB_MAX_PENT_INEQ);
    if (hcuts_v.size() < (size_t)BQB_MAX_HEPTA_INEQ) hcuts_v.resize(BQB_MAX_HEPTA_INEQ);
    const size_t pl = params.PentIneq > 0 ? (size_t)params.PentIneq : 1;
    const size_t hl = params.HeptaIneq > 0 ? (size_t)params.HeptaIneq : 1;
    if (plist_v.size() < pl) plist_v.resize(pl);
    if (hlist_v.size() < hl) hlist_v.resize(hl);
    if (dual_v.size() < mmax) dual_v.resize(mmax);
    if (X_v.size() < (size_t)N * N) X_v.resize((size_t)N * N);
    if (PPL.size() < (size_t)N * N) PPL.resize((size_t)N * N);
    PP.L = PPL.data();
}

Engine* engine_create(unsigned seed)
{
    rt();
    Engine* e = new Engine();
    BQB_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    e->rng.seed(seed);
    e->sa_seed = (uint64_t)seed << 32;
    return e;
}

template <class T>
static void free_dev(DevBuf<T>& b)
{
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
}

template <class T>
static void free_host(HostBuf<T>& b)
{
    if (b.p) cudaFreeHost(b.p);
    b.p = nullptr;
    b.cap = 0;
}

void engine_destroy(Engine* e)
{
    if (!e || e->is_default) return;
    cudaStreamSynchronize(e->stream);
    NodeDev& nd = e->nd;
    free_dev(nd.L);
    free_dev(nd.L0);
    free_dev(nd.X);
    free_dev(nd.out);
    free_dev(nd.P0L);
    free_dev(nd.cuts.rec);
    free_dev(nd.cuts.pair_uv);
    free_dev(nd.cuts.offsets);
    free_dev(nd.cuts.contrib);
    BundleDev& b = nd.b;
    free_dev(b.Xb);
    free_dev(b.G);
    free_dev(b.Fv);
    free_dev(b.slot);
    free_dev(b.slot_old);
    free_dev(b.lam);
    free_dev(b.gam);
    free_dev(b.gtest);
    free_dev(b.dgam);
    free_dev(b.eta);
    free_dev(b.dstate);
    free_dev(b.istate);
    free_dev(b.qp_ws);
    free_host(nd.hs);
    free_host(nd.hi);
    HeurState& h = e->heur;
    free_dev(h.Z);
    free_dev(h.V);
    free_dev(h.x);
    free_dev(h.sols);
    free_dev(h.vals);
    free_dev(h.best);
    free_dev(h.bestval);
    free_dev(h.fixed);
    free_dev(h.status);
    free_dev(h.P0L);
    free_dev(h.PL);
    free_dev(h.Xs);
    free_host(h.hV);
    free_host(h.hbest);
    free_host(h.hval);
    free_host(h.hstat);
    free_dev(e->sa.cost);
    free_dev(e->sa.perm);
    free_dev(e->sa.status);
    free_host(e->sa.hcost);
    free_host(e->sa.hperm);
    free_host(e->sa.hstat);
    TriSepState& t = e->tri;
    free_dev(t.XT);
    free_dev(t.cnt);
    free_dev(t.misc);
    free_dev(t.cand);
    free_dev(t.list);
    free_host(t.hmisc);
    free_host(t.hlist);
    free_dev(e->ipm_ws);
    cudaStreamDestroy(e->stream);
    delete e;
}

}  // namespace bqb
