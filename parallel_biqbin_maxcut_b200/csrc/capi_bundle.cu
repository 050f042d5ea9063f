// Drop-in bundle entry points (src/bundle.c): bundle_method, lambda_eta and
// solve_lambda with the reference's host-global contract.  The bundle runs
// on the device (bundle.cu); these functions move the globals in and out.
#include <string.h>

#include <vector>

#include "engine.h"
#include "internal.h"
#include "node.h"

using namespace bqb;

namespace {

// The drop-in bundle entry points work on the reference's globals (like the
// default engine) with device buffers of their own.
Engine& dropin_engine()
{
    static Engine* e = [] {
        Engine* d = new Engine();
        d->stream = rt().stream;
        d->is_default = true;
        return d;
    }();
    return *e;
}

void upload_identity_slots(BundleDev& b, int k, cudaStream_t s)
{
    std::vector<int> id(b.cap);
    for (int i = 0; i < b.cap; ++i) id[i] = i;
    BQB_CUDA(cudaMemcpyAsync(b.slot.p, id.data(), b.cap * sizeof(int), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    (void)k;
}

// Host G (m x k, column i at G + m*i) -> device columns 0..k-1 (ld = ldg).
void upload_G(BundleDev& b, const double* Gh, int m, int k, cudaStream_t s)
{
    if (m <= 0 || k <= 0) return;
    BQB_CUDA(cudaMemcpy2DAsync(b.G.p, (size_t)b.ldg * sizeof(double), Gh, (size_t)m * sizeof(double),
                               (size_t)m * sizeof(double), k, cudaMemcpyHostToDevice, s));
}

}  // namespace

BQB_API void bundle_method(Problem* P, double* t, int bdl_iter)
{
    rt();
    Engine& E = dropin_engine();
    cudaStream_t s = E.stream;
    NodeDev& nd = E.nd;
    const int n = P->n;
    const size_t nn = (size_t)n * n;
    const int m = P->NIneq + P->NPentIneq + P->NHeptaIneq;
    const int k = P->bundle;
    nd.n = n;
    nd.hs.ensure(8);
    nd.hi.ensure(8);
    nd.L.ensure(nn);
    nd.L0.ensure(nn);
    nd.X.ensure(nn);
    nd.out.ensure(4);
    BQB_CUDA(cudaMemcpyAsync(nd.L.p, P->L, nn * sizeof(double), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemcpyAsync(nd.X.p, X, nn * sizeof(double), cudaMemcpyHostToDevice, s));
    upload_cuts(E, E.host(), P);
    BundleDev& b = nd.b;
    b.ensure_cap(k + bdl_iter + 2, n, s);
    upload_identity_slots(b, k, s);
    if (k > 0) BQB_CUDA(cudaMemcpyAsync(b.Xb.p, X_bundle, (size_t)k * nn * sizeof(double), cudaMemcpyHostToDevice, s));
    upload_G(b, G, m, k, s);
    if (k > 0) BQB_CUDA(cudaMemcpyAsync(b.Fv.p, F, (size_t)k * sizeof(double), cudaMemcpyHostToDevice, s));
    if (m > 0) BQB_CUDA(cudaMemcpyAsync(b.gam.p, dual_gamma, (size_t)m * sizeof(double), cudaMemcpyHostToDevice, s));
    int* hi = nd.hi.p;
    for (int q = 0; q < 8; ++q) hi[q] = 0;
    hi[BI_K] = k;
    hi[BI_NEXT] = k;
    hi[BI_CAP] = b.cap;
    BQB_CUDA(cudaMemcpyAsync(b.istate.p, hi, BI_WORDS * sizeof(int), cudaMemcpyHostToDevice, s));
    nd.hs.p[BD_F] = f;
    nd.hs.p[BD_T] = *t;
    nd.hs.p[BD_FTEST] = 0.0;
    nd.hs.p[BD_DEL] = 0.0;
    BQB_CUDA(cudaMemcpyAsync(b.dstate.p, nd.hs.p, BD_WORDS * sizeof(double), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaStreamSynchronize(s));

    f = bundle_iterations(E, bdl_iter, t);

    const int k2 = nd.hi.p[BI_K];
    const int kold = nd.hi.p[BI_KOLD];
    const int last = nd.hi.p[BI_LAST];
    std::vector<int> slot(k2 > 0 ? k2 : 1);
    BQB_CUDA(cudaMemcpyAsync(slot.data(), b.slot.p, k2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    BQB_CUDA(cudaMemcpyAsync(X, nd.X.p, nn * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(X_test, b.Xb.p + (size_t)last * nn, nn * sizeof(double), cudaMemcpyDeviceToHost, s));
    for (int i = 0; i < k2; ++i) {
        BQB_CUDA(cudaMemcpyAsync(X_bundle + (size_t)i * nn, b.Xb.p + (size_t)slot[i] * nn, nn * sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
        if (m > 0)
            BQB_CUDA(cudaMemcpyAsync(G + (size_t)i * m, b.G.p + (size_t)slot[i] * b.ldg, m * sizeof(double),
                                     cudaMemcpyDeviceToHost, s));
    }
    BQB_CUDA(cudaMemcpyAsync(F, b.Fv.p, k2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (m > 0) {
        BQB_CUDA(cudaMemcpyAsync(g, b.G.p + (size_t)last * b.ldg, m * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaMemcpyAsync(dual_gamma, b.gam.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaMemcpyAsync(dgamma, b.dgam.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaMemcpyAsync(gamma_test, b.gtest.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaMemcpyAsync(eta, b.eta.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    BQB_CUDA(cudaMemcpyAsync(lambda, b.lam.p, kold * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    P->bundle = k2;
}

BQB_API void lambda_eta(const Problem* P, double* zeta, double* Gh, double* gam, double* dgam, double* lam,
                        double* et, double* t)
{
    rt();
    Engine& E = dropin_engine();
    cudaStream_t s = E.stream;
    NodeDev& nd = E.nd;
    const int m = P->NIneq + P->NPentIneq + P->NHeptaIneq;
    const int k = P->bundle;
    BundleDev& b = nd.b;
    nd.hs.ensure(8);
    nd.hi.ensure(8);
    b.ensure_cap(k + 2, b.n > 0 ? b.n : 1, s);
    b.ensure_m(m, s);
    if (b.G.cap < (size_t)b.ldg * b.cap) b.G.ensure((size_t)b.ldg * b.cap);
    upload_identity_slots(b, k, s);
    upload_G(b, Gh, m, k, s);
    static DevBuf<double> dz;
    dz.ensure(k > 0 ? k : 1);
    BQB_CUDA(cudaMemcpyAsync(dz.p, zeta, k * sizeof(double), cudaMemcpyHostToDevice, s));
    if (m > 0) BQB_CUDA(cudaMemcpyAsync(b.gam.p, gam, m * sizeof(double), cudaMemcpyHostToDevice, s));
    int* hi = nd.hi.p;
    for (int q = 0; q < 8; ++q) hi[q] = 0;
    hi[BI_K] = k;
    hi[BI_CAP] = b.cap;
    BQB_CUDA(cudaMemcpyAsync(b.istate.p, hi, BI_WORDS * sizeof(int), cudaMemcpyHostToDevice, s));
    nd.hs.p[BD_T] = *t;
    BQB_CUDA(cudaMemcpyAsync(b.dstate.p + BD_T, nd.hs.p + BD_T, sizeof(double), cudaMemcpyHostToDevice, s));
    lambda_eta_launch(b, dz.p, s);
    if (m > 0) {
        BQB_CUDA(cudaMemcpyAsync(dgam, b.dgam.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaMemcpyAsync(et, b.eta.p, m * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    BQB_CUDA(cudaMemcpyAsync(lam, b.lam.p, k * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(nd.hs.p, b.dstate.p, BD_WORDS * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(hi, b.istate.p, BI_WORDS * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    if (hi[BI_ERR] & 2) fatal("solve_lambda", "Problem in solving linear system");
    *t = nd.hs.p[BD_T];
}

BQB_API void solve_lambda(int k, double* Q, double* c, double* lam)
{
    Runtime& R = rt();
    cudaStream_t s = R.stream;
    static DevBuf<double> dQ, dc, dl;
    static DevBuf<int> derr;
    dQ.ensure((size_t)k * k);
    dc.ensure(k);
    dl.ensure(k);
    derr.ensure(1);
    BQB_CUDA(cudaMemcpyAsync(dQ.p, Q, (size_t)k * k * sizeof(double), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemcpyAsync(dc.p, c, k * sizeof(double), cudaMemcpyHostToDevice, s));
    solve_lambda_launch(k, dQ.p, dc.p, dl.p, derr.p, s);
    int err = 0;
    BQB_CUDA(cudaMemcpyAsync(lam, dl.p, k * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(&err, derr.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    if (err) fatal("solve_lambda", "Problem in solving linear system");
}
