// Drop-in C entry points for the SDP core: ipm_mc_pk, op_B, op_Bt, diag,
// Diag, fct_eval, plus the batched/device-pointer IPM.  Host buffers in and
// out, as the reference signatures require; the GPU does the work.
#include <string.h>

#include <vector>

#include "cuts.cuh"
#include "globals.h"
#include "internal.h"
#include "ipm.cuh"

namespace bqb {

std::vector<CutRec> pack_cuts(const Triangle_Inequality* tc, int mt, const Pentagonal_Inequality* pc, int mp,
                              const Heptagonal_Inequality* hc, int mh)
{
    std::vector<CutRec> v;
    v.reserve((size_t)mt + mp + mh);
    for (int c = 0; c < mt; ++c) {
        const int p[3] = {tc[c].i, tc[c].j, tc[c].k};
        v.push_back(pack_cut(3, p, tri_negmask(tc[c].type)));
    }
    for (int c = 0; c < mp; ++c) v.push_back(pack_cut(5, pc[c].permutation, pent_negmask(pc[c].type)));
    for (int c = 0; c < mh; ++c) v.push_back(pack_cut(7, hc[c].permutation, hept_negmask(hc[c].type)));
    return v;
}

// The reference's global cut arrays (first P->NIneq / NPentIneq / NHeptaIneq
// entries).
std::vector<CutRec> pack_global_cuts(const Problem* P)
{
    return pack_cuts(Cuts, P->NIneq, Pent_Cuts, P->NPentIneq, Hepta_Cuts, P->NHeptaIneq);
}

namespace {
struct CoreState {
    DevBuf<double> L, X, ws, out, y, t;
    DevBuf<IpmDesc> descs;
    HostBuf<double> hout;
    DevCuts cuts;
};
CoreState& core()
{
    static CoreState s;
    return s;
}

}  // namespace

void check_ipm_status_host(const double* out)
{
    const int status = (int)out[2];
    if (status == IPM_OK) return;
    const char* msg = status == IPM_Z_NOT_PD   ? "Problem with Cholesky factorization (Z not PD)"
                      : status == IPM_M_NOT_PD ? "problem in solving linear system (Zi.*X not PD)"
                      : status == IPM_LINESEARCH ? "line search found no positive definite step"
                      : status == IPM_SYNC ? "a grid barrier of the multi-CTA IPM gave up waiting"
                                                 : "iteration limit reached";
    fatal("ipm_mc_pk", msg);
}

// Device-level basic SDP bound for one problem (used by every caller).
// xslot (optional, device): write X into dX + (*xslot) * n * n.
void ipm_device(DevBuf<double>& wsbuf, const double* dL, double* dX, int n, double* dout, cudaStream_t s,
                const int* xslot, double* yout)
{
    if (n > IPM_REG_NMAX) {
        ipm_large(wsbuf, dL, dX, n, dout, s, xslot, yout);
        return;
    }
    size_t bytes = 0;
    const int place = ipm_place(n, rt().smem_optin, &bytes);
    double* ws = wsbuf.ensure(ipm_ws_doubles(n, place));
    IpmDesc d{dL, dX, ws, dout, xslot, n, 0, yout};
    ipm_launch_one(d, s);
}

}  // namespace bqb

using namespace bqb;

BQB_API void ipm_mc_pk(double* L, int n, double* Xout, double* phi, int print)
{
    (void)print;
    Runtime& R = rt();
    CoreState& c = core();
    const size_t nn = (size_t)n * n;
    double* dL = c.L.ensure(nn);
    double* dX = c.X.ensure(nn);
    double* dout = c.out.ensure(4);
    double* hout = c.hout.ensure(4);
    BQB_CUDA(cudaMemcpyAsync(dL, L, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    ipm_device(c.ws, dL, dX, n, dout, R.stream);
    BQB_CUDA(cudaMemcpyAsync(Xout, dX, nn * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaMemcpyAsync(hout, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaStreamSynchronize(R.stream));
    check_ipm_status_host(hout);
    *phi = hout[0];
}

BQB_API void diag(const double* Xm, double* y, int n)
{
    for (int i = 0; i < n; ++i) y[i] = Xm[i + (size_t)i * n];
}

BQB_API void Diag(double* Xm, const double* y, int n)
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) Xm[j + (size_t)i * n] = (i == j) ? y[i] : 0.0;
}

BQB_API void op_B(const Problem* P, double* y, const double* Xm)
{
    const int m = P->NIneq + P->NPentIneq + P->NHeptaIneq;
    if (m <= 0) return;
    Runtime& R = rt();
    CoreState& c = core();
    const int n = P->n;
    const size_t nn = (size_t)n * n;
    std::vector<CutRec> rec = pack_global_cuts(P);
    c.cuts.upload(rec, P->NIneq, P->NPentIneq, P->NHeptaIneq, R.stream);
    double* dX = c.X.ensure(nn);
    double* dy = c.y.ensure(m);
    BQB_CUDA(cudaMemcpyAsync(dX, Xm, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    BQB_CUDA(cudaMemcpyAsync(dy, y, m * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    opB_launch(c.cuts, dX, nn, nullptr, 1, n, dy, m, false, R.stream);
    BQB_CUDA(cudaMemcpyAsync(y, dy, m * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaStreamSynchronize(R.stream));
}

BQB_API void op_Bt(const Problem* P, double* Xm, const double* tt)
{
    const int m = P->NIneq + P->NPentIneq + P->NHeptaIneq;
    if (m <= 0) return;
    Runtime& R = rt();
    CoreState& c = core();
    const int n = P->n;
    const size_t nn = (size_t)n * n;
    std::vector<CutRec> rec = pack_global_cuts(P);
    c.cuts.upload(rec, P->NIneq, P->NPentIneq, P->NHeptaIneq, R.stream);
    double* dX = c.X.ensure(nn);
    double* dt = c.t.ensure(m);
    BQB_CUDA(cudaMemcpyAsync(dX, Xm, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    BQB_CUDA(cudaMemcpyAsync(dt, tt, m * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    opBt_launch(c.cuts, dX, n, dt, R.stream);
    BQB_CUDA(cudaMemcpyAsync(Xm, dX, nn * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaStreamSynchronize(R.stream));
}

// fct_eval (src/bundle.c:242-275): L0 = L - B^T(gamma); X = IPM(L0);
// f = phi + sum(gamma); g = 1 - B(X).  All on the device; X and g copied out.
BQB_API double fct_eval(const Problem* PP_, double* gam, double* Xout, double* gout)
{
    Runtime& R = rt();
    CoreState& c = core();
    const int n = PP_->n;
    const int m = PP_->NIneq + PP_->NPentIneq + PP_->NHeptaIneq;
    const size_t nn = (size_t)n * n;
    double* dL = c.L.ensure(nn);
    double* dX = c.X.ensure(nn);
    double* dout = c.out.ensure(4);
    double* hout = c.hout.ensure(4);
    BQB_CUDA(cudaMemcpyAsync(dL, PP_->L, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    if (m > 0) {
        std::vector<CutRec> rec = pack_global_cuts(PP_);
        c.cuts.upload(rec, PP_->NIneq, PP_->NPentIneq, PP_->NHeptaIneq, R.stream);
        double* dt = c.t.ensure(m);
        BQB_CUDA(cudaMemcpyAsync(dt, gam, m * sizeof(double), cudaMemcpyHostToDevice, R.stream));
        opBt_launch(c.cuts, dL, n, dt, R.stream);
    }
    ipm_device(c.ws, dL, dX, n, dout, R.stream);
    double* dy = nullptr;
    if (m > 0) {
        dy = c.y.ensure(m);
        opB_launch(c.cuts, dX, nn, nullptr, 1, n, dy, m, true, R.stream);
    }
    BQB_CUDA(cudaMemcpyAsync(Xout, dX, nn * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    if (m > 0) BQB_CUDA(cudaMemcpyAsync(gout, dy, m * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaMemcpyAsync(hout, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaStreamSynchronize(R.stream));
    check_ipm_status_host(hout);
    double fv = hout[0];
    // sum in index order, as src/bundle.c:264-265
    for (int i = 0; i < m; ++i) fv += gam[i];
    return fv;
}

// ---- batched basic bound ------------------------------------------------

struct bqb_ipm_plan {
    DevBuf<IpmDesc> descs;
    DevBuf<double> ws;
    int nprob = 0;
    int n_max = 0;
};

BQB_API bqb_ipm_plan* bqb_ipm_plan_create(const double* const* Ls, double* const* Xs, const int* ns,
                                          int nprob, double* out)
{
    Runtime& R = rt();
    bqb_ipm_plan* p = new bqb_ipm_plan();
    p->nprob = nprob;
    for (int i = 0; i < nprob; ++i) p->n_max = ns[i] > p->n_max ? ns[i] : p->n_max;
    size_t bytes = 0;
    const int place = ipm_place(p->n_max, R.smem_optin, &bytes);
    size_t total = 0;
    for (int i = 0; i < nprob; ++i) total += ipm_ws_doubles(ns[i], place);
    double* ws = p->ws.ensure(total > 0 ? total : 1);
    std::vector<IpmDesc> h(nprob > 0 ? nprob : 1);
    size_t off = 0;
    for (int i = 0; i < nprob; ++i) {
        h[i] = IpmDesc{Ls[i], Xs[i], ws + off, out + 4 * (size_t)i, nullptr, ns[i], 0};
        off += ipm_ws_doubles(ns[i], place);
    }
    IpmDesc* dd = p->descs.ensure(nprob > 0 ? nprob : 1);
    BQB_CUDA(cudaMemcpy(dd, h.data(), nprob * sizeof(IpmDesc), cudaMemcpyHostToDevice));
    return p;
}

BQB_API int bqb_ipm_plan_launch(bqb_ipm_plan* p, void* stream)
{
    if (!p || p->nprob <= 0) return 0;
    cudaStream_t s = stream ? (cudaStream_t)stream : rt().stream;
    ipm_launch(p->descs.p, p->nprob, p->n_max, s);
    return 0;
}

BQB_API void bqb_ipm_plan_destroy(bqb_ipm_plan* p)
{
    if (!p) return;
    if (p->descs.p) BQB_CUDA(cudaFree(p->descs.p));
    if (p->ws.p) BQB_CUDA(cudaFree(p->ws.p));
    delete p;
}

BQB_API int bqb_ipm_batch_device(const double* const* Ls, double* const* Xs, const int* ns, int nprob,
                                 double* out, void* stream)
{
    if (nprob <= 0) return 0;
    cudaStream_t s = stream ? (cudaStream_t)stream : rt().stream;
    bqb_ipm_plan* p = bqb_ipm_plan_create(Ls, Xs, ns, nprob, out);
    bqb_ipm_plan_launch(p, s);
    BQB_CUDA(cudaStreamSynchronize(s));
    bqb_ipm_plan_destroy(p);
    return 0;
}

BQB_API int bqb_ipm_batch(const double* const* Ls, double* const* Xs, const int* ns, int nprob,
                          double* phi, int* iters, int* status)
{
    if (nprob <= 0) return 0;
    Runtime& R = rt();
    size_t total = 0;
    for (int i = 0; i < nprob; ++i) total += (size_t)ns[i] * ns[i];
    DevBuf<double> dL, dX, dout;
    dL.ensure(total);
    dX.ensure(total);
    dout.ensure(4 * (size_t)nprob);
    std::vector<const double*> pl(nprob);
    std::vector<double*> px(nprob);
    size_t off = 0;
    for (int i = 0; i < nprob; ++i) {
        const size_t nn = (size_t)ns[i] * ns[i];
        pl[i] = dL.p + off;
        px[i] = dX.p + off;
        BQB_CUDA(cudaMemcpyAsync(dL.p + off, Ls[i], nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
        off += nn;
    }
    bqb_ipm_plan* p = bqb_ipm_plan_create(pl.data(), px.data(), ns, nprob, dout.p);
    bqb_ipm_plan_launch(p, R.stream);
    std::vector<double> hout(4 * (size_t)nprob);
    off = 0;
    for (int i = 0; i < nprob; ++i) {
        const size_t nn = (size_t)ns[i] * ns[i];
        BQB_CUDA(cudaMemcpyAsync(Xs[i], dX.p + off, nn * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
        off += nn;
    }
    BQB_CUDA(cudaMemcpyAsync(hout.data(), dout.p, hout.size() * sizeof(double), cudaMemcpyDeviceToHost,
                             R.stream));
    BQB_CUDA(cudaStreamSynchronize(R.stream));
    bqb_ipm_plan_destroy(p);
    BQB_CUDA(cudaFree(dL.p));
    BQB_CUDA(cudaFree(dX.p));
    BQB_CUDA(cudaFree(dout.p));
    for (int i = 0; i < nprob; ++i) {
        if (phi) phi[i] = hout[4 * i];
        if (iters) iters[i] = (int)hout[4 * i + 1];
        if (status) status[i] = (int)hout[4 * i + 2];
    }
    return 0;
}
