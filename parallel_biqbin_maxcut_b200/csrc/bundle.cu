// Proximal bundle method (src/bundle.c:9-653) on the device.
//
// lambda_eta_kernel: one CTA.  zeta = -F - G'gamma, Q = t G'G, then up to
//   50 rounds of c = zeta - t G'eta, lambda = QP(Q, c) (warp 0),
//   eta = max(0, -gamma/t + G lambda), dgamma = t (eta - G lambda), stopping
//   on the relative change of ||dgamma|| (src/bundle.c:292-373).
// warp_qp: the simplex-constrained QP of solve_lambda (src/bundle.c:390-653),
//   a primal-dual IPM with the reference's start, step rule, mu updates and
//   stopping test.  Its (k+1) x (k+1) KKT system [-Q-D e; e' 0] is solved by
//   the Schur complement on A = Q + D (positive definite since D = z./lambda
//   > 0): u = A\e, w = A\r, dy = (res_p + sum w)/sum u, dlambda = u dy - w;
//   the reference solves the same system with dsysv.
// bundle_step_kernel: the serious / null decision, t update, purge and append
//   of src/bundle.c:75-234, on slot indices (no matrix moves).
// bundle_xcomb_kernel: X = X_bundle * lambda after a serious step.
#include <math.h>

#include <mutex>

#include "bundle_body.cuh"
#include "globals.h"

namespace bqb {

namespace {

__global__ void __launch_bounds__(LE_THREADS) lambda_eta_kernel(LeArgs a)
{
    extern __shared__ __align__(16) double sm[];
    lambda_eta_body(a, sm);
}

__global__ void solve_lambda_kernel(int k, const double* Q, const double* c, double* lam, int* err,
                                    double* ws_global)
{
    extern __shared__ __align__(16) double sm[];
    solve_lambda_body(k, Q, c, lam, err, ws_global, sm);
}

__global__ void __launch_bounds__(LE_THREADS) bundle_step_kernel(StepArgs a) { bundle_step_body(a); }

__global__ void bundle_xcomb_kernel(const double* __restrict__ Xb, const int* __restrict__ slot_old,
                                    const double* __restrict__ lam, const int* __restrict__ istate,
                                    double* __restrict__ X, size_t nn)
{
    bundle_xcomb_body(Xb, slot_old, lam, istate, X, nn, (size_t)blockIdx.x * blockDim.x + threadIdx.x,
                      (size_t)gridDim.x * blockDim.x);
}

__global__ void __launch_bounds__(LE_THREADS) bundle_fval_kernel(const double* __restrict__ L,
                                                                 const double* __restrict__ Xb, int n,
                                                                 const int* __restrict__ slot_ptr,
                                                                 const int* __restrict__ pos_ptr,
                                                                 double* __restrict__ Fv)
{
    bundle_fval_body(L, Xb, n, slot_ptr, pos_ptr, Fv);
}

__global__ void bundle_append_kernel(int* __restrict__ slot, int* __restrict__ istate, int cap)
{
    bundle_append_body(slot, istate, cap);
}

}  // namespace

void BundleDev::ensure_cap(int need, int n_, cudaStream_t s)
{
    if (n_ != n) {   // a new problem size: the old contents are dead
        cap = 0;
        n = n_;
    }
    dstate.ensure(BD_WORDS);
    istate.ensure(BI_WORDS);
    if (need > BQB_MAX_BUNDLE + 2) need = BQB_MAX_BUNDLE + 2;
    if (need <= cap) return;
    const size_t nn = (size_t)n_ * n_;
    int newcap = need + 8;
    if (newcap > BQB_MAX_BUNDLE + 2) newcap = BQB_MAX_BUNDLE + 2;
    const int lg = ldg > 0 ? ldg : 1;
    Xb.grow_keep(newcap * nn, (size_t)cap * nn, s);
    G.grow_keep((size_t)lg * newcap, (size_t)lg * cap, s);
    Fv.grow_keep(newcap, cap, s);
    slot.grow_keep(newcap, cap, s);
    slot_old.grow_keep(newcap, cap, s);
    lam.grow_keep(newcap, cap, s);
    qp_ws.ensure((size_t)2 * newcap * newcap + 8 * (size_t)newcap);
    cap = newcap;
}

void BundleDev::ensure_m(int m_, cudaStream_t s)
{
    m = m_;
    const int need = m_ > 0 ? m_ : 1;
    gam.ensure(need);
    gtest.ensure(need);
    dgam.ensure(need);
    eta.ensure(need);
    if (need > ldg) {
        ldg = need + need / 4;
        G.ensure((size_t)ldg * (cap > 0 ? cap : 1));
    }
    (void)s;
}

extern std::atomic<int> g_eprof_on;

// lambda_eta counters of the engines and the fused kernel (with the engines'
// phase profile on): calls, rounds, sum of k, cycles in the QP, cycles, sum
// of m.
DevBuf<unsigned long long> g_le_prof;
std::mutex g_le_prof_mu;

unsigned long long* le_prof_device()
{
    if (!g_eprof_on.load()) return nullptr;
    std::lock_guard<std::mutex> lock(g_le_prof_mu);
    if (!g_le_prof.p) {
        g_le_prof.ensure(8);
        BQB_CUDA(cudaMemset(g_le_prof.p, 0, 8 * sizeof(unsigned long long)));
    }
    return g_le_prof.p;
}

void lambda_eta_launch(BundleDev& b, const double* zeta_in, cudaStream_t s)
{
    // k is only known on the device: size shared memory for any k <= cap.
    const int kcap = b.cap;
    size_t bytes = le_smem_bytes(kcap > QP_SMEM_K ? QP_SMEM_K : kcap);
    if (kcap > QP_SMEM_K && 3 * (size_t)kcap * sizeof(double) > bytes) bytes = 3 * (size_t)kcap * sizeof(double);
    BQB_SMEM_LIMIT(lambda_eta_kernel, bytes);
    LeArgs a{b.G.p, b.ldg, b.slot.p, b.m, zeta_in, b.Fv.p, b.gam.p, b.lam.p, b.eta.p, b.dgam.p,
             b.gtest.p, b.dstate.p, b.istate.p, b.qp_ws.p, -1};
    a.prof = le_prof_device();
    lambda_eta_kernel<<<1, LE_THREADS, bytes, s>>>(a);
    BQB_COUNT_LAUNCH();
    check_launch("lambda_eta_kernel");
}

void solve_lambda_launch(int k, const double* Q, const double* c, double* lambda, int* err, cudaStream_t s)
{
    static DevBuf<double> ws;
    double* w = ws.ensure((size_t)k * k + qp_a_doubles(k) + 8 * (size_t)k + 8);
    size_t bytes = 2 * (size_t)k * sizeof(double);
    if (k <= QP_SMEM_K) bytes += (qp_a_doubles(k) + 6 * (size_t)k) * sizeof(double);
    BQB_SMEM_LIMIT(solve_lambda_kernel, bytes);
    solve_lambda_kernel<<<1, 32, bytes, s>>>(k, Q, c, lambda, err, w);
    BQB_COUNT_LAUNCH();
    check_launch("solve_lambda_kernel");
}

void bundle_step_launch(BundleDev& b, const double* phi_out, const double* L, cudaStream_t s)
{
    StepArgs a{b.G.p, b.ldg, b.m, b.n, b.cap, L, b.Xb.p, phi_out, b.Fv.p, b.slot.p, b.slot_old.p,
               b.lam.p, b.gam.p, b.gtest.p, b.dstate.p, b.istate.p};
    bundle_step_kernel<<<1, LE_THREADS, 0, s>>>(a);
    BQB_COUNT_LAUNCH();
    check_launch("bundle_step_kernel");
}

void bundle_xcomb_launch(BundleDev& b, double* X, cudaStream_t s)
{
    const size_t nn = (size_t)b.n * b.n;
    int blocks = (int)((nn + 255) / 256);
    if (blocks > 4 * rt().num_sms) blocks = 4 * rt().num_sms;
    bundle_xcomb_kernel<<<blocks, 256, 0, s>>>(b.Xb.p, b.slot_old.p, b.lam.p, b.istate.p, X, nn);
    BQB_COUNT_LAUNCH();
    check_launch("bundle_xcomb_kernel");
}

void bundle_append_launch(BundleDev& b, cudaStream_t s)
{
    bundle_append_kernel<<<1, 32, 0, s>>>(b.slot.p, b.istate.p, b.cap);
    BQB_COUNT_LAUNCH();
    check_launch("bundle_append_kernel");
}

void bundle_fval_launch(BundleDev& b, const double* L, const int* slot_ptr, const int* pos_ptr, cudaStream_t s)
{
    bundle_fval_kernel<<<1, LE_THREADS, 0, s>>>(L, b.Xb.p, b.n, slot_ptr, pos_ptr, b.Fv.p);
    BQB_COUNT_LAUNCH();
    check_launch("bundle_fval_kernel");
}

}  // namespace bqb

using namespace bqb;

// The engines' lambda_eta counters (with bqb_engine_profile_enable(1)):
// out[6] = {calls, rounds of the lambda / eta alternation, sum of the bundle
// sizes k, SM cycles in the QP, SM cycles in the calls, sum of the cut
// counts m}; reset != 0 zeroes them after reading.  For profiling; no
// reference counterpart.
BQB_API void bqb_lambda_eta_profile(double* out, int reset)
{
    unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    std::lock_guard<std::mutex> lock(g_le_prof_mu);
    if (g_le_prof.p) {
        BQB_CUDA(cudaDeviceSynchronize());
        BQB_CUDA(cudaMemcpy(h, g_le_prof.p, sizeof(h), cudaMemcpyDeviceToHost));
        if (reset) BQB_CUDA(cudaMemset(g_le_prof.p, 0, sizeof(h)));
    }
    for (int i = 0; i < 6; ++i)
        if (out) out[i] = (double)h[i];
}
