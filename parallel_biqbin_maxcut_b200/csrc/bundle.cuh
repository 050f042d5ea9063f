// Proximal bundle method (src/bundle.c) on the device.
#pragma once
#include "../../include/bqb_gpu.h"
#include "bqb_common.cuh"
#include "cuts.cuh"

namespace bqb {

// Integer state words of a device bundle (BundleDev::istate).
enum BundleInt : int {
    BI_K = 0,          // bundle size (PP->bundle)
    BI_NEXT = 1,       // physical slot that receives the next X_test / g
    BI_KOLD = 2,       // bundle size before the last step (for X = X_bundle lambda)
    BI_SERIOUS = 3,    // last step was serious
    BI_ERR = 4,        // 1: bundle overflow (MaxBundle), 2: QP failure
    BI_CAP = 5,        // physical slot capacity
    BI_LAST = 6,       // slot written by the last fct_eval (X_test, g)
    BI_WORDS = 8
};
// Double state words (BundleDev::dstate).
enum BundleDbl : int { BD_F = 0, BD_T = 1, BD_FTEST = 2, BD_DEL = 3, BD_WORDS = 4 };

// Device-resident bundle of one node.  X_bundle and G are addressed
// through `slot` (bundle order -> physical slot), so purging and appending
// move only small index arrays: an evaluated X_test and its subgradient are
// written straight into a free physical slot.
struct BundleDev {
    int n = 0, m = 0;
    int cap = 0;                 // physical slots
    int ldg = 0;                 // leading dimension of G (>= m)
    DevBuf<double> Xb;           // cap * n * n
    DevBuf<double> G;            // ldg * cap
    DevBuf<double> Fv;           // cap (bundle order)
    DevBuf<int> slot, slot_old;  // cap
    DevBuf<double> lam;          // cap (bundle order of the step that produced it)
    DevBuf<double> gam, gtest, dgam, eta;  // m
    DevBuf<double> dstate;       // BD_WORDS
    DevBuf<int> istate;          // BI_WORDS
    DevBuf<double> qp_ws;        // QP scratch (global when k is large)
    // Grow physical capacity to >= need slots (keeps the first `keep` slots).
    void ensure_cap(int need, int n_, cudaStream_t s);
    void ensure_m(int m_, cudaStream_t s);
};

// lambda_eta (src/bundle.c:292-373) + gamma_test = gamma + dgamma, one CTA.
// When zeta_in is null, zeta = -F - G'gamma is formed first
// (src/bundle.c:57-63).  t is read and written through dstate[BD_T].
void lambda_eta_launch(BundleDev& b, const double* zeta_in, cudaStream_t s);

// solve_lambda (src/bundle.c:390-653) alone, one warp: Q (k x k, lower
// triangle used), c -> lambda.  *err set to 1 on a singular KKT system.
void solve_lambda_launch(int k, const double* Q, const double* c, double* lambda, int* err, cudaStream_t s);

// Serious / null step bookkeeping after fct_eval (src/bundle.c:75-234):
// f_test = phi + sum(gamma_test), del, the step decision, t update, purge,
// append of the slot the evaluation wrote (BI_NEXT), next free slot.
// phi_out: the IPM output word of the evaluation; L: PP->L.
void bundle_step_launch(BundleDev& b, const double* phi_out, const double* L, cudaStream_t s);

// X = X_bundle * lambda on a serious step (src/bundle.c:105-108); no-op
// after a null step (reads BI_SERIOUS on the device).
void bundle_xcomb_launch(BundleDev& b, double* X, cudaStream_t s);

// Append the element just evaluated into slot BI_NEXT at bundle position
// BI_K and choose the next free slot (src/bounding.c:291-318).
void bundle_append_launch(BundleDev& b, cudaStream_t s);

// F value <L, X> of bundle element stored in slot *slot_ptr
// (src/bounding.c:144-154): writes F[*pos_ptr].
void bundle_fval_launch(BundleDev& b, const double* L, const int* slot_ptr, const int* pos_ptr,
                        cudaStream_t s);

}  // namespace bqb
