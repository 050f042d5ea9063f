// Basic Max-Cut SDP interior-point method on the GPU: one CTA per problem,
// the whole predictor-corrector loop inside one launch.
#pragma once
#include "bqb_common.cuh"

namespace bqb {

constexpr int IPM_THREADS = 512;
constexpr int IPM_MAX_ITERS = 500;    // reference loops until gap <= 1e-2 with no cap
constexpr int IPM_MAX_TRIALS = 200;   // line-search halvings (0.8^200 ~ 4e-20)

// Status codes written to out[2] (0 = converged).
enum IpmStatus : int {
    IPM_OK = 0,
    IPM_Z_NOT_PD = 1,        // src/ipm_mc_pk.c:132-136 (dpotrf of Z failed)
    IPM_M_NOT_PD = 2,        // src/ipm_mc_pk.c:169-173 (dposv of Zi.*X failed)
    IPM_LINESEARCH = 3,      // line search did not find a PD step
    IPM_MAXITER = 4,
    IPM_SYNC = 5,            // n > 128: a grid barrier gave up waiting (2 s)
};

// One problem.  L: n x n column-major (ld = n), read only.  X: n x n output.
// ws: per-problem scratch of ipm_ws_doubles(n, place) doubles.
// out[0] = phi (dual value e'y), out[1] = iterations, out[2] = status,
// out[3] = final primal value <L,X>; yout (optional): y (phi = sum of y, in
// the IPM's order).  xslot (optional, device): the output
// matrix is X + (*xslot) * n * n, so a bundle can direct the result into a
// free slot chosen on the device.
struct IpmDesc {
    const double* L;
    double* X;
    double* ws;
    double* out;
    const int* xslot;
    int n;
    int pad_;
    double* yout = nullptr;   // (optional) the dual vector y of the last iterate, n doubles
};

// Shared-memory placement flags chosen on the host from the largest n of a
// launch: bit 0 = Cholesky workspace F in smem, bit 1 = Zi in smem.
int ipm_place(int n_max, size_t smem_limit, size_t* smem_bytes);
size_t ipm_ws_doubles(int n, int place);

// Launch the batched kernel over `nprob` descriptors already on the device.
void ipm_launch(const IpmDesc* d_descs, int nprob, int n_max, cudaStream_t s);
// Single problem: descriptor passed by value.
void ipm_launch_one(const IpmDesc& d, cudaStream_t s);
// Single problem with placement chosen by the caller; returns the launch
// status instead of raising it.
cudaError_t ipm_launch_prepared(const IpmDesc& d, int place, size_t smem_bytes, cudaStream_t s);

// Device address of the IPM work counters (for kernels in other files that
// run the IPM body).
double* ipm_stats_device();

}  // namespace bqb
