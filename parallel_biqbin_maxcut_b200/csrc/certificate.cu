// FP64 certificate of a basic SDP bound: an upper bound on
// max { <L, X> : diag(X) = e, X psd } from a dual vector y, valid whatever y
// is.  For any y, <L, X> = e'y - <Diag(y) - L, X> <= e'y + n max(0,
// -lambda_min(Diag(y) - L)) on the feasible set (trace X = n).  The IPM's
// bound is e'y with Z = Diag(y) - L positive definite up to rounding; the
// certificate adds a rigorous FP64 lower bound on lambda_min(Z):
//
//   If the floating-point Cholesky factorisation of a symmetric n x n A runs
//   to completion, R'R = A + dA with |dA| <= g_{n+1} |R'| |R|, g_k = k u /
//   (1 - k u), u = 2^-53 (Higham, Accuracy and Stability of Numerical
//   Algorithms, 2nd ed., Theorem 10.3; fused multiply-adds only tighten it).
//   Since ||R||_F^2 = trace(R'R) <= trace(A) + g_{n+1} ||R||_F^2, ||dA||_2 <=
//   g_{n+1} ||R||_F^2 <= g_{n+1} / (1 - g_{n+1}) trace(A), and R'R psd gives
//   lambda_min(A) >= -g_{n+1} / (1 - g_{n+1}) trace(A).
//
// A = fl(Z + t I) is factored with t = 0 first and a growing shift only if
// that fails; forming its diagonal costs at most 2u (|Z_ii| + t) per entry,
// and the sum e'y is bounded by fl(sum y) + g_n sum |y|.  Underflow is not
// accounted for (the entries are far above it).  No reference counterpart:
// the reference's bound is its IPM's dual value.
#include <math.h>

#include "internal.h"

namespace bqb {

namespace {

constexpr int CERT_THREADS = 512;
constexpr int CERT_SHIFTS = 64;   // doublings of the shift
constexpr int CERT_BISECT = 40;   // halvings of the bracket [failed, passed]

__device__ __forceinline__ double gam_k(int k)
{
    const double ku = (double)k * 0x1p-53;
    return ku / (1.0 - ku);
}

// The Cholesky factorisation of fl(Diag(y) - L + t I) (lower triangle, in
// A) runs to completion: every pivot positive.  Every thread returns the
// same answer.
__device__ bool chol_passes(const double* __restrict__ L, const double* __restrict__ y, int n, double t,
                            double* __restrict__ A)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const size_t nn = (size_t)n * n;
    __syncthreads();   // (a previous attempt's reads of A are done)
    for (size_t e = tid; e < nn; e += nt) {
        const int i = (int)(e % n), j = (int)(e / n);
        if (i >= j) A[e] = i == j ? (y[i] - L[e]) + t : -L[e];
    }
    __syncthreads();
    for (int j = 0; j < n; ++j) {
        const double d = A[j + (size_t)j * n];
        if (!(d > 0.0)) return false;
        const double r = sqrt(d);
        __syncthreads();   // every thread has read the pivot
        for (int i = j + 1 + tid; i < n; i += nt) A[i + (size_t)j * n] /= r;
        if (tid == 0) A[j + (size_t)j * n] = r;
        __syncthreads();
        const int m = n - j - 1;
        for (size_t q = tid; q < (size_t)m * m; q += nt) {
            const int i = j + 1 + (int)(q % m), k = j + 1 + (int)(q / m);
            if (i >= k) A[i + (size_t)k * n] = fma(-A[i + (size_t)j * n], A[k + (size_t)j * n], A[i + (size_t)k * n]);
        }
        __syncthreads();
    }
    return true;
}

// out: [0] certified bound, [1] the lower bound on lambda_min(Diag(y) - L),
// [2] the shift t of the factorisation that ran through, [3] status (0, or
// 1 when no shift up to 2^63 trace passed).  A: n x n scratch.
__global__ void __launch_bounds__(CERT_THREADS) cert_kernel(const double* __restrict__ L, const double* __restrict__ y,
                                                            int n, double* __restrict__ A, double* __restrict__ out)
{
    __shared__ double red[64];
    const int tid = threadIdx.x, nt = blockDim.x;
    double sy = 0.0, say = 0.0, tr = 0.0, mz = 0.0;
    for (int i = tid; i < n; i += nt) {
        const double z = y[i] - L[i + (size_t)i * n];
        sy += y[i];
        say += fabs(y[i]);
        tr += fabs(z);
        mz = fmax(mz, fabs(z));
    }
    sy = block_sum(sy, red);
    say = block_sum(say, red);
    tr = block_sum(tr, red);
    mz = block_max(mz, red);
    // (trace and sums up to a relative 2 n u of their computed values)
    const double slack = 1.0 + 4.0 * n * 0x1p-53;
    // the smallest shift that factors: 0, else doubling from tr 2^-40, then
    // bisection between the last shift that failed and the first that passed
    double t = 0.0;
    bool ok = chol_passes(L, y, n, 0.0, A);
    if (!ok) {
        double lo = 0.0;
        t = fmax(tr, 1.0) * 0x1p-40;
        for (int k = 0; k < CERT_SHIFTS && !(ok = chol_passes(L, y, n, t, A)); ++k) {
            lo = t;
            t *= 2.0;
        }
        if (ok)
            for (int k = 0; k < CERT_BISECT; ++k) {
                const double mid = 0.5 * (lo + t);
                if (!(mid > lo && mid < t)) break;
                if (chol_passes(L, y, n, mid, A))
                    t = mid;
                else
                    lo = mid;
            }
    }
    double lam = -INFINITY;
    if (ok) {
        const double g = gam_k(n + 1);
        const double trA = (tr + n * t) * slack;
        lam = -(g / (1.0 - g) * trA + t + 2.0 * 0x1p-53 * (mz + t)) * slack;
    }
    const int status = ok ? 0 : 1;
    if (tid == 0) {
        const double corr = lam < 0.0 ? n * -lam : 0.0;
        const double v = sy + gam_k(n) * say * slack + corr;
        out[0] = status == 0 ? v + fabs(v) * 0x1p-50 : INFINITY;   // (the last sums' rounding)
        out[1] = lam;
        out[2] = t;
        out[3] = (double)status;
    }
}

}  // namespace

void sdp_certificate(DevBuf<double>& ws, const double* dL, const double* dy, int n, double* dout, cudaStream_t s)
{
    double* A = ws.ensure((size_t)n * n);
    cert_kernel<<<1, CERT_THREADS, 0, s>>>(dL, dy, n, A, dout);
    BQB_COUNT_LAUNCH();
    check_launch("cert_kernel");
}

}  // namespace bqb

namespace {
// Device buffers of one C-ABI call, freed when it returns.
struct CallBufs {
    bqb::DevBuf<double> b[5];
    ~CallBufs()
    {
        for (auto& x : b)
            if (x.p) cudaFree(x.p);
    }
};
}  // namespace

using namespace bqb;

// Certified basic SDP bound of L (n x n, column-major, host) from a dual
// vector y (host): out[0] = an upper bound on max <L, X> over diag(X) = e,
// X psd, valid for any y (the sum of y plus n times the FP64 lower bound on
// -lambda_min(Diag(y) - L) when that is negative, with every rounding error
// bounded); out[1] = that lower bound on lambda_min; out[2] = the diagonal
// shift the certificate's Cholesky factorisation needed (0 when Diag(y) - L
// factors as it is); out[3] = 0, or 1 when no shift worked.  Returns 0, or 1
// on bad arguments.  No reference counterpart.
BQB_API int bqb_sdp_certificate(const double* L, const double* y, int n, double* out)
{
    if (!L || !y || !out || n < 1) {
        set_error("bqb_sdp_certificate", "L, y and out must be non-null and n >= 1");
        return 1;
    }
    Runtime& R = rt();
    const size_t nn = (size_t)n * n;
    CallBufs cb;
    DevBuf<double>&dL = cb.b[0], &dy = cb.b[1], &dout = cb.b[2], &ws = cb.b[3];
    BQB_CUDA(cudaMemcpyAsync(dL.ensure(nn), L, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    BQB_CUDA(cudaMemcpyAsync(dy.ensure(n), y, n * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    sdp_certificate(ws, dL.p, dy.p, n, dout.ensure(4), R.stream);
    BQB_CUDA(cudaMemcpyAsync(out, dout.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaStreamSynchronize(R.stream));
    return 0;
}

// ipm_mc_pk (src/ipm_mc_pk.c:28-359) that also returns the dual vector y of
// its last iterate (host y, n doubles; phi = its sum in the IPM's order):
// out[0..3] = phi, iterations, status, <L, X>.  X may be NULL.  Returns 0,
// or 1 on bad arguments.  No reference counterpart (the reference keeps y
// inside the IPM).
BQB_API int bqb_ipm_dual(const double* L, int n, double* X, double* y, double* out)
{
    if (!L || !y || !out || n < 1) {
        set_error("bqb_ipm_dual", "L, y and out must be non-null and n >= 1");
        return 1;
    }
    Runtime& R = rt();
    const size_t nn = (size_t)n * n;
    CallBufs cb;
    DevBuf<double>&dL = cb.b[0], &dX = cb.b[1], &dy = cb.b[2], &dout = cb.b[3], &ws = cb.b[4];
    BQB_CUDA(cudaMemcpyAsync(dL.ensure(nn), L, nn * sizeof(double), cudaMemcpyHostToDevice, R.stream));
    ipm_device(ws, dL.p, dX.ensure(nn), n, dout.ensure(4), R.stream, nullptr, dy.ensure(n));
    if (X) BQB_CUDA(cudaMemcpyAsync(X, dX.p, nn * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaMemcpyAsync(y, dy.p, n * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaMemcpyAsync(out, dout.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaStreamSynchronize(R.stream));
    return 0;
}
