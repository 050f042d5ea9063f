// The basic SDP interior-point method (src/ipm_mc_pk.c:28-359) for n above
// the register-resident limit (IPM_REG_NMAX = 128): the steps of
// ipm_body_reg, orchestrated from the host, each step a multi-CTA kernel, so
// that a factorisation is no longer paced by one SM reading global memory.
//
// Inverses (Zi = inv(Z), F = inv(Zi .* X)) use a blocked symmetric
// Gauss-Jordan sweep on panels of WL_B columns.  For a panel K with
// D = A_KK = Ld Ld^T (Cholesky in one CTA) and the columns C = A(:, K):
// V = C Ld^{-T}, A_ij -= V_i V_j^T (i, j not in K), A_iK = V_i Ld^{-1}
// (= C_i D^{-1}), A_KK = -D^{-1}; after the last panel A = -inv(A).  The
// Cholesky pivots are the Schur complements of A: a non-positive one means
// "not positive definite" and sets a flag.  The line searches' positive-
// definiteness tests run the trailing part of the same sweep only, which is
// a blocked right-looking Cholesky.  Going through Ld rather than the
// explicit D^{-1} matters: at n = 343 with couplings of 1e5, M reaches a
// condition number of 1e11 at the last iteration, and C D^{-1} C^T then
// turned a pivot of the positive definite M negative.
// Products with F replace the Cholesky solves, as in ipm_body_reg, each
// followed by one step of iterative refinement with M = Zi .* X
// (x <- x + F (b - M x)).
#include <math.h>

#include "bqb_common.cuh"
#include "internal.h"
#include "ipm.cuh"

namespace bqb {

double* ipm_stats_device();

namespace {

constexpr int WL_B = 32;     // panel width
constexpr int WL_T = 256;    // threads per CTA of the elementwise kernels
constexpr int WL_TILE = 32;  // tile of the update and GEMM kernels

unsigned wl_blocks(long long count) { return (unsigned)((count + WL_T - 1) / WL_T); }

// y_c = sum_r |L_rc| + 1.1, zd_c = y_c - L_cc (src/ipm_mc_pk.c:65-89)
__global__ void wl_init_vec(const double* __restrict__ L, int n, double* __restrict__ y, double* __restrict__ zd)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double acc = 0.0;
    const double* Lc = L + (size_t)c * n;
    for (int r = 0; r < n; ++r) acc += fabs(Lc[r]);
    y[c] = acc + 1.1;
    zd[c] = y[c] - L[c + (size_t)c * n];
}

__global__ void wl_identity(double* __restrict__ X, int n)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)n * n) return;
    X[e] = (e % n == e / n) ? 1.0 : 0.0;
}

// One CTA: sc[0] = sum_i a_i, sc[1] = sum_i b_i, sc[2] = sum_i c_i over
// vectors of n, or, with mode 1, the update sums zx, lx, ysum of
// src/ipm_mc_pk.c:313-334 over X (n x n), L, zd, y.
__global__ void wl_sums(int mode, int n, const double* __restrict__ L, const double* __restrict__ X,
                        const double* __restrict__ y, const double* __restrict__ zd, double* __restrict__ sc)
{
    __shared__ double red[64];
    double a = 0.0, b = 0.0, c = 0.0;
    if (mode == 0) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            a += L[i + (size_t)i * n];
            b += zd[i];
            c += y[i];
        }
    } else {
        const size_t nn = (size_t)n * n;
        for (size_t e = threadIdx.x; e < nn; e += blockDim.x) {
            const double xv = X[e], lv = L[e];
            b = fma(lv, xv, b);                       // lx
            if (e % n != e / n) a = fma(-lv, xv, a);  // zx, off-diagonal part
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            a = fma(zd[i], X[i + (size_t)i * n], a);
            c += y[i];
        }
    }
    a = block_sum(a, red);
    b = block_sum(b, red);
    c = block_sum(c, red);
    if (threadIdx.x == 0) {
        sc[0] = a;
        sc[1] = b;
        sc[2] = c;
    }
}

// A = Diag(d + alpha dd) - L off the diagonal (dd may be null)
__global__ void wl_fill_z(const double* __restrict__ L, const double* __restrict__ d, const double* __restrict__ dd,
                          double alpha, int n, double* __restrict__ A)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)n * n) return;
    const int i = (int)(e % n), j = (int)(e / n);
    A[e] = i == j ? (dd ? fma(alpha, dd[i], d[i]) : d[i]) : -L[e];
}

// A = X + alpha dX
__global__ void wl_axpy(const double* __restrict__ X, const double* __restrict__ dX, double alpha, size_t nn,
                        double* __restrict__ A)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nn) A[e] = fma(alpha, dX[e], X[e]);
}

__global__ void wl_hadamard(const double* __restrict__ A, const double* __restrict__ B, size_t nn,
                            double* __restrict__ C)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nn) C[e] = A[e] * B[e];
}

__global__ void wl_negate(double* __restrict__ A, size_t nn)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nn) A[e] = -A[e];
}

// ---- panel sweep ---------------------------------------------------------

// One CTA: the Cholesky factor Ld of D = A[K, K] (b x b) by sequential
// rank-1 updates in shared memory, Linv = Ld^{-1} (forward substitution,
// one column per thread) and Dinv = Linv^T Linv.  A non-positive pivot sets
// *flag.  Linv and Dinv are stored with leading dimension WL_B.
__global__ void wl_panel_factor(const double* __restrict__ A, int n, int k0, int b, double* __restrict__ Linv,
                                double* __restrict__ Dinv, double* __restrict__ flag)
{
    __shared__ double S[WL_B][WL_B + 1];
    __shared__ double Li[WL_B][WL_B + 1];
    const int tid = threadIdx.x;
    for (int e = tid; e < WL_B * WL_B; e += blockDim.x) {
        const int p = e % WL_B, q = e / WL_B;
        S[p][q] = p < b && q < b ? A[(k0 + p) + (size_t)(k0 + q) * n] : 0.0;
        Li[p][q] = 0.0;
    }
    __syncthreads();
    bool pd = true;
    // S becomes Ld column by column (lower triangle; the strict upper
    // triangle keeps stale values and is not read)
    for (int q = 0; q < b; ++q) {
        const double d = S[q][q];
        if (!(d > 0.0)) {   // d is the same value in every thread: all leave together
            if (tid == 0) *flag = 1.0;
            pd = false;
            break;
        }
        const double l = sqrt(d);
        __syncthreads();
        if (tid >= q && tid < b) S[tid][q] = tid == q ? l : S[tid][q] / l;
        __syncthreads();
        for (int e = tid; e < b * b; e += blockDim.x) {
            const int p = e % b, r = e / b;
            if (p > q && r > q && r <= p) S[p][r] -= S[p][q] * S[r][q];
        }
        __syncthreads();
    }
    if (!pd) return;
    // Li(:, t) = Ld^{-1} e_t: rows t..b-1, in order
    if (tid < b) {
        const int t = tid;
        for (int i = t; i < b; ++i) {
            double acc = i == t ? 1.0 : 0.0;
            for (int k = t; k < i; ++k) acc = fma(-S[i][k], Li[k][t], acc);
            Li[i][t] = acc / S[i][i];
        }
    }
    __syncthreads();
    for (int e = tid; e < WL_B * WL_B; e += blockDim.x) {
        const int p = e % WL_B, q = e / WL_B;
        Linv[p + (size_t)q * WL_B] = Li[p][q];
        double acc = 0.0;
        for (int k = p > q ? p : q; k < b; ++k) acc = fma(Li[k][p], Li[k][q], acc);
        Dinv[p + (size_t)q * WL_B] = acc;
    }
}

// One warp per row i outside the panel, lane q: V(i, q) = sum_{p <= q}
// A(i, k0 + p) Linv(q, p) (V = C Ld^{-T}) and, with `full`, W(i, q) =
// sum_{p >= q} V(i, p) Linv(p, q) (W = V Ld^{-1} = C D^{-1}; formed from V,
// not as C times the explicit D^{-1}, whose rounding near convergence at
// n = 343 sent the iteration off).  Panel rows get V = W = 0.
__global__ void wl_panel_vw(const double* __restrict__ A, int n, int k0, int b, const double* __restrict__ Linv,
                            int full, double* __restrict__ V, double* __restrict__ W)
{
    const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;   // whole warps leave together
    const bool outside = i < k0 || i >= k0 + b;
    const double c = outside && lane < b ? A[i + (size_t)(k0 + lane) * n] : 0.0;
    double v = 0.0;
    for (int p = 0; p < b; ++p) {
        const double cp = __shfl_sync(0xffffffffu, c, p);
        if (p <= lane) v = fma(cp, Linv[lane + (size_t)p * WL_B], v);
    }
    if (lane < b) V[i + (size_t)lane * n] = v;
    if (!full) return;
    double w = 0.0;
    for (int p = 0; p < b; ++p) {
        const double vp = __shfl_sync(0xffffffffu, v, p);
        if (p >= lane) w = fma(vp, Linv[p + (size_t)lane * WL_B], w);
    }
    if (lane < b) W[i + (size_t)lane * n] = w;
}

// A(i, j) -= sum_q V(i, q) V(j, q) for i, j outside the panel (with
// `trailing`, only i, j >= k0 + b): the Schur complement through the
// panel's Cholesky factor, which keeps the trailing pivots as accurate as
// a blocked Cholesky (the form C D^{-1} C^T loses ~eps cond(D) and turned
// pivots of a positive definite M negative at cond 1e11).  32 x 32 tiles,
// 256 threads, 4 entries each; the product is symmetric in i and j.
__global__ void wl_panel_update(double* __restrict__ A, int n, int k0, int b, const double* __restrict__ V,
                                int trailing)
{
    __shared__ double si[WL_TILE][WL_B + 1];
    __shared__ double sj[WL_TILE][WL_B + 1];
    const int i0 = blockIdx.x * WL_TILE, j0 = blockIdx.y * WL_TILE;
    const int lo = trailing ? k0 + b : 0;
    if (i0 + WL_TILE <= lo || j0 + WL_TILE <= lo) return;
    const int tid = threadIdx.x;
    for (int e = tid; e < WL_TILE * b; e += blockDim.x) {
        const int r = e % WL_TILE, q = e / WL_TILE;
        const int i = i0 + r, j = j0 + r;
        si[r][q] = i < n ? V[i + (size_t)q * n] : 0.0;
        sj[r][q] = j < n ? V[j + (size_t)q * n] : 0.0;
    }
    __syncthreads();
    const int r = tid % WL_TILE, c0 = tid / WL_TILE;   // c0 in 0..7
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int c = c0 + 8 * t;
        const int i = i0 + r, j = j0 + c;
        if (i >= n || j >= n || i < lo || j < lo) continue;
        if ((i >= k0 && i < k0 + b) || (j >= k0 && j < k0 + b)) continue;
        double acc = 0.0;
        for (int q = 0; q < b; ++q) acc = fma(si[r][q], sj[c][q], acc);
        A[i + (size_t)j * n] -= acc;
    }
}

// A(i, K) = A(K, i)^T = W(i, :) for i outside the panel; A(K, K) = -Dinv.
__global__ void wl_panel_fix(double* __restrict__ A, int n, int k0, int b, const double* __restrict__ W,
                             const double* __restrict__ Dinv)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n * b) return;
    const int i = (int)(e % n), q = (int)(e / n);
    if (i >= k0 && i < k0 + b) {
        const int p = i - k0;
        A[i + (size_t)(k0 + q) * n] = -Dinv[p + (size_t)q * WL_B];
    } else {
        const double v = W[i + (size_t)q * n];
        A[i + (size_t)(k0 + q) * n] = v;
        A[(k0 + q) + (size_t)i * n] = v;
    }
}

// ---- products --------------------------------------------------------------

// out = F v (v null: v = -e); one warp per row r, reading column r (F is
// symmetric).
__global__ void wl_matvec(const double* __restrict__ F, int n, const double* __restrict__ v, double* __restrict__ out)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double* col = F + (size_t)warp * n;
    double acc = 0.0;
    for (int c = lane; c < n; c += 32) acc = fma(col[c], v ? v[c] : -1.0, acc);
    acc = warp_sum(acc);
    if (lane == 0) out[warp] = acc;
}

// rhs_r = mu Zi_rr - sum_c Zi_rc dX1_rc dy1_c (columns r by symmetry)
// r = b - M x (b null: b = -e); one warp per row (columns by symmetry)
__global__ void wl_resid(const double* __restrict__ M, int n, const double* __restrict__ b,
                         const double* __restrict__ x, double* __restrict__ r)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double* col = M + (size_t)warp * n;
    double acc = 0.0;
    for (int c = lane; c < n; c += 32) acc = fma(col[c], x[c], acc);
    acc = warp_sum(acc);
    if (lane == 0) r[warp] = (b ? b[warp] : -1.0) - acc;
}

__global__ void wl_rhs(const double* __restrict__ Zi, const double* __restrict__ dX1, const double* __restrict__ dy1,
                       double mu, int n, double* __restrict__ rhs)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const size_t o = (size_t)warp * n;
    double acc = 0.0;
    for (int c = lane; c < n; c += 32) acc = fma(Zi[o + c] * dX1[o + c], dy1[c], acc);
    acc = warp_sum(acc);
    if (lane == 0) rhs[warp] = mu * Zi[o + warp] - acc;
}

// out(r, c) = sum_k Zi(r, k) (a_k X(k, c) + b_k Y(k, c)) + e1 E1(r, c) + e2 E2(r, c)
// (b, Y, E2 may be null).  32 x 32 tiles, k in chunks of 32.
__global__ void wl_gemm(const double* __restrict__ Zi, const double* __restrict__ a, const double* __restrict__ X,
                        const double* __restrict__ bv, const double* __restrict__ Y, double e1,
                        const double* __restrict__ E1, double e2, const double* __restrict__ E2, int n,
                        double* __restrict__ out)
{
    __shared__ double sa[WL_TILE][WL_TILE + 1];
    __shared__ double sb[WL_TILE][WL_TILE + 1];
    const int r0 = blockIdx.x * WL_TILE, c0 = blockIdx.y * WL_TILE;
    const int tid = threadIdx.x;
    const int r = tid % WL_TILE, cc = tid / WL_TILE;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k0 = 0; k0 < n; k0 += WL_TILE) {
        for (int e = tid; e < WL_TILE * WL_TILE; e += blockDim.x) {
            const int p = e % WL_TILE, q = e / WL_TILE;
            const int rr = r0 + p, kk = k0 + q;
            sa[p][q] = (rr < n && kk < n) ? Zi[rr + (size_t)kk * n] : 0.0;
            const int kb = k0 + p, cb = c0 + q;
            double v = 0.0;
            if (kb < n && cb < n) {
                const size_t idx = kb + (size_t)cb * n;
                v = a[kb] * X[idx];
                if (bv) v = fma(bv[kb], Y[idx], v);
            }
            sb[p][q] = v;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < WL_TILE; ++k) {
            const double av = sa[r][k];
#pragma unroll
            for (int t = 0; t < 4; ++t) acc[t] = fma(av, sb[k][cc + 8 * t], acc[t]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int rr = r0 + r, c = c0 + cc + 8 * t;
        if (rr >= n || c >= n) continue;
        const size_t idx = rr + (size_t)c * n;
        double v = acc[t] + e1 * E1[idx];
        if (E2) v += e2 * E2[idx];
        out[idx] = v;
    }
}

__global__ void wl_symmetrize(double* __restrict__ A, int n)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)n * n) return;
    const int i = (int)(e % n), j = (int)(e / n);
    if (i <= j) return;
    const double v = 0.5 * (A[i + (size_t)j * n] + A[j + (size_t)i * n]);
    A[i + (size_t)j * n] = v;
    A[j + (size_t)i * n] = v;
}

// out = alpha a
__global__ void wl_scale(const double* __restrict__ a, double alpha, int n, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = alpha * a[i];
}

// c = a + b elementwise; c may be a (no __restrict__ on a and c)
__global__ void wl_vadd(const double* a, const double* __restrict__ b, int n, double* c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) c[i] = a[i] + b[i];
}

// X += ap dX; y += ad dy; zd += ad dy
__global__ void wl_step(double* __restrict__ X, const double* __restrict__ dX, double ap, size_t nn,
                        double* __restrict__ y, double* __restrict__ zd, const double* __restrict__ dy, double ad,
                        int n)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nn) X[e] = fma(ap, dX[e], X[e]);
    if (e < (size_t)n) {
        y[e] = fma(ad, dy[e], y[e]);
        zd[e] = fma(ad, dy[e], zd[e]);
    }
}

__global__ void wl_out(double* __restrict__ out, double phi, int iter, int status, double psi, double* stats,
                       double n3, int ls_total)
{
    out[0] = phi;
    out[1] = (double)iter;
    out[2] = (double)status;
    out[3] = psi;
    if (stats) {
        atomicAdd(&stats[0], iter * n3);
        atomicAdd(&stats[1], 1.0);
        atomicAdd(&stats[2], (double)iter);
        atomicAdd(&stats[3], (double)ls_total);
    }
}

}  // namespace

namespace {

struct WlBufs {
    double *Zi, *F, *M, *T, *dX, *dX1, *W, *V, *Dinv, *Linv, *y, *zd, *dy, *dy1, *dy2, *r, *t, *sc, *flag;
};

// The panel sweep of A (n x n) on stream s.  full: the whole sweep (A
// becomes inv(A)); otherwise only the trailing updates, for the pivots.
// Non-positive pivots set *flag (not cleared here).
void wl_sweep(double* A, int n, bool full, const WlBufs& w, cudaStream_t s)
{
    const unsigned tiles = (unsigned)((n + WL_TILE - 1) / WL_TILE);
    for (int k0 = 0; k0 < n; k0 += WL_B) {
        const int b = n - k0 < WL_B ? n - k0 : WL_B;
        wl_panel_factor<<<1, WL_T, 0, s>>>(A, n, k0, b, w.Linv, w.Dinv, w.flag);
        BQB_COUNT_LAUNCH();
        if (!full && k0 + b >= n) break;
        wl_panel_vw<<<wl_blocks((long long)n * 32), WL_T, 0, s>>>(A, n, k0, b, w.Linv, full ? 1 : 0, w.V, w.W);
        BQB_COUNT_LAUNCH();
        wl_panel_update<<<dim3(tiles, tiles), WL_T, 0, s>>>(A, n, k0, b, w.V, full ? 0 : 1);
        BQB_COUNT_LAUNCH();
        if (full) {
            wl_panel_fix<<<wl_blocks((long long)n * b), WL_T, 0, s>>>(A, n, k0, b, w.W, w.Dinv);
            BQB_COUNT_LAUNCH();
        }
    }
    if (full) {
        wl_negate<<<wl_blocks((long long)n * n), WL_T, 0, s>>>(A, (size_t)n * n);
        BQB_COUNT_LAUNCH();
    }
    check_launch("ipm_large sweep");
}

double read_flag(const WlBufs& w, cudaStream_t s)
{
    double f = 0.0;
    BQB_CUDA(cudaMemcpyAsync(&f, w.flag, sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    return f;
}

}  // namespace

size_t ipm_large_ws_doubles(int n)
{
    const size_t nn = (size_t)n * n;
    return 6 * nn + 2 * (size_t)n * WL_B + 2 * (size_t)WL_B * WL_B + 8 * (size_t)n + 16;
}

// ipm_mc_pk for n > IPM_REG_NMAX: the same steps as ipm_body_reg, each a
// multi-CTA kernel on stream s; synchronises with the host at every
// positive-definiteness decision.  xslot (optional, device): write X into
// dXbase + (*xslot) * n * n.  Results in dout[0..3] (phi, iterations,
// status, psi).
void ipm_large(DevBuf<double>& wsbuf, const double* L, double* Xbase, int n, double* dout, cudaStream_t s,
               const int* xslot)
{
    const size_t nn = (size_t)n * n;
    double* p = wsbuf.ensure(ipm_large_ws_doubles(n));
    WlBufs w;
    w.Zi = p;
    w.F = w.Zi + nn;
    w.M = w.F + nn;
    w.T = w.M + nn;
    w.dX = w.T + nn;
    w.dX1 = w.dX + nn;
    w.W = w.dX1 + nn;
    w.V = w.W + (size_t)n * WL_B;
    w.Dinv = w.V + (size_t)n * WL_B;
    w.Linv = w.Dinv + (size_t)WL_B * WL_B;
    w.y = w.Linv + (size_t)WL_B * WL_B;
    w.zd = w.y + n;
    w.dy = w.zd + n;
    w.dy1 = w.dy + n;
    w.dy2 = w.dy1 + n;
    w.r = w.dy2 + n;
    w.t = w.r + n;
    w.sc = w.t + n;
    w.flag = w.sc + 8;
    double* X = Xbase;
    if (xslot) {
        int slot = 0;
        BQB_CUDA(cudaMemcpyAsync(&slot, xslot, sizeof(int), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaStreamSynchronize(s));
        X += (size_t)slot * nn;
    }
    const unsigned bn = wl_blocks(n), bnn = wl_blocks((long long)nn), bw = wl_blocks((long long)n * 32);
    const unsigned tiles = (unsigned)((n + WL_TILE - 1) / WL_TILE);
    double hs[3];
    // x = M^{-1} b (b null: -e): x = F b, then one refinement step
    auto solve = [&](const double* b, double* x) {
        wl_matvec<<<bw, WL_T, 0, s>>>(w.F, n, b, x);
        BQB_COUNT_LAUNCH();
        wl_resid<<<bw, WL_T, 0, s>>>(w.M, n, b, x, w.r);
        BQB_COUNT_LAUNCH();
        wl_matvec<<<bw, WL_T, 0, s>>>(w.F, n, w.r, w.t);
        BQB_COUNT_LAUNCH();
        wl_vadd<<<bn, WL_T, 0, s>>>(x, w.t, n, x);
        BQB_COUNT_LAUNCH();
    };
    auto sums = [&](int mode) {
        wl_sums<<<1, 1024, 0, s>>>(mode, n, L, X, w.y, w.zd, w.sc);
        BQB_COUNT_LAUNCH();
        BQB_CUDA(cudaMemcpyAsync(hs, w.sc, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaStreamSynchronize(s));
    };

    // ---- initial point (src/ipm_mc_pk.c:65-99) ----
    wl_init_vec<<<bn, WL_T, 0, s>>>(L, n, w.y, w.zd);
    BQB_COUNT_LAUNCH();
    wl_identity<<<bnn, WL_T, 0, s>>>(X, n);
    BQB_COUNT_LAUNCH();
    sums(0);
    double psi = hs[0];
    double mu = hs[1] / (2.0 * n);
    double phi = hs[2];
    double gap = fabs(phi - psi);
    int iter = 0, ls_total = 0, status = IPM_OK;

    while (gap > 1e-2) {
        if (++iter > IPM_MAX_ITERS) {
            status = IPM_MAXITER;
            break;
        }
        BQB_CUDA(cudaMemsetAsync(w.flag, 0, sizeof(double), s));
        // Zi = inv(Z), Z = Diag(zd) - L off the diagonal
        wl_fill_z<<<bnn, WL_T, 0, s>>>(L, w.zd, nullptr, 0.0, n, w.Zi);
        BQB_COUNT_LAUNCH();
        wl_sweep(w.Zi, n, true, w, s);
        if (read_flag(w, s) != 0.0) {
            status = IPM_Z_NOT_PD;
            break;
        }
        // F = inv(Zi .* X); dy1 = F (-e)
        wl_hadamard<<<bnn, WL_T, 0, s>>>(w.Zi, X, nn, w.M);
        BQB_COUNT_LAUNCH();
        BQB_CUDA(cudaMemcpyAsync(w.F, w.M, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
        wl_sweep(w.F, n, true, w, s);
        if (read_flag(w, s) != 0.0) {
            status = IPM_M_NOT_PD;
            break;
        }
        solve(nullptr, w.dy1);
        // dX1 = Zi (-Diag(dy1) X) - X, symmetrised; the sign goes into the
        // row scale: a_k = -dy1_k
        wl_scale<<<bn, WL_T, 0, s>>>(w.dy1, -1.0, n, w.dy2);   // dy2 = -dy1 (scratch)
        BQB_COUNT_LAUNCH();
        wl_gemm<<<dim3(tiles, tiles), WL_T, 0, s>>>(w.Zi, w.dy2, X, nullptr, nullptr, -1.0, X, 0.0, nullptr, n,
                                                     w.dX1);
        BQB_COUNT_LAUNCH();
        wl_symmetrize<<<bnn, WL_T, 0, s>>>(w.dX1, n);
        BQB_COUNT_LAUNCH();
        // corrector: rhs = mu diag(Zi) - (Zi .* dX1) dy1; dy2 = F rhs
        wl_rhs<<<bw, WL_T, 0, s>>>(w.Zi, w.dX1, w.dy1, mu, n, w.dy);
        BQB_COUNT_LAUNCH();
        solve(w.dy, w.dy2);
        // dX = Zi (-Diag(dy2) X - Diag(dy1) dX1) + mu Zi + dX1, symmetrised
        wl_scale<<<bn, WL_T, 0, s>>>(w.dy2, -1.0, n, w.dy);   // dy = -dy2
        BQB_COUNT_LAUNCH();
        wl_scale<<<bn, WL_T, 0, s>>>(w.dy1, -1.0, n, w.T);    // T[0..n) = -dy1 (T is free here)
        BQB_COUNT_LAUNCH();
        wl_gemm<<<dim3(tiles, tiles), WL_T, 0, s>>>(w.Zi, w.dy, X, w.T, w.dX1, 1.0, w.dX1, mu, w.Zi, n, w.dX);
        BQB_COUNT_LAUNCH();
        wl_symmetrize<<<bnn, WL_T, 0, s>>>(w.dX, n);
        BQB_COUNT_LAUNCH();
        wl_vadd<<<bn, WL_T, 0, s>>>(w.dy1, w.dy2, n, w.dy);
        BQB_COUNT_LAUNCH();

        // primal line search: X + ap dX positive definite
        double ap = 1.0;
        int trials = 0;
        bool ok = false;
        while (true) {
            BQB_CUDA(cudaMemsetAsync(w.flag, 0, sizeof(double), s));
            wl_axpy<<<bnn, WL_T, 0, s>>>(X, w.dX, ap, nn, w.T);
            BQB_COUNT_LAUNCH();
            wl_sweep(w.T, n, false, w, s);
            if (read_flag(w, s) == 0.0) {
                ok = true;
                break;
            }
            if (++trials >= IPM_MAX_TRIALS) break;
            ap *= 0.8;
        }
        ls_total += trials + 1;
        if (!ok) {
            status = IPM_LINESEARCH;
            break;
        }
        if (ap < 1.0) ap *= 0.95;
        // dual line search: Z + ad Diag(dy) positive definite
        double ad = 1.0;
        trials = 0;
        ok = false;
        while (true) {
            BQB_CUDA(cudaMemsetAsync(w.flag, 0, sizeof(double), s));
            wl_fill_z<<<bnn, WL_T, 0, s>>>(L, w.zd, w.dy, ad, n, w.T);
            BQB_COUNT_LAUNCH();
            wl_sweep(w.T, n, false, w, s);
            if (read_flag(w, s) == 0.0) {
                ok = true;
                break;
            }
            if (++trials >= IPM_MAX_TRIALS) break;
            ad *= 0.8;
        }
        ls_total += trials + 1;
        if (!ok) {
            status = IPM_LINESEARCH;
            break;
        }
        if (ad < 1.0) ad *= 0.95;

        // update (src/ipm_mc_pk.c:313-334)
        wl_step<<<bnn, WL_T, 0, s>>>(X, w.dX, ap, nn, w.y, w.zd, w.dy, ad, n);
        BQB_COUNT_LAUNCH();
        sums(1);
        mu = hs[0] / (2.0 * n);
        if (ap + ad > 1.6) mu *= 0.5;
        if (ap + ad > 1.9) mu *= 0.2;
        phi = hs[2];
        psi = hs[1];
        gap = fabs(phi - psi);
    }
    wl_out<<<1, 1, 0, s>>>(dout, phi, iter, status, psi, ipm_stats_device(), (double)n * n * n, ls_total);
    BQB_COUNT_LAUNCH();
    check_launch("ipm_large");
}

}  // namespace bqb
