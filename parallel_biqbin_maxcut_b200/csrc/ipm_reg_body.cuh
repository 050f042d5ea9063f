// Register-resident IPM body for n <= 128 (one CTA of IPM_THREADS threads
// per problem), shared by the IPM kernels (ipm.cu) and the fused node kernel
// (nodek.cu) so both run the same arithmetic.
#pragma once
#include <math.h>

#include "cta_linalg.cuh"
#include "ipm.cuh"
#include "reg_linalg.cuh"

namespace bqb {

// ---------------------------------------------------------------------------
// Register-resident variant for n <= 128: the matrices being factored or
// inverted (Z, Zi.*X and the two line-search trial matrices) live in
// registers, 4 x 8 entries per thread (reg_linalg.cuh), one barrier per
// elimination step.  The steps are ipm_body's, except that the Schur matrix
// M = Zi.*X is inverted by the Gauss-Jordan sweep (F = M^{-1}) and both of
// its solves are products with F: n barrier steps on 512 threads replace
// the Cholesky plus two one-warp triangular solves of 2n steps each.  The
// line searches need only "positive definite or not": the pivots of the
// elimination, without forming the factor.
// Shared memory: red[64], y, zd, dy, dy1, rhs (nv each), the GEMM stage
// tile (which also holds the factorisations' 2 x 130 pivot-column buffers:
// the GEMM and the factorisations never run at the same time), F (n^2), and
// Zi (n^2) when it fits; global scratch: dX, dX1, and Zi otherwise.
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t ipm_reg_fixed_smem_doubles(int n)
{
    const size_t nv = (size_t)((n + 1) & ~1);
    return 64 + 5 * nv + (size_t)CTA_KC * STG_LD;
}

// out = M^{-1} v (v null: v = -e) with Minv stored full, n x n; one warp per
// row, reading Minv's column r (contiguous; Minv is symmetric).
__device__ inline void ipm_minv_apply(const double* Minv, int n, const double* v, double* out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r = warp; r < n; r += nw) {
        const double* col = Minv + (size_t)r * n;
        double acc = 0.0;
        for (int c = lane; c < n; c += 32) acc = fma(col[c], v ? v[c] : -1.0, acc);
        acc = warp_sum(acc);
        if (lane == 0) out[r] = acc;
    }
    __syncthreads();
}

// stats (optional, device): the work counters [iterations n^3, problems,
// iterations, line-search trials] are added there.
__device__ inline void ipm_body_reg(const IpmDesc& d, double* smem, int zi_in_smem, double* stats)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const int n = d.n;
    const size_t nn = (size_t)n * n;
    const size_t nv = (size_t)((n + 1) & ~1);
    const double* __restrict__ L = d.L;
    double* __restrict__ X = d.X + (d.xslot ? (size_t)(*d.xslot) * nn : 0);
    double* red = smem;
    double* y = red + 64;
    double* zd = y + nv;
    double* dy = zd + nv;
    double* dy1 = dy + nv;
    double* rhs = dy1 + nv;
    double* stage = rhs + nv;
    double* F = stage + (size_t)CTA_KC * STG_LD;
    double* ws = d.ws;
    double* dX = ws;
    double* dX1 = ws + nn;
    double* Zi = zi_in_smem ? F + nn : ws + 2 * nn;
    double* cbuf = stage;   // 2 * RM_BUF pivot-column buffers (the stage is idle then)
    static_assert(CTA_KC * STG_LD >= 2 * RM_BUF, "pivot buffers exceed the GEMM stage");

    // ---- initial point (src/ipm_mc_pk.c:65-99) ----
    for (int c = tid; c < n; c += nt) {
        double acc = 0.0;
        const double* Lc = L + (size_t)c * n;
        for (int r = 0; r < n; ++r) acc += fabs(Lc[r]);
        y[c] = acc + 1.1;
    }
    for (size_t e = tid; e < nn; e += nt) X[e] = 0.0;
    __syncthreads();
    for (int i = tid; i < n; i += nt) {
        X[i + (size_t)i * n] = 1.0;
        zd[i] = y[i] - L[i + (size_t)i * n];
    }
    __syncthreads();
    double a0 = 0.0, b0 = 0.0, p0 = 0.0;
    for (int i = tid; i < n; i += nt) {
        a0 += L[i + (size_t)i * n];
        b0 += zd[i];
        p0 += y[i];
    }
    double psi = block_sum(a0, red);
    double mu = block_sum(b0, red) / (2.0 * n);
    double phi = block_sum(p0, red);
    double gap = fabs(phi - psi);
    int iter = 0, ls_total = 0;
    int status = IPM_OK;
    RegMat R;

    while (gap > 1e-2) {
        if (++iter > IPM_MAX_ITERS) { status = IPM_MAXITER; break; }

        // ---- Zi = inv(Z), Z = Diag(zd) - L off the diagonal ----
        rm_fill(R, n, [&](int r, int c) { return r == c ? zd[r] : -L[r + (size_t)c * n]; });
        if (!rm_spd_inverse(R, n, cbuf)) { status = IPM_Z_NOT_PD; break; }
        rm_store(R, Zi, n);
        // ---- M = Zi .* X, factor, dy1 = M \ (-e) ----
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const int c = rm_col(b);
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const int r = rm_row(a);
                if (r < n && c < n) R.m[a][b] *= X[r + (size_t)c * n];
            }
        }
        __syncthreads();
        // M^{-1} by the register Gauss-Jordan sweep (its pivots are M's Schur
        // complements: a non-positive one is where the reference's dposv
        // fails), then both solves are products with it
        if (!rm_spd_inverse(R, n, cbuf)) { status = IPM_M_NOT_PD; break; }
        rm_store(R, F, n);
        __syncthreads();
        ipm_minv_apply(F, n, nullptr, dy1);

        // ---- dX1 = Zi * (-Diag(dy1) X) - X, symmetrised ----
        cta_gemm(
            Zi, n, n, [=] __device__(int k, int c) { return -dy1[k] * X[k + (size_t)c * n]; },
            [=] __device__(int r, int c, double acc) { dX1[r + (size_t)c * n] = acc - X[r + (size_t)c * n]; },
            stage);
        cta_symmetrize(dX1, n);

        // ---- corrector rhs = mu diag(Zi) - (Zi .* dX1) dy1 ----
        for (int r = warp; r < n; r += nw) {
            double acc = 0.0;
            for (int c = lane; c < n; c += 32)
                acc = fma(Zi[r + (size_t)c * n] * dX1[r + (size_t)c * n], dy1[c], acc);
            acc = warp_sum(acc);
            if (lane == 0) rhs[r] = mu * Zi[r + (size_t)r * n] - acc;
        }
        __syncthreads();
        ipm_minv_apply(F, n, rhs, dy);

        // ---- dX = Zi * (-Diag(dy2) X - Diag(dy1) dX1) + mu Zi + dX1 ----
        {
            const double* dy2 = dy;
            const double muc = mu;
            const double* Zc = Zi;
            cta_gemm(
                Zi, n, n,
                [=] __device__(int k, int c) {
                    const size_t e = k + (size_t)c * n;
                    return -dy2[k] * X[e] + -dy1[k] * dX1[e];
                },
                [=] __device__(int r, int c, double acc) {
                    const size_t e = r + (size_t)c * n;
                    dX[e] = dX1[e] + (acc + muc * Zc[e]);
                },
                stage);
            cta_symmetrize(dX, n);
        }
        for (int i = tid; i < n; i += nt) dy[i] = dy1[i] + dy[i];
        __syncthreads();

        // ---- primal line search: X + ap dX positive definite (the reference's chol) ----
        double ap = 1.0;
        int trials = 0;
        bool ok = false;
        while (true) {
            const double al = ap;
            rm_fill(R, n, [&](int r, int c) {
                const size_t e = r + (size_t)c * n;
                return fma(al, dX[e], X[e]);
            });
            if (rm_posdef(R, n, cbuf)) { ok = true; break; }
            __syncthreads();
            if (++trials >= IPM_MAX_TRIALS) break;
            ap *= 0.8;
        }
        ls_total += trials + 1;
        if (!ok) { status = IPM_LINESEARCH; break; }
        if (ap < 1.0) ap *= 0.95;

        // ---- dual line search: Z + ad Diag(dy) positive definite ----
        double ad = 1.0;
        trials = 0;
        ok = false;
        while (true) {
            const double al = ad;
            rm_fill(R, n, [&](int r, int c) {
                return r == c ? fma(al, dy[r], zd[r]) : -L[r + (size_t)c * n];
            });
            if (rm_posdef(R, n, cbuf)) { ok = true; break; }
            __syncthreads();
            if (++trials >= IPM_MAX_TRIALS) break;
            ad *= 0.8;
        }
        ls_total += trials + 1;
        if (!ok) { status = IPM_LINESEARCH; break; }
        if (ad < 1.0) ad *= 0.95;

        // ---- update (src/ipm_mc_pk.c:313-334) ----
        double zx = 0.0, lx = 0.0;
        for (int j = warp; j < n; j += nw) {
            for (int i = lane; i < n; i += 32) {
                const size_t e = i + (size_t)j * n;
                const double xv = fma(ap, dX[e], X[e]);
                X[e] = xv;
                const double lv = L[e];
                lx = fma(lv, xv, lx);
                if (i != j) zx = fma(-lv, xv, zx);
            }
        }
        __syncthreads();
        double ysum = 0.0;
        for (int i = tid; i < n; i += nt) {
            const double yi = fma(ad, dy[i], y[i]);
            const double zi = fma(ad, dy[i], zd[i]);
            y[i] = yi;
            zd[i] = zi;
            ysum += yi;
            zx = fma(zi, X[i + (size_t)i * n], zx);
        }
        zx = block_sum(zx, red);
        lx = block_sum(lx, red);
        ysum = block_sum(ysum, red);
        mu = zx / (2.0 * n);
        if (ap + ad > 1.6) mu *= 0.5;
        if (ap + ad > 1.9) mu *= 0.2;
        phi = ysum;
        psi = lx;
        gap = fabs(phi - psi);
    }

    if (d.yout)
        for (int i = tid; i < n; i += nt) d.yout[i] = y[i];
    if (tid == 0) {
        d.out[0] = phi;
        d.out[1] = (double)iter;
        d.out[2] = (double)status;
        d.out[3] = psi;
        const double n3 = (double)n * n * n;
        if (stats) {
            atomicAdd(&stats[0], iter * n3);
            atomicAdd(&stats[1], 1.0);
            atomicAdd(&stats[2], (double)iter);
            atomicAdd(&stats[3], (double)ls_total);
        }
    }
}

}  // namespace bqb
