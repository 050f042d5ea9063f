// CTA-level FP64 dense linear algebra used inside single-CTA kernels.
// All routines are called by every thread of the block; matrices are
// column-major and may live in shared or global memory (generic pointers).
#pragma once
#include "bqb_common.cuh"

namespace bqb {

constexpr int CTA_KC = 16;      // k-chunk of the staged GEMM B operand
constexpr int CTA_TILE = 128;   // GEMM supertile (rows and cols)

// Cholesky of the lower triangle of A (in place).  Returns false, uniformly
// over the block, at the first non-positive pivot (the line-search test).
__device__ inline bool cta_potrf_lower(double* A, int n, int ld, double* col)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int k = 0; k < n; ++k) {
        const double d = A[k + (size_t)k * ld];
        if (!(d > 0.0)) return false;
        const double s = sqrt(d);
        const double inv = 1.0 / s;
        for (int i = k + 1 + tid; i < n; i += nt) {
            const double v = A[i + (size_t)k * ld] * inv;
            col[i] = v;
            A[i + (size_t)k * ld] = v;
        }
        __syncthreads();
        if (tid == 0) A[k + (size_t)k * ld] = s;
        for (int j = k + 1 + warp; j < n; j += nw) {
            const double cj = col[j];
            double* Aj = A + (size_t)j * ld;
            for (int i = j + lane; i < n; i += 32) Aj[i] = fma(-col[i], cj, Aj[i]);
        }
        __syncthreads();
    }
    return true;
}

// In-place inverse of a symmetric positive definite matrix held in the lower
// triangle (symmetric sweep / Gauss-Jordan without pivoting).  On success A
// holds the full symmetric inverse (both triangles).
__device__ inline bool cta_spd_inverse(double* A, int n, int ld, double* col)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int k = 0; k < n; ++k) {
        const double d = A[k + (size_t)k * ld];
        if (!(d > 0.0)) return false;
        for (int i = tid; i < n; i += nt)
            col[i] = (i >= k) ? A[i + (size_t)k * ld] : A[k + (size_t)i * ld];
        __syncthreads();
        const double inv = 1.0 / d;
        for (int j = warp; j < n; j += nw) {
            double* Aj = A + (size_t)j * ld;
            if (j == k) {
                for (int i = j + lane; i < n; i += 32) Aj[i] = (i == k) ? -inv : col[i] * inv;
            } else {
                const double tj = col[j] * inv;
                for (int i = j + lane; i < n; i += 32)
                    Aj[i] = (i == k) ? tj : fma(-col[i], tj, Aj[i]);
            }
        }
        __syncthreads();
    }
    // the sweep leaves -inv(A); negate and mirror to the upper triangle
    for (int j = warp; j < n; j += nw) {
        for (int i = j + lane; i < n; i += 32) {
            const double v = -A[i + (size_t)j * ld];
            A[i + (size_t)j * ld] = v;
            A[j + (size_t)i * ld] = v;
        }
    }
    __syncthreads();
    return true;
}

// Solve (F F^T) x = b with F the lower Cholesky factor; one warp; b in smem.
__device__ inline void warp_chol_solve(const double* F, int n, int ld, double* b)
{
    const int lane = threadIdx.x & 31;
    for (int k = 0; k < n; ++k) {
        const double bk = b[k] / F[k + (size_t)k * ld];
        __syncwarp();
        if (lane == 0) b[k] = bk;
        const double* Fk = F + (size_t)k * ld;
        for (int i = k + 1 + lane; i < n; i += 32) b[i] = fma(-Fk[i], bk, b[i]);
        __syncwarp();
    }
    for (int k = n - 1; k >= 0; --k) {
        const double xk = b[k] / F[k + (size_t)k * ld];
        __syncwarp();
        if (lane == 0) b[k] = xk;
        for (int i = lane; i < k; i += 32) b[i] = fma(-F[k + (size_t)i * ld], xk, b[i]);
        __syncwarp();
    }
}

// Exact symmetrisation A = (A + A^T)/2 as the reference writes it
// (src/ipm_mc_pk.c:196-199): both entries get 0.5*(a_ij + a_ji).
__device__ inline void cta_symmetrize(double* A, int n)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = warp; j < n; j += nw) {
        for (int i = j + 1 + lane; i < n; i += 32) {
            const double v = 0.5 * (A[j + (size_t)i * n] + A[i + (size_t)j * n]);
            A[i + (size_t)j * n] = v;
            A[j + (size_t)i * n] = v;
        }
    }
    __syncthreads();
}

// C = A * B' with A (n x n, column-major, read in place) and B'(k, c) formed
// on the fly by `bfun` and staged through shared memory in k-chunks.  Each
// thread owns a 4 x 8 register tile of a 128 x 128 supertile.  The k sum is
// sequential, so results are deterministic.  `epi(r, c, acc)` stores.
// Called by CTAs of CTA_GEMM_THREADS threads.
constexpr int STG_LD = CTA_TILE + 1;
constexpr int CTA_GEMM_THREADS = 512;   // cta_gemm is called by 512-thread CTAs

template <class BF, class EF>
__device__ inline void cta_gemm(const double* A, int n, int lda, BF bfun, EF epi, double* stage)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int tr = tid & 31;
    const int tc = tid >> 5;   // 0..15
    for (int r0 = 0; r0 < n; r0 += CTA_TILE) {
        for (int c0 = 0; c0 < n; c0 += CTA_TILE) {
            double acc[4][8];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] = 0.0;
            // The next chunk of B' is formed into registers while the current
            // one is multiplied, so its global loads overlap the FMAs.
            constexpr int PRE = CTA_KC * CTA_TILE / CTA_GEMM_THREADS;   // chunk entries per thread
            double pre[PRE];
            auto form = [&](int k0) {
#pragma unroll
                for (int q = 0; q < PRE; ++q) {
                    const int e = tid + q * nt;
                    double v = 0.0;
                    if (e < CTA_KC * CTA_TILE) {
                        const int kk = e % CTA_KC, cc = e / CTA_KC;
                        const int k = k0 + kk, c = c0 + cc;
                        if (k < n && c < n) v = bfun(k, c);
                    }
                    pre[q] = v;
                }
            };
            form(0);
            for (int k0 = 0; k0 < n; k0 += CTA_KC) {
#pragma unroll
                for (int q = 0; q < PRE; ++q) {
                    const int e = tid + q * nt;
                    if (e < CTA_KC * CTA_TILE) stage[(e % CTA_KC) * STG_LD + e / CTA_KC] = pre[q];
                }
                __syncthreads();
                if (k0 + CTA_KC < n) form(k0 + CTA_KC);
                const int kmax = min(CTA_KC, n - k0);
                for (int kk = 0; kk < kmax; ++kk) {
                    const double* Ak = A + (size_t)(k0 + kk) * lda;
                    double av[4], bv[8];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        const int r = r0 + tr + 32 * a;
                        av[a] = (r < n) ? Ak[r] : 0.0;
                    }
#pragma unroll
                    for (int b = 0; b < 8; ++b) bv[b] = stage[kk * STG_LD + tc + 16 * b];
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int b = 0; b < 8; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
                }
                __syncthreads();
            }
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const int r = r0 + tr + 32 * a;
                if (r >= n) continue;
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    const int c = c0 + tc + 16 * b;
                    if (c < n) epi(r, c, acc[a][b]);
                }
            }
        }
    }
    __syncthreads();
}

}  // namespace bqb
