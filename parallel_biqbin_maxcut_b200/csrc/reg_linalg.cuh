// Register-resident dense FP64 matrices for one 512-thread CTA, n <= 128.
//
// Thread t = 32*tc + tr owns rows R_a = tr + 32a (a < 4) and columns
// C_b = tc + 16b (b < 8): a 4 x 8 tile of a 128 x 128 matrix, held in
// registers for the whole factorisation.  An elimination step publishes only
// the pivot column (by its 32 owner threads) into a double-buffered shared
// vector; every thread then updates its 32 entries with register FMAs.
// Because step k writes buffer k&1 and reads it only after the barrier, and
// step k+2 (the next writer of that buffer) starts after every thread has
// passed step k+1's barrier, one __syncthreads() per step suffices.
#pragma once
#include "bqb_common.cuh"

namespace bqb {

constexpr int RM_NMAX = 128;
constexpr int RM_THREADS = 512;

struct RegMat {
    double m[4][8];
};

__device__ __forceinline__ int rm_row(int a) { return (threadIdx.x & 31) + 32 * a; }
__device__ __forceinline__ int rm_col(int b) { return (threadIdx.x >> 5) + 16 * b; }

// Load an n x n column-major matrix (entries outside n read as 0).
template <class F>
__device__ __forceinline__ void rm_fill(RegMat& M, int n, F f)
{
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const int c = rm_col(b);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int r = rm_row(a);
            M.m[a][b] = (r < n && c < n) ? f(r, c) : 0.0;
        }
    }
}

__device__ __forceinline__ void rm_store(const RegMat& M, double* A, int n)
{
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const int c = rm_col(b);
        if (c >= n) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int r = rm_row(a);
            if (r < n) A[r + (size_t)c * n] = M.m[a][b];
        }
    }
}

// Store only the lower triangle (r >= c).
__device__ __forceinline__ void rm_store_lower(const RegMat& M, double* A, int n)
{
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const int c = rm_col(b);
        if (c >= n) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int r = rm_row(a);
            if (r < n && r >= c) A[r + (size_t)c * n] = M.m[a][b];
        }
    }
}

// Publish column k (rows < n) into buf: done by the 32 owner threads.
__device__ __forceinline__ void rm_publish_col(const RegMat& M, int n, int k, double* buf)
{
    if ((threadIdx.x >> 5) != (k & 15)) return;
    const int kb = k >> 4;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        if (b != kb) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int r = rm_row(a);
            if (r < n) buf[r] = M.m[a][b];
        }
    }
}

// Cholesky A = L L^T (L in the lower triangle of M; the upper triangle is
// left with symmetric leftovers).  col2: 2 * RM_NMAX doubles of shared
// memory.  Returns false, uniformly, at the first non-positive pivot.
// Step k: the owners publish column k unscaled (a_ik, with a_kk the pivot);
// every thread applies A_ij -= a_ik a_jk / a_kk to its entries with i,j > k;
// the owners turn their column into L_ik = a_ik / sqrt(a_kk).
__device__ __forceinline__ bool rm_potrf(RegMat& M, int n, double* col2)
{
    rm_publish_col(M, n, 0, col2);
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double* col = col2 + (k & 1) * RM_NMAX;
        const double d = col[k];
        if (!(d > 0.0)) return false;
        const double inv = 1.0 / d;
        const double rs = 1.0 / sqrt(d);
        const int kb = k >> 4;
        const bool owner = (threadIdx.x >> 5) == (k & 15);
        double cr[4], cc[8];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int r = rm_row(a);
            cr[a] = (r > k && r < n) ? col[r] * inv : 0.0;
        }
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const int c = rm_col(b);
            cc[b] = (c > k && c < n) ? col[c] : 0.0;
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) M.m[a][b] = fma(-cr[a], cc[b], M.m[a][b]);
        if (owner) {
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                if (b != kb) continue;
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const int r = rm_row(a);
                    if (r > k) M.m[a][b] = col[r] * rs;
                    else if (r == k) M.m[a][b] = d * rs;   // sqrt(d)
                }
            }
        }
        if (k + 1 < n) rm_publish_col(M, n, k + 1, col2 + ((k + 1) & 1) * RM_NMAX);
        __syncthreads();
    }
    return true;
}

// In-place inverse of a symmetric positive definite matrix (full storage),
// symmetric Gauss-Jordan sweep: at step k, with d = A_kk and the column
// c = A(:,k) before the step, A_ij -= c_i c_j / d (i,j != k),
// A_ik = A_ki = c_i / d, A_kk = -1/d; the result is -inv(A), negated at the
// end.  The pivots are the Schur complements of A, so a non-positive pivot
// means "not positive definite" (returned uniformly).  The update uses the
// product c_i c_j, which is the same for (i,j) and (j,i): the result is
// exactly symmetric.
__device__ __forceinline__ bool rm_spd_inverse(RegMat& M, int n, double* col2)
{
    rm_publish_col(M, n, 0, col2);
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double* col = col2 + (k & 1) * RM_NMAX;
        const double d = col[k];
        if (!(d > 0.0)) return false;
        const double inv = 1.0 / d;
        double cr[4], cc[8];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int r = rm_row(a);
            cr[a] = (r < n) ? col[r] : 0.0;
        }
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const int c = rm_col(b);
            cc[b] = (c < n) ? col[c] : 0.0;
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int r = rm_row(a);
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const int c = rm_col(b);
                double v = fma(-(cr[a] * cc[b]), inv, M.m[a][b]);
                if (r == k) v = cc[b] * inv;
                if (c == k) v = cr[a] * inv;
                if (r == k && c == k) v = -inv;
                M.m[a][b] = v;
            }
        }
        if (k + 1 < n) rm_publish_col(M, n, k + 1, col2 + ((k + 1) & 1) * RM_NMAX);
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) M.m[a][b] = -M.m[a][b];
    return true;
}

}  // namespace bqb
