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

// Pivot-column buffers of RM_BUF doubles: the column (zeros where the step
// must not act) and the pivot at RM_NMAX.
constexpr int RM_BUF = RM_NMAX + 2;

// Owner warp of column k: publish rows r > k of column k (zeros elsewhere,
// so the update needs no index tests) and the pivot.
__device__ __forceinline__ void rm_publish_tail(const RegMat& M, int k, double* buf)
{
    if ((threadIdx.x >> 5) != (k & 15)) return;
    const int kb = k >> 4;
    double v[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) v[a] = 0.0;
#pragma unroll
    for (int b = 0; b < 8; ++b)
        if (b == kb)
#pragma unroll
            for (int a = 0; a < 4; ++a) v[a] = M.m[a][b];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int r = rm_row(a);
        buf[r] = r > k ? v[a] : 0.0;
        if (r == k) buf[RM_NMAX] = v[a];
    }
}

// Is the symmetric matrix in M (lower triangle read) positive definite?
// The pivots of the symmetric elimination, as a Cholesky factorisation
// meets them: step k reads the published tail of column k (rows r > k;
// zeros for r <= k, and the padding rows hold zeros, so the update needs no
// index tests) and the pivot a_kk, and every thread applies
// A_ij -= (a_ik / a_kk) a_jk to its 32 entries (a no-op where either factor
// is zero).  Only the pivots are needed, so the factor itself is not formed
// (the owner warp has no extra work on the step's critical path).  Returns
// false, uniformly, at the first non-positive pivot; M is overwritten.
// col2: 2 * RM_BUF doubles of shared memory.
__device__ __forceinline__ bool rm_posdef(RegMat& M, int n, double* col2)
{
    rm_publish_tail(M, 0, col2);
    __syncthreads();
    const int lane = threadIdx.x & 31, tc = threadIdx.x >> 5;
    for (int k = 0; k < n; ++k) {
        const double* col = col2 + (k & 1) * RM_BUF;
        const double d = col[RM_NMAX];
        if (!(d > 0.0)) return false;
        const double rs = rsqrt(d);   // 1/sqrt(d); the pivots stay well conditioned here
        const double inv = rs * rs;
        double cr[4], cc[8];
#pragma unroll
        for (int a = 0; a < 4; ++a) cr[a] = col[lane + 32 * a] * inv;
#pragma unroll
        for (int b = 0; b < 8; ++b) cc[b] = col[tc + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) M.m[a][b] = fma(-cr[a], cc[b], M.m[a][b]);
        if (k + 1 < n) rm_publish_tail(M, k + 1, col2 + ((k + 1) & 1) * RM_BUF);
        __syncthreads();
    }
    return true;
}

// Owner warp of column k: publish the whole column (rows beyond n hold 0).
__device__ __forceinline__ void rm_publish_full(const RegMat& M, int k, double* buf)
{
    if ((threadIdx.x >> 5) != (k & 15)) return;
    const int kb = k >> 4;
#pragma unroll
    for (int b = 0; b < 8; ++b)
        if (b == kb)
#pragma unroll
            for (int a = 0; a < 4; ++a) buf[rm_row(a)] = M.m[a][b];
}

// In-place inverse of a symmetric positive definite matrix (full storage),
// symmetric Gauss-Jordan sweep: at step k, with d = A_kk and the column
// c = A(:,k) before the step, A_ij -= c_i c_j / d (i,j != k),
// A_ik = A_ki = c_i / d, A_kk = -1/d; the result is -inv(A), negated at the
// end.  The pivots are the Schur complements of A, so a non-positive pivot
// means "not positive definite" (returned uniformly).  Each thread scales
// its eight column values by 1/d (= rsqrt(d)^2) once and applies
// A_ij -= c_i (c_j / d) with one FMA per entry; then the lane holding row k
// (one per warp, inside a warp-uniform branch on the row block) and the
// owner warp of column k overwrite the pivot row and column.  (i,j) and
// (j,i) round c_i (c_j / d) and c_j (c_i / d): symmetric up to the last bit.
__device__ __forceinline__ bool rm_spd_inverse(RegMat& M, int n, double* col2)
{
    rm_publish_full(M, 0, col2);
    __syncthreads();
    const int lane = threadIdx.x & 31, tc = threadIdx.x >> 5;
    for (int k = 0; k < n; ++k) {
        const double* col = col2 + (k & 1) * RM_BUF;
        const double d = col[k];
        if (!(d > 0.0)) return false;
        const double rq = rsqrt(d);
        const double inv = rq * rq;   // 1/d
        double cr[4], sc[8];
#pragma unroll
        for (int a = 0; a < 4; ++a) cr[a] = col[lane + 32 * a];
#pragma unroll
        for (int b = 0; b < 8; ++b) sc[b] = col[tc + 16 * b] * inv;   // c_j / d
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) M.m[a][b] = fma(-cr[a], sc[b], M.m[a][b]);
        // row k (one lane per warp): c_j / d
        {
            const bool rowk = lane == (k & 31);
            const int ak = k >> 5;
#pragma unroll
            for (int a = 0; a < 4; ++a)
                if (a == ak)
#pragma unroll
                    for (int b = 0; b < 8; ++b) M.m[a][b] = rowk ? sc[b] : M.m[a][b];
        }
        // column k (the owner warp): c_i / d, and -1/d on the diagonal
        if (tc == (k & 15)) {
            const int kb = k >> 4;
#pragma unroll
            for (int b = 0; b < 8; ++b)
                if (b == kb)
#pragma unroll
                    for (int a = 0; a < 4; ++a) M.m[a][b] = (lane + 32 * a == k) ? -inv : cr[a] * inv;
        }
        if (k + 1 < n) rm_publish_full(M, k + 1, col2 + ((k + 1) & 1) * RM_BUF);
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) M.m[a][b] = -M.m[a][b];
    return true;
}
}  // namespace bqb
