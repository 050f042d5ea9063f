// The basic SDP interior-point method (src/ipm_mc_pk.c:28-359) for n above
// the register-resident limit (IPM_REG_NMAX = 128): ONE cooperative launch
// per call.  Every CTA (one per SM at most) runs the whole predictor-
// corrector loop; the phases of an iteration (the inverses, the solves, the
// two products, the line searches' positive-definiteness tests, the step)
// are separated by a grid barrier, and every decision (a failed pivot, the
// line-search step, the stopping test) is taken by every CTA from the same
// data with the same arithmetic, so all CTAs follow one control path with no
// host round trip.
//
// Inverses (Zi = inv(Z), F = inv(Zi .* X)) use a blocked symmetric
// Gauss-Jordan sweep on panels of CB = 32 columns.  For panel K with
// D = A_KK = Ld Ld^T and the panel columns C = A(:, K): V = C Ld^{-T},
// A_ij -= V_i V_j^T (i, j outside K), A_iK = W_i = V_i Ld^{-1} (= C_i D^{-1}),
// A_KK = -D^{-1}; after the last panel A = -inv(A).  The Cholesky pivots are
// the Schur complements of A: a non-positive one means "not positive
// definite".  The line searches' tests run the trailing part of the sweep
// only (a blocked right-looking Cholesky).  The Schur update goes through
// Ld, not the explicit D^{-1}: at n = 343 with couplings of 1e5, M reaches a
// condition number of 1e11 at the last iteration, and C D^{-1} C^T then
// turned a pivot of the positive definite M negative.
//
// One grid barrier per panel: every CTA factors the 32 x 32 panel block
// itself (the same arithmetic in every CTA, hence the same decision), and
// the owner of a 32 x 32 tile of A computes the V rows it needs itself.  The
// writes of panel K's own row and column blocks (W and -D^{-1}) would race
// with the other CTAs' reads of the panel columns, so they are deferred:
// panel K leaves W_K and D^{-1}_K in side buffers, and in the next phase the
// owner of each tile in row or column block K writes them before its own
// update (readers of those entries take them from the side buffers).
//
// Products with F replace the Cholesky solves, each followed by one step of
// iterative refinement with M = Zi .* X (x <- x + F (b - M x)).
//
// The grid barrier is a counter and a generation word in global memory;
// every wait is bounded (2 s), after which the barrier sets an error word,
// no CTA waits any more, every loop ends, and the call reports status
// IPM_SYNC (a fatal error on the host).
#include <math.h>

#include <map>
#include <mutex>
#include <vector>

#include "bqb_common.cuh"
#include "internal.h"
#include "ipm.cuh"

namespace bqb {

double* ipm_stats_device();

namespace {

constexpr int CB = 32;          // panel and tile width
constexpr int CT = 256;         // threads per CTA
constexpr int CW = CT / 32;     // warps per CTA
constexpr int LDS = CB + 1;     // padded shared-memory row
static_assert(CT == CW * 32 && CB == 32 && 4 * CW == CB, "a CTA's threads cover a tile as 32 rows x 8 columns, 4 times");
constexpr unsigned long long BAR_TIMEOUT_NS = 2000000000ull;

struct CoopArgs {
    const double* L;     // n x n, read only
    double* Xbase;       // output matrix (X = Xbase + (*xslot) n^2)
    const int* xslot;
    double* out;         // phi, iterations, status, <L,X>
    double* stats;       // IPM work counters (may be null)
    double *Zi, *F, *M, *T, *T2, *dX, *dX1;   // n x n each (T, T2: the line searches' trial matrices)
    double *Wb, *Db;                     // 2 x (n x CB), 2 x (CB x CB)
    double *y, *zd, *dy, *dy1, *dy2, *r, *t;
    double* part;        // gridDim.x x 4 partial sums
    unsigned* bar;       // [0] arrivals, [1] generation, [2] error
    unsigned long long* prof;   // (may be null) CTA 0's nanoseconds per part, COOP_PROF_* slots
    double* yout;        // (may be null) y of the last iterate
    int n;
};

// Parts of the time CTA 0 spends in a call (bqb_ipm_coop_profile).
enum CoopProf : int {
    COOP_PROF_BARRIER,   // waiting at grid barriers
    COOP_PROF_FACTOR,    // the panel factorisations (every CTA factors each panel block)
    COOP_PROF_TILES,     // the sweeps' tile updates
    COOP_PROF_GEMM,      // the two symmetric products
    COOP_PROF_TOTAL,     // the whole call
    COOP_PROF_BARRIERS,  // count of grid barriers
    COOP_PROF_PHASES,    // count of sweep phases
    COOP_PROF_PF_LOAD,   // the part of the panel factorisations spent loading the panel block
    COOP_PROF_WORDS = 8
};

// Trial sweeps a line-search round runs together (each with its own panel
// factor in shared memory).
constexpr int NTRIAL = 4;

// One panel's factorisation.
struct PanelF {
    double Lc[CB][CB];       // the panel's factor by columns (row Q = column Q)
    double Lr[CB][CB + 2];   // the panel's factor by rows (rows 16-byte aligned)
    double D[CB][LDS];       // the panel block
    double Li[CB][LDS];      // inverse of the factor (lower)
    double R[CB];            // reciprocals of the factor's diagonal
};

struct Smem {
    PanelF pf[NTRIAL];
    double A1[CB][LDS];   // C_I, or a GEMM operand tile
    double A2[CB][LDS];   // C_J, or a GEMM operand tile
    double V1[CB][LDS];   // V_I, or a GEMM operand tile
    double V2[CB][LDS];   // V_J, or a GEMM operand tile
    double red[CW * 4];
    double tot[4];
    int ok;
    int pd[NTRIAL];
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier with a bounded wait.  Returns false once any CTA has given up
// (then nothing waits any more).  The fences around the arrival make every
// write before the barrier visible to every read after it.
__device__ bool grid_sync(unsigned* bar, Smem& sm, unsigned long long* prof = nullptr)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long tb = prof && blockIdx.x == 0 ? global_ns() : 0ull;
        volatile unsigned* vb = bar;
        int ok = vb[2] == 0u;
        if (ok) {
            const unsigned gen = vb[1];
            __threadfence();
            if (atomicAdd(bar, 1u) == gridDim.x - 1) {
                atomicExch(bar, 0u);
                __threadfence();
                atomicAdd(bar + 1, 1u);
            } else {
                const unsigned long long t0 = global_ns();
                while (vb[1] == gen) {
                    if (vb[2] != 0u) {
                        ok = 0;
                        break;
                    }
                    if (global_ns() - t0 > BAR_TIMEOUT_NS) {
                        atomicExch(bar + 2, 1u);
                        ok = 0;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            __threadfence();
        }
        sm.ok = ok;
        if (prof && blockIdx.x == 0) {
            prof[COOP_PROF_BARRIER] += global_ns() - tb;
            prof[COOP_PROF_BARRIERS] += 1;
        }
    }
    __syncthreads();
    return sm.ok != 0;
}

// The sums over all entries (the starting point's, the step's) are taken
// over a fixed partition into VCTA parts, one block of CT threads each with
// the entries of a CTA of a VCTA-CTA grid; a CTA of a smaller grid takes
// several parts in turn.  The totals are then the same bits for any grid.
constexpr int VCTA = 148;

// Block-reduce four partial sums into part[v * 4 + k] (the CTA's part v).
__device__ void block_partials(double a, double b, double c, double d, Smem& sm, double* part, int v)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    d = warp_sum(d);
    if (lane == 0) {
        sm.red[w * 4 + 0] = a;
        sm.red[w * 4 + 1] = b;
        sm.red[w * 4 + 2] = c;
        sm.red[w * 4 + 3] = d;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int q = 0; q < CW; ++q) s += sm.red[q * 4 + threadIdx.x];
        part[v * 4 + threadIdx.x] = s;
    }
    __syncthreads();   // sm.red is reused by the CTA's next part
}

// The totals of the partial sums (after a barrier), in part order: the same
// value in every CTA.
__device__ void grid_totals(const double* part, Smem& sm)
{
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int g = 0; g < VCTA; ++g) s += part[g * 4 + threadIdx.x];
        sm.tot[threadIdx.x] = s;
    }
    __syncthreads();
}

// ---- the panel sweep ---------------------------------------------------------

// Step Q of the register Cholesky of a 32 x 32 block held by one warp
// (lane p holds row p in s[]): column Q of the factor, then the rank-1
// update of the rows below.  The column goes to the warp through shared
// memory (one store per lane, then broadcast reads of two entries at a
// time), which costs fewer issue slots than a shuffle per entry.
// Instantiated for every Q so that every index into s[] is a constant and
// s[] stays in registers.  No early exit: after a non-positive pivot (the
// same d in every lane) the steps go on with a unit pivot and the caller
// discards the result.  Lane Q keeps the pivot's reciprocal square root, the
// reciprocal of its diagonal entry of the factor.
template <int Q>
__device__ __forceinline__ void chol_step(double (&s)[CB], int p, int& pd, double& rdiag, double (*Lc)[CB])
{
    if constexpr (Q < CB) {
        double d = __shfl_sync(0xffffffffu, s[Q], Q);
        if (!(d > 0.0)) {
            pd = 0;
            d = 1.0;
        }
        const double rs = rsqrt(d);
        const double l = d * rs;
        const double lpq = p == Q ? l : s[Q] * rs;
        if (p == Q) rdiag = rs;
        s[Q] = lpq;
        Lc[Q][p] = lpq;
        __syncwarp();
        constexpr int r0 = (Q + 1) & ~1;
#pragma unroll
        for (int r = r0; r < CB; r += 2) {
            const double2 v = *reinterpret_cast<const double2*>(&Lc[Q][r]);
            if (r > Q && r <= p) s[r] = fma(-lpq, v.x, s[r]);
            if (r + 1 <= p) s[r + 1] = fma(-lpq, v.y, s[r + 1]);
        }
        chol_step<Q + 1>(s, p, pd, rdiag, Lc);
    }
}

// Step I of the inverse of the lower factor for the calling lane's column t:
// li[I] = (delta_It - sum_{k < I} Lr[I][k] li[k]) / Lr[I][I] (zero above the
// diagonal, where every term is zero).  Instantiated for every I so that li[]
// stays in registers; the factor's entries are shared-memory broadcasts read
// two at a time that do not depend on the chain.  The sum runs in four
// interleaved partial sums, so the dependent chain per step is a quarter as
// long.
template <int I>
__device__ __forceinline__ void linv_step(double (&li)[CB], const PanelF& sm, int t)
{
    if constexpr (I < CB) {
        double a0 = I == t ? 1.0 : 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
        for (int k = 0; k + 3 < I; k += 4) {
            const double2 u = *reinterpret_cast<const double2*>(&sm.Lr[I][k]);
            const double2 w = *reinterpret_cast<const double2*>(&sm.Lr[I][k + 2]);
            a0 = fma(-u.x, li[k], a0);
            a1 = fma(-u.y, li[k + 1], a1);
            a2 = fma(-w.x, li[k + 2], a2);
            a3 = fma(-w.y, li[k + 3], a3);
        }
#pragma unroll
        for (int k = I & ~3; k < I; ++k) a0 = fma(-sm.Lr[I][k], li[k], a0);
        li[I] = ((a0 + a1) + (a2 + a3)) * sm.R[I];
        linv_step<I + 1>(li, sm, t);
    }
}

// The panel block D = A[K, K] (b x b, padded to 32 x 32 with the identity)
// into f.D; every thread of the CTA takes part (no barrier).
__device__ __forceinline__ void panel_load(const double* A, int n, int k0, int b, PanelF& f)
{
    for (int e = threadIdx.x; e < CB * CB; e += CT) {
        const int p = e % CB, q = e / CB;
        f.D[p][q] = p < b && q < b ? A[(k0 + p) + (size_t)(k0 + q) * n] : (p == q ? 1.0 : 0.0);
    }
}

// One warp: the Cholesky factor Ld of f.D and Li = Ld^{-1} in f (lane p
// holds row p in registers), then lane t forms column t of Li by forward
// substitution.  *pd_out = 0 on a non-positive pivot (then f is partial).
__device__ void panel_chol(PanelF& sm, int* pd_out)
{
    {
        const int p = threadIdx.x & 31;
        double s[CB];
#pragma unroll
        for (int r = 0; r < CB; ++r) s[r] = sm.D[p][r];
        int pd = 1;
        double rdiag = 1.0;
        chol_step<0>(s, p, pd, rdiag, sm.Lc);
        if (p == 0) *pd_out = pd;
        if (pd) {
#pragma unroll
            for (int r = 0; r < CB; r += 2)
                *reinterpret_cast<double2*>(&sm.Lr[p][r]) = make_double2(r <= p ? s[r] : 0.0, r + 1 <= p ? s[r + 1] : 0.0);
            sm.R[p] = rdiag;
        }
        __syncwarp();
        if (pd) {
            double li[CB];
            linv_step<0>(li, sm, p);
#pragma unroll
            for (int i = 0; i < CB; ++i) sm.Li[i][p] = li[i];
        }
    }
}

// Every CTA: the Cholesky factor Ld of D = A[K, K] (b x b) and Li = Ld^{-1}
// in sm.pf[0] (warp 0 factors).  Returns false (in every thread) on a
// non-positive pivot.
__device__ bool panel_factor(const double* A, int n, int k0, int b, Smem& sm, unsigned long long* load_ns)
{
    const unsigned long long t0 = load_ns ? global_ns() : 0ull;
    panel_load(A, n, k0, b, sm.pf[0]);
    __syncthreads();
    if (load_ns) *load_ns += global_ns() - t0;
    if (threadIdx.x < 32) panel_chol(sm.pf[0], &sm.pd[0]);
    __syncthreads();
    return sm.pd[0] != 0;
}

// C rows of tile block I (32 x b): the panel columns of A for rows I, or, for
// the row block of the previous panel (whose entries still wait for their
// fix), W_{K-1} transposed.  Then V = C Ld^{-T}: V(r, q) = sum_{p <= q}
// C(r, p) Li(q, p).  Not inlined: its registers are then allocated apart
// from the panel factorisation's, and the kernel needs no spill slots.
__device__ __noinline__ void load_v(const double* A, int n, int I, int k0, int b, const double* Wprev, bool from_w,
                       double (*Cs)[LDS], double (*Vs)[LDS], const PanelF& f)
{
    const int i0 = I * CB;
    for (int e = threadIdx.x; e < CB * CB; e += CT) {
        const int r = e % CB, p = e / CB;
        const int i = i0 + r;
        double v = 0.0;
        if (i < n && p < b) v = from_w ? Wprev[(k0 + p) + (size_t)r * n] : A[i + (size_t)(k0 + p) * n];
        Cs[r][p] = v;
    }
    __syncthreads();
    // thread (r, c0) forms V(r, c0 + 8 j), j = 0..3, reading C(r, p) once for
    // all four; Li(q, p) = 0 for p > q, so running p to the largest q adds
    // exact zeros to the smaller ones
    {
        const int r = threadIdx.x % CB, c0 = threadIdx.x / CB;
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int p = 0; p <= c0 + 3 * CW; ++p) {
            const double cp = Cs[r][p];
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = fma(cp, f.Li[c0 + CW * j][p], v[j]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) Vs[r][c0 + CW * j] = c0 + CW * j < b ? v[j] : 0.0;
    }
    __syncthreads();
}

// Phase K of the sweep for tile (I, J).  FULL: the pending fix of panel
// K - 1 (tiles in its row or column block), the update (I, J != K), W_K of
// row block I (diagonal tiles) and D^{-1}_K (tile (K, K)).  Trailing only:
// the update.
template <bool FULL>
__device__ void tile_step(double* A, int n, int K, int k0, int b, int I, int J, const double* Wprev,
                          const double* Dprev, double* Wcur, double* Dcur, Smem& sm, const PanelF& f)
{
    const bool fixI = FULL && K > 0 && I == K - 1;
    const bool fixJ = FULL && K > 0 && J == K - 1;
    const bool upd = I != K && J != K;
    if (!upd && !fixI && !fixJ && !(FULL && I == K && J == K)) return;
    if (upd) {
        load_v(A, n, I, k0, b, Wprev, fixI, sm.A1, sm.V1, f);
        if (J != I) load_v(A, n, J, k0, b, Wprev, fixJ, sm.A2, sm.V2, f);
    }
    double (*VJ)[LDS] = J != I ? sm.V2 : sm.V1;
    const int i0 = I * CB, j0 = J * CB, kp0 = (K - 1) * CB;
    // thread (r, c0) owns the entries (r, c0 + 8 j), j = 0..3, of the tile
    // and reads V1(r, q) once for all four
    const int r = threadIdx.x % CB, c0 = threadIdx.x / CB;
    if (upd || fixI || fixJ) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        if (upd)
            for (int q = 0; q < b; ++q) {
                const double a = sm.V1[r][q];
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) acc[jj] = fma(a, VJ[c0 + CW * jj][q], acc[jj]);
            }
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int c = c0 + CW * jj;
            const int i = i0 + r, j = j0 + c;
            if (i >= n || j >= n) continue;
            double v;
            if (fixI && fixJ) v = -Dprev[(i - kp0) + (size_t)(j - kp0) * CB];
            else if (fixJ) v = Wprev[i + (size_t)(j - kp0) * n];
            else if (fixI) v = Wprev[j + (size_t)(i - kp0) * n];
            else v = A[i + (size_t)j * n];
            if (upd) v -= acc[jj];
            A[i + (size_t)j * n] = v;
        }
    }
    if (FULL && upd && I == J) {
        // W_K(i, q) = sum_{p >= q} V(i, p) Li(p, q); Li(p, q) = 0 for p < q,
        // so starting p at the smallest q adds exact zeros to the others
        double w[4] = {0.0, 0.0, 0.0, 0.0};
        for (int p = c0; p < b; ++p) {
            const double vp = sm.V1[r][p];
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) w[jj] = fma(vp, f.Li[p][c0 + CW * jj], w[jj]);
        }
        const int i = i0 + r;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int q = c0 + CW * jj;
            if (i < n && q < b) Wcur[i + (size_t)q * n] = w[jj];
        }
    }
    if (FULL && I == K && J == K) {
        // D^{-1}_K = Li^T Li
        for (int e = threadIdx.x; e < CB * CB; e += CT) {
            const int p = e % CB, q = e / CB;
            double acc = 0.0;
            for (int k = p > q ? p : q; k < b; ++k) acc = fma(f.Li[k][p], f.Li[k][q], acc);
            Dcur[p + (size_t)q * CB] = acc;
        }
    }
    __syncthreads();
}

// The final phase of a full sweep: the fix of the last panel's row and
// column blocks, and A = -A; with Xm, also Mout = Fout = A .* Xm (Xm + ap dXm
// with dXm).  No barrier.
__device__ void sweep_final(double* A, const CoopArgs& a, const double* Xm, double* Mout, double* Fout,
                            const double* dXm, double ap)
{
    const int n = a.n;
    const int T = (n + CB - 1) / CB;
    {
        const int K = T;
        const double* Wl = a.Wb + (size_t)((K + 1) & 1) * n * CB;
        const double* Dl = a.Db + (size_t)((K + 1) & 1) * CB * CB;
        const int kp0 = (K - 1) * CB;
        for (int q = blockIdx.x; q < T * T; q += gridDim.x) {
            const int I = q % T, J = q / T;
            const bool fixI = I == K - 1, fixJ = J == K - 1;
            for (int e = threadIdx.x; e < CB * CB; e += CT) {
                const int i = I * CB + e % CB, j = J * CB + e / CB;
                if (i >= n || j >= n) continue;
                double v;
                if (fixI && fixJ) v = -Dl[(i - kp0) + (size_t)(j - kp0) * CB];
                else if (fixJ) v = Wl[i + (size_t)(j - kp0) * n];
                else if (fixI) v = Wl[j + (size_t)(i - kp0) * n];
                else v = A[i + (size_t)j * n];
                const size_t ij = i + (size_t)j * n;
                A[ij] = -v;
                if (Xm) {
                    const double xm = dXm ? fma(ap, dXm[ij], Xm[ij]) : Xm[ij];
                    const double m = -v * xm;
                    Mout[ij] = m;
                    Fout[ij] = m;
                }
            }
        }
    }
}

// The panel sweep of A (n x n).  FULL: A becomes inv(A); otherwise only the
// trailing updates run, for the pivots.  With Xm (FULL only), the final
// phase also writes Mout = Fout = inv(A) .* Xm for its tiles (the next
// inverse's input), saving a phase; with dXm as well, Xm + ap dXm (rounded
// as the step's update rounds it) takes the place of Xm.  Returns 1
// (positive definite), 0 (a non-positive pivot; every CTA returns 0 at the
// same panel) or -1 (a barrier gave up).
template <bool FULL>
__device__ int sweep(double* A, const CoopArgs& a, Smem& sm, const double* Xm = nullptr, double* Mout = nullptr,
                     double* Fout = nullptr, const double* dXm = nullptr, double ap = 0.0)
{
    const int n = a.n;
    const int T = (n + CB - 1) / CB;
    for (int K = 0; K < T; ++K) {
        const int k0 = K * CB, b = n - k0 < CB ? n - k0 : CB;
        const bool rec = a.prof && blockIdx.x == 0 && threadIdx.x == 0;
        unsigned long long tp = rec ? global_ns() : 0ull;
        if (!panel_factor(A, n, k0, b, sm, rec ? a.prof + COOP_PROF_PF_LOAD : nullptr)) return 0;
        if (rec) {
            const unsigned long long t = global_ns();
            a.prof[COOP_PROF_FACTOR] += t - tp;
            a.prof[COOP_PROF_PHASES] += 1;
            tp = t;
        }
        if (!FULL && K == T - 1) return 1;
        const double* Wprev = a.Wb + (size_t)((K + 1) & 1) * n * CB;
        const double* Dprev = a.Db + (size_t)((K + 1) & 1) * CB * CB;
        double* Wcur = a.Wb + (size_t)(K & 1) * n * CB;
        double* Dcur = a.Db + (size_t)(K & 1) * CB * CB;
        const int t0 = FULL ? 0 : K + 1;
        const int Tt = T - t0;
        for (int q = blockIdx.x; q < Tt * Tt; q += gridDim.x)
            tile_step<FULL>(A, n, K, k0, b, t0 + q % Tt, t0 + q / Tt, Wprev, Dprev, Wcur, Dcur, sm, sm.pf[0]);
        if (a.prof) __syncthreads();
        if (rec) a.prof[COOP_PROF_TILES] += global_ns() - tp;
        if (!grid_sync(a.bar, sm, a.prof)) return -1;
    }
    if (FULL) {
        // the last panel's fix, and A = -A
        sweep_final(A, a, Xm, Mout, Fout, dXm, ap);
        if (!grid_sync(a.bar, sm, a.prof)) return -1;
    }
    return 1;
}

// Trial sweeps run together: nt matrices, each the trailing sweep (its
// pivots) or, for at most one, the full sweep (its inverse).  state[t]
// becomes 1 (positive definite) or -1 (a non-positive pivot); every CTA takes
// the same decisions.
struct TrialSet {
    double* A[NTRIAL];
    int full[NTRIAL];
    int state[NTRIAL];
    int nt;
};

// In each phase every running trial's panel block is factored by its own
// warp (warp t for trial t) and the tiles of all running trials are spread
// over the CTAs; a trial drops out at its first non-positive pivot, a
// trailing sweep is done at its last panel's factorisation, a full sweep
// after its final phase.  Returns false when a barrier gave up.  The last
// phase has no barrier when no full sweep runs on (the caller's next fill
// goes to other matrices or follows a barrier).
__device__ bool msweep(TrialSet& ts, const CoopArgs& a, Smem& sm)
{
    const int n = a.n;
    const int T = (n + CB - 1) / CB;
    const bool rec = a.prof && blockIdx.x == 0 && threadIdx.x == 0;
    for (int t = 0; t < ts.nt; ++t) ts.state[t] = 0;
    for (int K = 0; K < T; ++K) {
        const int k0 = K * CB, b = n - k0 < CB ? n - k0 : CB;
        unsigned long long tp = rec ? global_ns() : 0ull;
        for (int t = 0; t < ts.nt; ++t)
            if (ts.state[t] == 0) panel_load(ts.A[t], n, k0, b, sm.pf[t]);
        __syncthreads();
        {
            const int w = threadIdx.x >> 5;
            if (w < ts.nt && ts.state[w] == 0) panel_chol(sm.pf[w], &sm.pd[w]);
        }
        __syncthreads();
        bool running = false;
        int tiles[NTRIAL];
        int total = 0;
        for (int t = 0; t < ts.nt; ++t) {
            tiles[t] = 0;
            if (ts.state[t] != 0) continue;
            if (!sm.pd[t]) {
                ts.state[t] = -1;
            } else if (!ts.full[t] && K == T - 1) {
                ts.state[t] = 1;
            } else {
                running = true;
                const int tt = ts.full[t] ? T : T - K - 1;
                tiles[t] = tt * tt;
                total += tiles[t];
            }
        }
        if (rec) {
            const unsigned long long tn = global_ns();
            a.prof[COOP_PROF_FACTOR] += tn - tp;
            a.prof[COOP_PROF_PHASES] += 1;
            tp = tn;
        }
        if (!running) return true;
        const double* Wprev = a.Wb + (size_t)((K + 1) & 1) * n * CB;
        const double* Dprev = a.Db + (size_t)((K + 1) & 1) * CB * CB;
        double* Wcur = a.Wb + (size_t)(K & 1) * n * CB;
        double* Dcur = a.Db + (size_t)(K & 1) * CB * CB;
        for (int q = blockIdx.x; q < total; q += gridDim.x) {
            int t = 0, r = q;
            while (r >= tiles[t]) {
                r -= tiles[t];
                ++t;
            }
            if (ts.full[t]) {
                tile_step<true>(ts.A[t], n, K, k0, b, r % T, r / T, Wprev, Dprev, Wcur, Dcur, sm, sm.pf[t]);
            } else {
                const int tt = T - K - 1;
                tile_step<false>(ts.A[t], n, K, k0, b, K + 1 + r % tt, K + 1 + r / tt, Wprev, Dprev, Wcur, Dcur, sm,
                                 sm.pf[t]);
            }
        }
        if (a.prof) __syncthreads();
        if (rec) a.prof[COOP_PROF_TILES] += global_ns() - tp;
        if (!grid_sync(a.bar, sm, a.prof)) return false;
    }
    for (int t = 0; t < ts.nt; ++t)
        if (ts.state[t] == 0 && ts.full[t]) {
            sweep_final(ts.A[t], a, nullptr, nullptr, nullptr, nullptr, 0.0);
            if (!grid_sync(a.bar, sm, a.prof)) return false;
            ts.state[t] = 1;
        }
    return true;
}

// ---- products ------------------------------------------------------------------

// out = sym(Zi (Diag(-a) X + Diag(-b) Y) + e1 E1 + e2 E2) (b, Y, E2 may be
// null; the row scales enter negated, -(a_k X_kc) being exactly
// (-a_k) X_kc): the owner of the tile pair (I, J), (J, I) forms both
// products and writes the symmetric part.  k in chunks of 32; thread
// (r, cc) holds P(I0 + r, J0 + c) and P(J0 + c, I0 + r) for c = cc + 8t.
__device__ void gemm_sym(const double* Zi, const double* av, const double* X, const double* bv, const double* Y,
                         double e1, const double* E1, double e2, const double* E2, int n, double* out, Smem& sm)
{
    const int T = (n + CB - 1) / CB;
    const int tid = threadIdx.x, r = tid % CB, cc = tid / CB;
    const int npairs = T * (T + 1) / 2;
    for (int pq = blockIdx.x; pq < npairs; pq += gridDim.x) {
        int I = 0, rem = pq;
        while (rem >= T - I) {
            rem -= T - I;
            ++I;
        }
        const int J = I + rem;
        const int i0 = I * CB, j0 = J * CB;
        double acc1[4] = {0.0, 0.0, 0.0, 0.0}, acc2[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k0 = 0; k0 < n; k0 += CB) {
            for (int e = tid; e < CB * CB; e += CT) {
                const int p = e % CB, q = e / CB;
                const int kk = k0 + q, kb = k0 + p;
                sm.A1[p][q] = (i0 + p < n && kk < n) ? Zi[(i0 + p) + (size_t)kk * n] : 0.0;
                sm.A2[p][q] = (j0 + p < n && kk < n) ? Zi[(j0 + p) + (size_t)kk * n] : 0.0;
                double v1 = 0.0, v2 = 0.0;
                if (kb < n && j0 + q < n) {
                    const size_t idx = kb + (size_t)(j0 + q) * n;
                    v1 = -av[kb] * X[idx];
                    if (bv) v1 = fma(-bv[kb], Y[idx], v1);
                }
                if (kb < n && i0 + q < n) {
                    const size_t idx = kb + (size_t)(i0 + q) * n;
                    v2 = -av[kb] * X[idx];
                    if (bv) v2 = fma(-bv[kb], Y[idx], v2);
                }
                sm.V1[p][q] = v1;   // B(k, J0 + q)
                sm.V2[p][q] = v2;   // B(k, I0 + q)
            }
            __syncthreads();
#pragma unroll 4
            for (int k = 0; k < CB; ++k) {
                const double a1 = sm.A1[r][k];
                const double b2 = sm.V2[k][r];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int c = cc + 8 * t;
                    acc1[t] = fma(a1, sm.V1[k][c], acc1[t]);
                    acc2[t] = fma(sm.A2[c][k], b2, acc2[t]);
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int i = i0 + r, j = j0 + cc + 8 * t;
            if (i >= n || j >= n) continue;
            const size_t ij = i + (size_t)j * n, ji = j + (size_t)i * n;
            double vij = acc1[t] + e1 * E1[ij];
            double vji = acc2[t] + e1 * E1[ji];
            if (E2) {
                vij += e2 * E2[ij];
                vji += e2 * E2[ji];
            }
            const double v = i == j ? vij : 0.5 * (vij + vji);
            out[ij] = v;
            out[ji] = v;
        }
    }
}

// One warp per row i (the grid's warps in turn): out_i = sum_c F(c, i) v_c
// (F symmetric; v null: v = -e).
__device__ void warp_rows_matvec(const double* F, int n, const double* v, double* out)
{
    const int lane = threadIdx.x & 31;
    const int nw = gridDim.x * CW;
    for (int i = blockIdx.x * CW + (threadIdx.x >> 5); i < n; i += nw) {
        const double* col = F + (size_t)i * n;
        double acc = 0.0;
        for (int c = lane; c < n; c += 32) acc = fma(col[c], v ? v[c] : -1.0, acc);
        acc = warp_sum(acc);
        if (lane == 0) out[i] = acc;
    }
}

// r_i = b_i - sum_c M(c, i) x_c (b null: -1)
__device__ void warp_rows_resid(const double* M, int n, const double* b, const double* x, double* r)
{
    const int lane = threadIdx.x & 31;
    const int nw = gridDim.x * CW;
    for (int i = blockIdx.x * CW + (threadIdx.x >> 5); i < n; i += nw) {
        const double* col = M + (size_t)i * n;
        double acc = 0.0;
        for (int c = lane; c < n; c += 32) acc = fma(col[c], x[c], acc);
        acc = warp_sum(acc);
        if (lane == 0) r[i] = (b ? b[i] : -1.0) - acc;
    }
}

// t = F r; x += t (row i of both by the same warp)
__device__ void warp_rows_refine(const double* F, int n, const double* r, double* t, double* x)
{
    const int lane = threadIdx.x & 31;
    const int nw = gridDim.x * CW;
    for (int i = blockIdx.x * CW + (threadIdx.x >> 5); i < n; i += nw) {
        const double* col = F + (size_t)i * n;
        double acc = 0.0;
        for (int c = lane; c < n; c += 32) acc = fma(col[c], r[c], acc);
        acc = warp_sum(acc);
        if (lane == 0) {
            t[i] = acc;
            x[i] = x[i] + acc;
        }
    }
}

// rhs_i = mu Zi_ii - sum_c Zi_ic dX1_ic dy1_c (columns i by symmetry)
__device__ void warp_rows_rhs(const double* Zi, const double* dX1, const double* dy1, double mu, int n, double* rhs)
{
    const int lane = threadIdx.x & 31;
    const int nw = gridDim.x * CW;
    for (int i = blockIdx.x * CW + (threadIdx.x >> 5); i < n; i += nw) {
        const size_t o = (size_t)i * n;
        double acc = 0.0;
        for (int c = lane; c < n; c += 32) acc = fma(Zi[o + c] * dX1[o + c], dy1[c], acc);
        acc = warp_sum(acc);
        if (lane == 0) rhs[i] = mu * Zi[o + i] - acc;
    }
}

// x = M^{-1} b (b null: -e): x = F b, then one refinement step.  Three
// phases; returns false when a barrier gave up.
__device__ bool solve(const CoopArgs& a, const double* F, const double* b, double* x, Smem& sm)
{
    warp_rows_matvec(F, a.n, b, x);
    if (!grid_sync(a.bar, sm, a.prof)) return false;
    warp_rows_resid(a.M, a.n, b, x, a.r);
    if (!grid_sync(a.bar, sm, a.prof)) return false;
    warp_rows_refine(F, a.n, a.r, a.t, x);
    return grid_sync(a.bar, sm, a.prof);
}

__global__ void __launch_bounds__(CT, 1) ipm_coop_kernel(CoopArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
    const int n = a.n;
    const size_t nn = (size_t)n * n;
    const size_t gtid = (size_t)blockIdx.x * CT + threadIdx.x, gstride = (size_t)gridDim.x * CT;
    const double* __restrict__ L = a.L;
    double* X = a.Xbase + (a.xslot ? (size_t)(*a.xslot) * nn : 0);
    const unsigned long long t_call = a.prof && blockIdx.x == 0 ? global_ns() : 0ull;

    // ---- initial point (src/ipm_mc_pk.c:65-99): y_c = sum_r |L_rc| + 1.1,
    // zd = y - diag(L), X = I; psi = trace(L), mu = sum(zd) / 2n, phi = sum(y)
    const size_t vstride = (size_t)VCTA * CT;
    for (int v = blockIdx.x; v < VCTA; v += gridDim.x) {
        const size_t vt = (size_t)v * CT + threadIdx.x;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (size_t c = vt; c < (size_t)n; c += vstride) {
            double acc = 0.0;
            const double* Lc = L + c * n;
            for (int r = 0; r < n; ++r) acc += fabs(Lc[r]);
            const double yc = acc + 1.1;
            const double zc = yc - Lc[c];
            a.y[c] = yc;
            a.zd[c] = zc;
            s0 += Lc[c];
            s1 += zc;
            s2 += yc;
        }
        block_partials(s0, s1, s2, 0.0, sm, a.part, v);
    }
    for (size_t e = gtid; e < nn; e += gstride) X[e] = (e % n == e / n) ? 1.0 : 0.0;
    bool alive = grid_sync(a.bar, sm, a.prof);
    grid_totals(a.part, sm);
    double psi = sm.tot[0];
    double mu = sm.tot[1] / (2.0 * n);
    double phi = sm.tot[2];
    double gap = fabs(phi - psi);
    int iter = 0, ls_total = 0, status = IPM_OK;
    // When the dual line search's first trial (ad = 1) passes, its full sweep
    // leaves inv(Z) of the new point in Zi (the same matrix, with the same
    // arithmetic, as this iteration's own sweep would), and the next
    // iteration only forms M = F = Zi .* X.
    double* const Zi = a.Zi;
    double* const F = a.F;
    bool have_zi = false;

    while (alive && gap > 1e-2) {
        if (++iter > IPM_MAX_ITERS) {
            status = IPM_MAXITER;
            break;
        }
        int pd = 1;
        if (!have_zi) {
            // Zi = inv(Z), Z = Diag(zd) - L off the diagonal
            for (size_t e = gtid; e < nn; e += gstride) {
                const int i = (int)(e % n), j = (int)(e / n);
                Zi[e] = i == j ? a.zd[i] : -L[e];
            }
            if (!(alive = grid_sync(a.bar, sm, a.prof))) break;
            // (its last phase also writes M = Zi .* X and F = M)
            pd = sweep<true>(Zi, a, sm, X, a.M, F);
            if (pd < 0) {
                alive = false;
                break;
            }
            if (!pd) {
                status = IPM_Z_NOT_PD;
                break;
            }
        } else {
            for (size_t e = gtid; e < nn; e += gstride) {
                const double m = Zi[e] * X[e];
                a.M[e] = m;
                F[e] = m;
            }
            if (!(alive = grid_sync(a.bar, sm, a.prof))) break;
        }
        have_zi = false;
        // F = inv(M); dy1 = F (-e)
        pd = sweep<true>(F, a, sm);
        if (pd < 0) {
            alive = false;
            break;
        }
        if (!pd) {
            status = IPM_M_NOT_PD;
            break;
        }
        if (!(alive = solve(a, F, nullptr, a.dy1, sm))) break;
        // dX1 = sym(Zi (-Diag(dy1) X) - X)
        unsigned long long tg = a.prof && blockIdx.x == 0 ? global_ns() : 0ull;
        gemm_sym(Zi, a.dy1, X, nullptr, nullptr, -1.0, X, 0.0, nullptr, n, a.dX1, sm);
        if (a.prof) __syncthreads();
        if (a.prof && blockIdx.x == 0 && threadIdx.x == 0) a.prof[COOP_PROF_GEMM] += global_ns() - tg;
        if (!(alive = grid_sync(a.bar, sm, a.prof))) break;
        // corrector: rhs = mu diag(Zi) - (Zi .* dX1) dy1; dy2 = F rhs
        warp_rows_rhs(Zi, a.dX1, a.dy1, mu, n, a.dy);
        if (!(alive = grid_sync(a.bar, sm, a.prof))) break;
        if (!(alive = solve(a, F, a.dy, a.dy2, sm))) break;
        // dX = sym(Zi (-Diag(dy2) X - Diag(dy1) dX1) + mu Zi + dX1)
        tg = a.prof && blockIdx.x == 0 ? global_ns() : 0ull;
        gemm_sym(Zi, a.dy2, X, a.dy1, a.dX1, 1.0, a.dX1, mu, Zi, n, a.dX, sm);
        if (a.prof) __syncthreads();
        if (a.prof && blockIdx.x == 0 && threadIdx.x == 0) a.prof[COOP_PROF_GEMM] += global_ns() - tg;
        if (!(alive = grid_sync(a.bar, sm, a.prof))) break;

        // line searches (src/ipm_mc_pk.c:281-309): the primal search
        // (X + ap dX positive definite) and the dual search (Z + ad Diag(dy)
        // positive definite) each try 1, 0.8, 0.64, ... and keep the first
        // step that passes.  Here a round sweeps the next two trials of each
        // unfinished search together (primal in T, T2; dual in Zi, F, all free
        // by now); every trial's pivots are those of its own sweep, so the
        // steps kept are the one-at-a-time searches' steps.  The dual's first
        // trial (ad = 1, the step itself when it passes) is a full sweep whose
        // inverse starts the next iteration.
        double ap = 1.0, ad = 1.0;   // the next trial step of each search
        int pi = 0, di = 0;          // its trial index
        int pres = 0, dres = 0;      // 1 found, -1 gave up
        double ap_ok = 1.0, ad_ok = 1.0;
        int rounds = 0;
        while (pres == 0 || dres == 0) {
            // a CTA may still read the last round's panel blocks
            if (rounds++ > 0 && !(alive = grid_sync(a.bar, sm, a.prof))) break;
            TrialSet ts;
            double alpha[NTRIAL];
            int dual[NTRIAL];
            ts.nt = 0;
            auto add = [&](double* buf, double al, bool du, bool full) {
                ts.A[ts.nt] = buf;
                ts.full[ts.nt] = full ? 1 : 0;
                alpha[ts.nt] = al;
                dual[ts.nt] = du ? 1 : 0;
                ++ts.nt;
            };
            const int np0 = ts.nt;
            if (pres == 0) {
                add(a.T, ap, false, false);
                if (pi + 1 < IPM_MAX_TRIALS) add(a.T2, ap * 0.8, false, false);
            }
            const int nd0 = ts.nt;
            if (dres == 0) {
                add(Zi, ad, true, di == 0);
                if (di + 1 < IPM_MAX_TRIALS) add(F, ad * 0.8, true, false);
            }
            // (dy_i = dy1_i + dy2_i)
            for (size_t e = gtid; e < nn; e += gstride) {
                const int i = (int)(e % n), j = (int)(e / n);
                for (int t = 0; t < ts.nt; ++t)
                    ts.A[t][e] = dual[t] ? (i == j ? fma(alpha[t], a.dy1[i] + a.dy2[i], a.zd[i]) : -L[e])
                                         : fma(alpha[t], a.dX[e], X[e]);
            }
            if (!(alive = grid_sync(a.bar, sm, a.prof))) break;
            if (!(alive = msweep(ts, a, sm))) break;
            // each search: the first of its trials that passed, in order
            auto decide = [&](int t0, int t1, int& res, int& idx, double& step, double& ok_step) {
                for (int t = t0; t < t1; ++t) {
                    if (ts.state[t] == 1) {
                        res = 1;
                        ok_step = alpha[t];
                        ls_total += idx + (t - t0) + 1;
                        return t - t0;
                    }
                }
                idx += t1 - t0;
                step = alpha[t1 - 1] * 0.8;
                if (idx >= IPM_MAX_TRIALS) res = -1;
                return -1;
            };
            if (pres == 0) decide(np0, nd0, pres, pi, ap, ap_ok);
            if (dres == 0) {
                const bool first = di == 0;
                if (decide(nd0, ts.nt, dres, di, ad, ad_ok) == 0 && first) have_zi = true;
            }
            if (pres < 0 || dres < 0) break;
        }
        if (!alive) break;
        if (pres < 0 || dres < 0) {
            status = IPM_LINESEARCH;
            break;
        }
        ap = ap_ok;
        ad = ad_ok;
        if (ap < 1.0) ap *= 0.95;
        if (ad < 1.0) ad *= 0.95;

        // update (src/ipm_mc_pk.c:313-334): X += ap dX, y += ad dy,
        // zd += ad dy (dy = dy1 + dy2), and the sums zx = <Z, X>, lx = <L, X>,
        // sum(y) of the new point.  The diagonal of X goes with the vectors
        // (the thread that moves zd_i also moves X_ii).
        for (int v = blockIdx.x; v < VCTA; v += gridDim.x) {
            const size_t vt = (size_t)v * CT + threadIdx.x;
            double zx = 0.0, lx = 0.0, ys = 0.0;
            for (size_t e = vt; e < nn; e += vstride) {
                const int i = (int)(e % n), j = (int)(e / n);
                if (i == j) continue;
                const double xv = fma(ap, a.dX[e], X[e]);
                X[e] = xv;
                const double lv = L[e];
                lx = fma(lv, xv, lx);
                zx = fma(-lv, xv, zx);
            }
            for (size_t c = vt; c < (size_t)n; c += vstride) {
                const size_t e = c * n + c;
                const double xv = fma(ap, a.dX[e], X[e]);
                X[e] = xv;
                const double dyc = a.dy1[c] + a.dy2[c];
                const double yv = fma(ad, dyc, a.y[c]);
                const double zv = fma(ad, dyc, a.zd[c]);
                a.y[c] = yv;
                a.zd[c] = zv;
                lx = fma(L[e], xv, lx);
                zx = fma(zv, xv, zx);
                ys += yv;
            }
            block_partials(zx, lx, ys, 0.0, sm, a.part, v);
        }
        if (!(alive = grid_sync(a.bar, sm, a.prof))) break;
        grid_totals(a.part, sm);
        mu = sm.tot[0] / (2.0 * n);
        if (ap + ad > 1.6) mu *= 0.5;
        if (ap + ad > 1.9) mu *= 0.2;
        phi = sm.tot[2];
        psi = sm.tot[1];
        gap = fabs(phi - psi);
        // (the partials are rewritten only after the next iteration's
        // barriers, so no barrier is needed here)
    }
    if (!alive) status = IPM_SYNC;
    // (y's last writes came before the update's barrier)
    if (a.yout)
        for (size_t c = gtid; c < (size_t)n; c += gstride) a.yout[c] = a.y[c];
    if (a.prof && blockIdx.x == 0 && threadIdx.x == 0) a.prof[COOP_PROF_TOTAL] += global_ns() - t_call;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = phi;
        a.out[1] = (double)iter;
        a.out[2] = (double)status;
        a.out[3] = psi;
        if (a.stats) {
            const double n3 = (double)n * n * n;
            atomicAdd(&a.stats[0], iter * n3);
            atomicAdd(&a.stats[1], 1.0);
            atomicAdd(&a.stats[2], (double)iter);
            atomicAdd(&a.stats[3], (double)ls_total);
        }
    }
}

struct CoopConfig {
    int grid = 0;
    size_t smem = 0;
};

// Per-part timing of CTA 0 (off unless bqb_ipm_coop_profile_enable(1)).
std::atomic<int> g_coop_prof_on{0};
DevBuf<unsigned long long> g_coop_prof;
std::mutex g_coop_prof_mu;

unsigned long long* coop_prof_device()
{
    if (!g_coop_prof_on.load()) return nullptr;
    std::lock_guard<std::mutex> lock(g_coop_prof_mu);
    if (!g_coop_prof.p) {
        g_coop_prof.ensure(COOP_PROF_WORDS);
        BQB_CUDA(cudaMemset(g_coop_prof.p, 0, COOP_PROF_WORDS * sizeof(unsigned long long)));
    }
    return g_coop_prof.p;
}

// The per-size schedule: the grid (CTAs) to use for T = ceil(n / 32) tiles
// per dimension, filled by the autotuner (bqb_ipm_autotune) or set by hand
// (bqb_ipm_schedule_set); sizes without an entry use one CTA per tile.
std::mutex g_sched_mu;
std::map<int, int> g_sched;

}  // namespace

// Engines bounding nodes above IPM_REG_NMAX right now (node.cu counts them):
// each multi-CTA IPM launch then takes its share of the co-resident CTAs, so
// the IPMs of concurrent engines run side by side instead of one after
// another.  The IPM's result does not depend on its grid.
std::atomic<int> g_large_share{0};

namespace {

// Grid size for n: the schedule's entry for its tile count, else one CTA
// per 32 x 32 tile of the sweep; at most as many as can be co-resident (one
// per SM at this register count), divided by the number of engines bounding
// large nodes at the time.
CoopConfig coop_config(int n)
{
    static int max_blocks = -1;
    static std::atomic<int> ready{0};
    CoopConfig c;
    c.smem = sizeof(Smem);
    BQB_SMEM_LIMIT(ipm_coop_kernel, c.smem);   // per device (cached)
    if (!ready.load()) {
        int per_sm = 0;
        BQB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ipm_coop_kernel, CT, c.smem));
        max_blocks = per_sm * rt().num_sms;
        ready.store(1);
    }
    const int T = (n + CB - 1) / CB;
    int g = T * T;
    {
        std::lock_guard<std::mutex> lock(g_sched_mu);
        auto it = g_sched.find(T);
        if (it != g_sched.end()) g = it->second;
    }
    const int share = g_large_share.load();
    const int cap = share > 1 ? max_blocks / share : max_blocks;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    c.grid = g;
    return c;
}

}  // namespace

size_t ipm_large_ws_doubles(int n)
{
    const size_t nn = (size_t)n * n;
    return 7 * nn + 2 * (size_t)n * CB + 2 * (size_t)CB * CB + 8 * (size_t)n + 4 * 1024 + 16;
}

// ipm_mc_pk for n > IPM_REG_NMAX: one cooperative launch on stream s, no
// host synchronisation.  xslot (optional, device): write X into
// Xbase + (*xslot) * n * n.  Results in dout[0..3] (phi, iterations, status,
// psi); status IPM_SYNC when a grid barrier gave up waiting.
void ipm_large(DevBuf<double>& wsbuf, const double* L, double* Xbase, int n, double* dout, cudaStream_t s,
               const int* xslot, double* yout)
{
    const size_t nn = (size_t)n * n;
    double* p = wsbuf.ensure(ipm_large_ws_doubles(n));
    CoopArgs a;
    a.L = L;
    a.Xbase = Xbase;
    a.xslot = xslot;
    a.out = dout;
    a.stats = ipm_stats_device();
    a.prof = coop_prof_device();
    a.yout = yout;
    a.n = n;
    a.Zi = p;
    a.F = a.Zi + nn;
    a.M = a.F + nn;
    a.T = a.M + nn;
    a.T2 = a.T + nn;
    a.dX = a.T2 + nn;
    a.dX1 = a.dX + nn;
    a.Wb = a.dX1 + nn;
    a.Db = a.Wb + 2 * (size_t)n * CB;
    a.y = a.Db + 2 * (size_t)CB * CB;
    a.zd = a.y + n;
    a.dy = a.zd + n;
    a.dy1 = a.dy + n;
    a.dy2 = a.dy1 + n;
    a.r = a.dy2 + n;
    a.t = a.r + n;
    a.part = a.t + n;
    a.bar = reinterpret_cast<unsigned*>(a.part + 4 * 1024);
    const CoopConfig c = coop_config(n);
    BQB_CUDA(cudaMemsetAsync(a.bar, 0, 4 * sizeof(unsigned), s));
    void* args[] = {&a};
    BQB_CUDA(cudaLaunchCooperativeKernel((const void*)ipm_coop_kernel, dim3(c.grid), dim3(CT), args, c.smem, s));
    BQB_COUNT_LAUNCH();
    check_launch("ipm_large");
}

}  // namespace bqb

using namespace bqb;

// Use `grid` CTAs for the multi-CTA IPM of every n with the same tile count
// as n (grid <= 0 removes the entry).  No reference counterpart.
BQB_API void bqb_ipm_schedule_set(int n, int grid)
{
    if (n <= 0) return;
    const int T = (n + CB - 1) / CB;
    std::lock_guard<std::mutex> lock(g_sched_mu);
    if (grid > 0) g_sched[T] = grid;
    else g_sched.erase(T);
}

// Autotune the multi-CTA IPM's grid for size n (> 128): time `reps` calls
// for each candidate (one CTA per tile, half, a quarter, an eighth, and the
// SM count) on a seeded problem of that size (the Laplacian of a random
// +-1 graph, as the B&B's subproblems are), keep the fastest in the
// schedule.  best_grid / best_ms (may be null) receive the choice and its
// time per call.  Returns 0, 1 for n <= 128.  No reference counterpart.
BQB_API int bqb_ipm_autotune(int n, int reps, int* best_grid, double* best_ms)
{
    if (n <= 128) return 1;
    if (reps < 1) reps = 1;
    Runtime& R = rt();
    cudaStream_t s = R.stream;
    const size_t nn = (size_t)n * n;
    std::vector<double> L(nn, 0.0);
    unsigned long long z = 0x5eedull + (unsigned long long)n;
    auto next = [&]() {
        z += 0x9E3779B97F4A7C15ull;
        unsigned long long x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return x ^ (x >> 31);
    };
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) {
            const unsigned long long r = next();
            if (r & 1) continue;                       // edge with probability 1/2
            const double w = (r & 2) ? 1.0 : -1.0;     // weight +-1
            L[i + (size_t)j * n] = L[j + (size_t)i * n] = -w;
            L[i + (size_t)i * n] += w;
            L[j + (size_t)j * n] += w;
        }
    for (double& v : L) v *= 0.25;
    DevBuf<double> dL, dX, ws, out;
    BQB_CUDA(cudaMemcpy(dL.ensure(nn), L.data(), nn * sizeof(double), cudaMemcpyHostToDevice));
    dX.ensure(nn);
    out.ensure(4);
    const int T = (n + CB - 1) / CB;
    std::vector<int> cand = {T * T, (T * T + 1) / 2, (T * T + 3) / 4, (T * T + 7) / 8, R.num_sms};
    cudaEvent_t e0, e1;
    BQB_CUDA(cudaEventCreate(&e0));
    BQB_CUDA(cudaEventCreate(&e1));
    int bg = T * T;
    double bms = 1e300;
    for (int g : cand) {
        if (g < 1) continue;
        bqb_ipm_schedule_set(n, g);
        ipm_large(ws, dL.p, dX.p, n, out.p, s, nullptr);   // warm-up
        BQB_CUDA(cudaEventRecord(e0, s));
        for (int r = 0; r < reps; ++r) ipm_large(ws, dL.p, dX.p, n, out.p, s, nullptr);
        BQB_CUDA(cudaEventRecord(e1, s));
        BQB_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        BQB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        double h[4];
        BQB_CUDA(cudaMemcpy(h, out.p, sizeof h, cudaMemcpyDeviceToHost));
        if ((int)h[2] == IPM_OK && ms / reps < bms) {
            bms = ms / reps;
            bg = g;
        }
    }
    BQB_CUDA(cudaEventDestroy(e0));
    BQB_CUDA(cudaEventDestroy(e1));
    // (DevBuf does not free: the tuning problem's buffers go here)
    for (double* q : {dL.p, dX.p, ws.p, out.p})
        if (q) BQB_CUDA(cudaFree(q));
    bqb_ipm_schedule_set(n, bg);   // the fastest candidate stays in the schedule
    if (best_grid) *best_grid = bg;
    if (best_ms) *best_ms = bms;
    return 0;
}

// Time the multi-CTA IPM spends per part (its CTA 0, summed over calls since
// the last reset): enable (on != 0) or disable the timing; out[8] = {barrier
// waits, panel factorisations, tile updates, products, whole calls (ms),
// grid barriers, sweep phases, the panel factorisations' block loads (ms)};
// reset != 0 zeroes after reading.  For
// profiling; no reference counterpart.
BQB_API void bqb_ipm_coop_profile_enable(int on) { g_coop_prof_on.store(on != 0); }

BQB_API void bqb_ipm_coop_profile(double* out, int reset)
{
    unsigned long long h[COOP_PROF_WORDS] = {};
    std::lock_guard<std::mutex> lock(g_coop_prof_mu);
    if (g_coop_prof.p) {
        BQB_CUDA(cudaMemcpy(h, g_coop_prof.p, sizeof h, cudaMemcpyDeviceToHost));
        if (reset) BQB_CUDA(cudaMemset(g_coop_prof.p, 0, sizeof h));
    }
    for (int i = 0; i < COOP_PROF_WORDS; ++i)
        out[i] = (i < COOP_PROF_BARRIERS || i == COOP_PROF_PF_LOAD) ? 1e-6 * (double)h[i] : (double)h[i];
}
