// Basic Max-Cut SDP interior-point method (FP64), one CTA per problem.
//
// Restates the primal-dual predictor-corrector loop of the reference
// ipm_mc_pk (src/ipm_mc_pk.c:28-359):
//   max <L,X> s.t. diag(X) = e, X psd;   min e'y s.t. Z = Diag(y) - L psd.
// Start y = 1.1 + column sums of |L|, X = I, Z = Diag(y) - L (:65-99); loop
// while |phi - psi| > 1e-2 (:124-126).  Per iteration: Zi = inv(Z)
// (:129-150), predictor dy1 = (Zi.*X) \ (-e) (:157-173),
// dX1 = -Zi Diag(dy1) X - X symmetrised (:181-199), corrector
// dy2 = (Zi.*X) \ (mu diag(Zi) - (Zi.*dX1) dy1) (:207-230),
// dX2 = mu Zi - Zi (Diag(dy2) X + Diag(dy1) dX1) (:238-260), dX = dX1 + dX2
// symmetrised, dZ = Diag(dy) (:265-275), line searches alpha *= 0.8 until
// the Cholesky of X + a dX / Z + a dZ succeeds, then *0.95 (:281-309),
// updates and mu heuristics (:313-324).
//
// Z is never stored: off the diagonal Z = -L exactly (Diag(y) - L, and dZ is
// diagonal), so only its diagonal zd is kept and updated as the reference
// updates Z_ii.  The Schur matrix M = Zi.*X is factored once per iteration
// and reused for the corrector solve (the reference refactors the same
// matrix).  Zi is formed by a symmetric Gauss-Jordan sweep on the lower
// triangle; its pivots are the Schur complements of Z, so a non-positive
// pivot is exactly "Z not positive definite".
#include "ipm.cuh"
#include "cta_linalg.cuh"
#include "reg_linalg.cuh"
#include "ipm_reg_body.cuh"

#include <math.h>

#include <mutex>
#include <vector>

namespace bqb {

// Work counters for the roofline: [0] sum over finished problems of
// iterations * n^3, [1] problems, [2] iterations, [3] line-search trials.
__device__ double g_ipm_stats[4];

namespace {

struct Layout {
    double* red;   // 64
    double* y;     // n
    double* zd;    // n   diagonal of Z
    double* dy;    // n
    double* dy1;   // n
    double* rhs;   // n
    double* col;   // n
    double* stage; // CTA_KC * STG_LD
    double* F;     // n*n  Cholesky workspace
    double* Zi;    // n*n
    double* dX;    // n*n
    double* dX1;   // n*n
};

__host__ __device__ inline size_t ipm_fixed_smem_doubles(int n)
{
    return 64 + 6 * (size_t)((n + 1) & ~1) + (size_t)CTA_KC * STG_LD;
}

__device__ Layout make_layout(const IpmDesc& d, double* smem, int place)
{
    const int n = d.n;
    const size_t nn = (size_t)n * n;
    const size_t nv = (size_t)((n + 1) & ~1);
    Layout l;
    l.red = smem;
    l.y = l.red + 64;
    l.zd = l.y + nv;
    l.dy = l.zd + nv;
    l.dy1 = l.dy + nv;
    l.rhs = l.dy1 + nv;
    l.col = l.rhs + nv;
    l.stage = l.col + nv;
    double* after = l.stage + (size_t)CTA_KC * STG_LD;
    double* ws = d.ws;
    if (place & 1) { l.F = after; after += nn; } else { l.F = ws; ws += nn; }
    if (place & 2) { l.Zi = after; after += nn; } else { l.Zi = ws; ws += nn; }
    l.dX = ws; ws += nn;
    l.dX1 = ws;
    return l;
}

__device__ void ipm_body(const IpmDesc& d, double* smem, int place)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const int n = d.n;
    const size_t nn = (size_t)n * n;
    const double* __restrict__ L = d.L;
    double* __restrict__ X = d.X + (d.xslot ? (size_t)(*d.xslot) * nn : 0);
    Layout s = make_layout(d, smem, place);

    // ---- initial point (src/ipm_mc_pk.c:65-99) ----
    for (int c = tid; c < n; c += nt) {
        double acc = 0.0;
        const double* Lc = L + (size_t)c * n;
        for (int r = 0; r < n; ++r) acc += fabs(Lc[r]);
        s.y[c] = acc + 1.1;
    }
    for (size_t e = tid; e < nn; e += nt) X[e] = 0.0;
    __syncthreads();
    for (int i = tid; i < n; i += nt) {
        X[i + (size_t)i * n] = 1.0;
        s.zd[i] = s.y[i] - L[i + (size_t)i * n];
    }
    __syncthreads();
    {
        double a = 0.0, b = 0.0;
        for (int i = tid; i < n; i += nt) { a += L[i + (size_t)i * n]; b += s.zd[i]; }
        a = block_sum(a, s.red);
        b = block_sum(b, s.red);
        double phi = 0.0;
        for (int i = tid; i < n; i += nt) phi += s.y[i];
        phi = block_sum(phi, s.red);
        double psi = a;
        double mu = b / (2.0 * n);
        double gap = fabs(phi - psi);
        int iter = 0;
        int ls_total = 0;
        int status = IPM_OK;

        while (gap > 1e-2) {
            if (++iter > IPM_MAX_ITERS) { status = IPM_MAXITER; break; }

            // ---- Zi = inv(Z), Z = Diag(zd) - L off the diagonal ----
            for (int j = warp; j < n; j += nw)
                for (int i = j + lane; i < n; i += 32)
                    s.Zi[i + (size_t)j * n] = (i == j) ? s.zd[i] : -L[i + (size_t)j * n];
            __syncthreads();
            if (!cta_spd_inverse(s.Zi, n, n, s.col)) { status = IPM_Z_NOT_PD; break; }

            // ---- predictor: M = Zi .* X, dy1 = M \ (-e) ----
            for (int j = warp; j < n; j += nw)
                for (int i = j + lane; i < n; i += 32)
                    s.F[i + (size_t)j * n] = s.Zi[i + (size_t)j * n] * X[i + (size_t)j * n];
            for (int i = tid; i < n; i += nt) s.rhs[i] = -1.0;
            __syncthreads();
            if (!cta_potrf_lower(s.F, n, n, s.col)) { status = IPM_M_NOT_PD; break; }
            if (warp == 0) warp_chol_solve(s.F, n, n, s.rhs);
            __syncthreads();
            for (int i = tid; i < n; i += nt) s.dy1[i] = s.rhs[i];
            __syncthreads();

            // ---- dX1 = Zi * (-Diag(dy1) X) - X, symmetrised ----
            {
                const double* dy1 = s.dy1;
                double* dX1 = s.dX1;
                cta_gemm(
                    s.Zi, n, n,
                    [=] __device__(int k, int c) { return -dy1[k] * X[k + (size_t)c * n]; },
                    [=] __device__(int r, int c, double acc) {
                        dX1[r + (size_t)c * n] = acc - X[r + (size_t)c * n];
                    },
                    s.stage);
                cta_symmetrize(dX1, n);
            }

            // ---- corrector rhs = mu diag(Zi) - (Zi .* dX1) dy1 ----
            for (int r = warp; r < n; r += nw) {
                double acc = 0.0;
                for (int c = lane; c < n; c += 32)
                    acc = fma(s.Zi[r + (size_t)c * n] * s.dX1[r + (size_t)c * n], s.dy1[c], acc);
                acc = warp_sum(acc);
                if (lane == 0) s.rhs[r] = mu * s.Zi[r + (size_t)r * n] - acc;
            }
            __syncthreads();
            if (warp == 0) warp_chol_solve(s.F, n, n, s.rhs);
            __syncthreads();

            // ---- dX = Zi * (-Diag(dy2) X - Diag(dy1) dX1) + mu Zi + dX1 ----
            {
                const double* dy1 = s.dy1;
                const double* dy2 = s.rhs;
                const double* dX1 = s.dX1;
                const double* Zi = s.Zi;
                double* dX = s.dX;
                const double muc = mu;
                cta_gemm(
                    s.Zi, n, n,
                    [=] __device__(int k, int c) {
                        const size_t e = k + (size_t)c * n;
                        return -dy2[k] * X[e] + -dy1[k] * dX1[e];
                    },
                    [=] __device__(int r, int c, double acc) {
                        const size_t e = r + (size_t)c * n;
                        dX[e] = dX1[e] + (acc + muc * Zi[e]);
                    },
                    s.stage);
                cta_symmetrize(dX, n);
            }
            for (int i = tid; i < n; i += nt) s.dy[i] = s.dy1[i] + s.rhs[i];
            __syncthreads();

            // ---- primal line search: chol(X + ap dX) ----
            double ap = 1.0;
            int trials = 0;
            bool ok = false;
            while (true) {
                for (int j = warp; j < n; j += nw)
                    for (int i = j + lane; i < n; i += 32) {
                        const size_t e = i + (size_t)j * n;
                        s.F[e] = fma(ap, s.dX[e], X[e]);
                    }
                __syncthreads();
                if (cta_potrf_lower(s.F, n, n, s.col)) { ok = true; break; }
                __syncthreads();
                if (++trials >= IPM_MAX_TRIALS) break;
                ap *= 0.8;
            }
            ls_total += trials + 1;
            if (!ok) { status = IPM_LINESEARCH; break; }
            if (ap < 1.0) ap *= 0.95;

            // ---- dual line search: chol(Z + ad Diag(dy)) ----
            double ad = 1.0;
            trials = 0;
            ok = false;
            while (true) {
                for (int j = warp; j < n; j += nw)
                    for (int i = j + lane; i < n; i += 32)
                        s.F[i + (size_t)j * n] =
                            (i == j) ? fma(ad, s.dy[i], s.zd[i]) : -L[i + (size_t)j * n];
                __syncthreads();
                if (cta_potrf_lower(s.F, n, n, s.col)) { ok = true; break; }
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
                    const double xv = fma(ap, s.dX[e], X[e]);
                    X[e] = xv;
                    const double lv = L[e];
                    lx = fma(lv, xv, lx);
                    if (i != j) zx = fma(-lv, xv, zx);
                }
            }
            __syncthreads();
            double ysum = 0.0;
            for (int i = tid; i < n; i += nt) {
                const double yi = fma(ad, s.dy[i], s.y[i]);
                const double zi = fma(ad, s.dy[i], s.zd[i]);
                s.y[i] = yi;
                s.zd[i] = zi;
                ysum += yi;
                zx = fma(zi, X[i + (size_t)i * n], zx);
            }
            zx = block_sum(zx, s.red);
            lx = block_sum(lx, s.red);
            ysum = block_sum(ysum, s.red);
            mu = zx / (2.0 * n);
            if (ap + ad > 1.6) mu *= 0.5;
            if (ap + ad > 1.9) mu *= 0.2;
            phi = ysum;
            psi = lx;
            gap = fabs(phi - psi);
        }

        if (tid == 0) {
            d.out[0] = phi;
            d.out[1] = (double)iter;
            d.out[2] = (double)status;
            d.out[3] = psi;
            const double n3 = (double)n * n * n;
            atomicAdd(&g_ipm_stats[0], iter * n3);
            atomicAdd(&g_ipm_stats[1], 1.0);
            atomicAdd(&g_ipm_stats[2], (double)iter);
            atomicAdd(&g_ipm_stats[3], (double)ls_total);
        }
    }
}

__global__ void __launch_bounds__(IPM_THREADS, 1)
ipm_reg_one_kernel(IpmDesc d, int zi_in_smem)
{
    extern __shared__ __align__(16) double smem[];
    if (d.n <= 0) return;
    ipm_body_reg(d, smem, zi_in_smem, g_ipm_stats);
}

__global__ void __launch_bounds__(IPM_THREADS, 1)
ipm_reg_batched_kernel(const IpmDesc* __restrict__ descs, int zi_in_smem)
{
    extern __shared__ __align__(16) double smem[];
    const IpmDesc d = descs[blockIdx.x];
    if (d.n <= 0) return;
    ipm_body_reg(d, smem, zi_in_smem, g_ipm_stats);
}

__global__ void __launch_bounds__(IPM_THREADS, 1)
ipm_batched_kernel(const IpmDesc* __restrict__ descs, int place)
{
    extern __shared__ __align__(16) double smem[];
    const IpmDesc d = descs[blockIdx.x];
    if (d.n <= 0) return;
    ipm_body(d, smem, place);
}

__global__ void __launch_bounds__(IPM_THREADS, 1)
ipm_one_kernel(IpmDesc d, int place)
{
    extern __shared__ __align__(16) double smem[];
    if (d.n <= 0) return;
    ipm_body(d, smem, place);
}

}  // namespace

int ipm_place(int n_max, size_t smem_limit, size_t* smem_bytes)
{
    const size_t fixed = ipm_fixed_smem_doubles(n_max) * sizeof(double);
    const size_t mat = (size_t)n_max * n_max * sizeof(double);
    int place = 0;
    size_t bytes = fixed;
    if (fixed + 2 * mat <= smem_limit) {
        place = 3;
        bytes = fixed + 2 * mat;
    } else if (fixed + mat <= smem_limit) {
        place = 1;
        bytes = fixed + mat;
    }
    if (smem_bytes) *smem_bytes = bytes;
    return place;
}

size_t ipm_ws_doubles(int n, int place)
{
    const size_t nn = (size_t)n * n;
    return nn * (2 + ((place & 1) ? 0 : 1) + ((place & 2) ? 0 : 1));
}



// Optional CUDA-event timing of every IPM launch on its stream (for the
// benchmark's per-kernel roofline figure).  Each host thread records its
// begin/end event pairs in a thread-local list, so concurrent engines never
// serialise on the timer; a thread's totals are folded into the process
// totals when it exits or when the totals are read.
struct IpmTotals {
    std::atomic<bool> on{false};
    std::mutex mu;
    double ms = 0.0;
    long launches = 0;
    std::atomic<unsigned> epoch{0};   // bumped by a reset: older thread counts are dropped
};
static IpmTotals g_totals;

struct IpmThreadTimer {
    std::vector<cudaEvent_t> ev;
    size_t used = 0;
    double ms = 0.0;
    long launches = 0;
    unsigned epoch = 0;
    bool fresh = true;   // epoch is taken at the first event after creation or a fold
    template <class Launch>
    void timed(cudaStream_t s, Launch launch)
    {
        if (!g_totals.on.load()) {
            launch();
            return;
        }
        mark(s);
        launch();
        mark(s);
        if (used > 4096) collect();
    }
    void mark(cudaStream_t s)
    {
        if (fresh) {
            epoch = g_totals.epoch.load();
            fresh = false;
        }
        if (used == ev.size()) {
            cudaEvent_t e;
            BQB_CUDA(cudaEventCreate(&e));
            ev.push_back(e);
        }
        BQB_CUDA(cudaEventRecord(ev[used++], s));
    }
    void collect()
    {
        if (used >= 2 && cudaEventSynchronize(ev[used - 1]) == cudaSuccess) {
            for (size_t i = 0; i + 1 < used; i += 2) {
                float t = 0.f;
                if (cudaEventElapsedTime(&t, ev[i], ev[i + 1]) != cudaSuccess) continue;
                ms += t;
                ++launches;
            }
        }
        used = 0;
    }
    // Fold this thread's counts into the process totals.
    void fold()
    {
        collect();
        std::lock_guard<std::mutex> lock(g_totals.mu);
        if (!fresh && epoch == g_totals.epoch.load()) {
            g_totals.ms += ms;
            g_totals.launches += launches;
        }
        fresh = true;
        ms = 0.0;
        launches = 0;
    }
    ~IpmThreadTimer()
    {
        if (used > 0) fold();
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
};
static thread_local IpmThreadTimer t_timer;

// Register path (n <= 128): F always in shared memory; Zi too when it fits.
// Its fixed shared-memory part is smaller than the staged path's
// (ipm_fixed_smem_doubles), so whenever ipm_place puts both matrices in
// shared memory this path does too, and the workspace ipm_ws_doubles gives
// for ipm_place's placement always covers it (2 or 3 n^2 doubles).
static int ipm_reg_place(int n_max, size_t smem_limit, size_t* smem_bytes)
{
    const size_t fixed = ipm_reg_fixed_smem_doubles(n_max) * sizeof(double);
    const size_t mat = (size_t)n_max * n_max * sizeof(double);
    const int zi = fixed + 2 * mat <= smem_limit ? 1 : 0;
    *smem_bytes = fixed + (zi ? 2 : 1) * mat;
    return zi;
}

void ipm_launch(const IpmDesc* d_descs, int nprob, int n_max, cudaStream_t s)
{
    if (nprob <= 0) return;
    size_t bytes = 0;
    if (n_max <= RM_NMAX) {
        const int zi = ipm_reg_place(n_max, rt().smem_optin, &bytes);
        BQB_SMEM_LIMIT(ipm_reg_batched_kernel, bytes);
        t_timer.timed(s, [&] { ipm_reg_batched_kernel<<<nprob, IPM_THREADS, bytes, s>>>(d_descs, zi); });
        BQB_COUNT_LAUNCH();
        check_launch("ipm_reg_batched_kernel");
        return;
    }
    const int place = ipm_place(n_max, rt().smem_optin, &bytes);
    BQB_SMEM_LIMIT(ipm_batched_kernel, bytes);
    t_timer.timed(s, [&] { ipm_batched_kernel<<<nprob, IPM_THREADS, bytes, s>>>(d_descs, place); });
    BQB_COUNT_LAUNCH();
    check_launch("ipm_batched_kernel");
}

void ipm_launch_one(const IpmDesc& d, cudaStream_t s)
{
    size_t bytes = 0;
    if (d.n <= RM_NMAX) {
        const int zi = ipm_reg_place(d.n, rt().smem_optin, &bytes);
        BQB_SMEM_LIMIT(ipm_reg_one_kernel, bytes);
        t_timer.timed(s, [&] { ipm_reg_one_kernel<<<1, IPM_THREADS, bytes, s>>>(d, zi); });
        BQB_COUNT_LAUNCH();
        check_launch("ipm_reg_one_kernel");
        return;
    }
    const int place = ipm_place(d.n, rt().smem_optin, &bytes);
    BQB_SMEM_LIMIT(ipm_one_kernel, bytes);
    t_timer.timed(s, [&] { ipm_one_kernel<<<1, IPM_THREADS, bytes, s>>>(d, place); });
    BQB_COUNT_LAUNCH();
    check_launch("ipm_one_kernel");
}

// Single-problem launch for callers that manage the scratch (d.ws) and the
// placement themselves; records no timing events and allocates nothing.
cudaError_t ipm_launch_prepared(const IpmDesc& d, int place, size_t smem_bytes, cudaStream_t s)
{
    cudaError_t e = raise_smem_limit((const void*)ipm_one_kernel, smem_bytes);
    if (e != cudaSuccess) return e;
    ipm_one_kernel<<<1, IPM_THREADS, smem_bytes, s>>>(d, place);
    BQB_COUNT_LAUNCH();
    return cudaGetLastError();
}

}  // namespace bqb

namespace bqb {

double* ipm_stats_device()
{
    void* p = nullptr;
    BQB_CUDA(cudaGetSymbolAddress(&p, g_ipm_stats));
    return (double*)p;
}

}  // namespace bqb

// ---- work/timing counters of the IPM kernels ------------------------------

extern "C" __attribute__((visibility("default"))) void bqb_stats_enable(int on)
{
    bqb::rt();
    bqb::g_totals.on.store(on != 0);
}

extern "C" __attribute__((visibility("default"))) void bqb_stats_reset(void)
{
    bqb::rt();
    bqb::t_timer.collect();
    {
        std::lock_guard<std::mutex> lock(bqb::g_totals.mu);
        ++bqb::g_totals.epoch;
        bqb::g_totals.ms = 0.0;
        bqb::g_totals.launches = 0;
    }
    bqb::t_timer.fresh = true;
    bqb::t_timer.ms = 0.0;
    bqb::t_timer.launches = 0;
    const double z[4] = {0, 0, 0, 0};
    BQB_CUDA(cudaMemcpyToSymbol(bqb::g_ipm_stats, z, sizeof z));
}

// out[0] sum(iterations * n^3), out[1] problems, out[2] iterations,
// out[3] line-search factorizations, out[4] summed kernel time (ms, CUDA
// events), out[5] timed launches.
extern "C" __attribute__((visibility("default"))) void bqb_ipm_stats(double* out)
{
    bqb::rt();
    BQB_CUDA(cudaDeviceSynchronize());
    bqb::t_timer.fold();
    BQB_CUDA(cudaMemcpyFromSymbol(out, bqb::g_ipm_stats, 4 * sizeof(double)));
    std::lock_guard<std::mutex> lock(bqb::g_totals.mu);
    out[4] = bqb::g_totals.ms;
    out[5] = (double)bqb::g_totals.launches;
}

extern "C" __attribute__((visibility("default"))) void* bqb_stream(void)
{
    return (void*)bqb::rt().stream;
}
