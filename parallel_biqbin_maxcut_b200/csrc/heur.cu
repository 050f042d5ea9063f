// Goemans-Williamson rounding with 1-opt local search (src/heuristic.c) on
// the GPU.
//
//  * potrf_kernel: Cholesky of the n x n Z (shared memory when it fits).
//  * gw_project_kernel: s = L v for every hyperplane v (one thread per
//    (hyperplane, row)), summed over j <= i in the reference's order with
//    separate multiply and add, so the sign is the reference's sign of the
//    same factor; x = sign(s) with sign(0) = +1 (src/heuristic.c:145-165).
//  * one_opt_kernel: one warp per cut.  Lx, delta and x live in shared
//    memory; the argmax is a warp shuffle reduction that keeps the first
//    index among equal maxima, as the reference's strict `>` scan does
//    (src/heuristic.c:227-234, 279-286).  All values are multiples of 1/4 of
//    integers, so Lx and the cost are exact whatever the summation order.
//  * eval_kernel: lift each cut to the 0/1 vector of the original problem
//    (fixed variables from the node) and evaluate sum_ij L_ij s_i s_j
//    exactly (src/heuristic.c:170-181, src/bab_functions.c:96-107).
//  * select_kernel: first index of the maximum (update_best replaces only
//    on strict improvement, src/heuristic.c:311-315).
#include <math.h>

#include "cta_linalg.cuh"
#include "heur.cuh"

namespace bqb {

namespace {

constexpr int POTRF_THREADS = 512;

__global__ void __launch_bounds__(POTRF_THREADS) potrf_kernel(double* Z, int n, int* status, int in_smem)
{
    extern __shared__ __align__(16) double sm[];
    double* col = sm;
    double* A = in_smem ? sm + ((n + 1) & ~1) : Z;
    const size_t nn = (size_t)n * n;
    if (in_smem) {
        for (size_t e = threadIdx.x; e < nn; e += blockDim.x) A[e] = Z[e];
        __syncthreads();
    }
    const bool ok = cta_potrf_lower(A, n, n, col);
    __syncthreads();
    if (in_smem && ok) {
        for (size_t e = threadIdx.x; e < nn; e += blockDim.x) Z[e] = A[e];
    }
    if (threadIdx.x == 0) *status = ok ? 0 : 1;
}

__global__ void remix_kernel(double* __restrict__ Z, const double* __restrict__ X,
                             const double* __restrict__ xh, double c, int n)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)n * n) return;
    const int i = (int)(e % n), j = (int)(e / n);
    const double a = (1.0 - c) * X[e];
    Z[e] = a + xh[i] * (c * xh[j]);
}

__global__ void gw_project_kernel(const double* __restrict__ Lf, const double* __restrict__ V, int n,
                                  int* __restrict__ x)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int h = blockIdx.y;
    if (i >= n) return;
    const double* v = V + (size_t)h * n;
    double acc = 0.0;
    for (int j = 0; j <= i; ++j) acc = __dadd_rn(acc, __dmul_rn(v[j], Lf[i + (size_t)j * n]));
    x[(size_t)h * n + i] = (acc < 0) ? -1 : 1;
}

// One warp per cut; shared: d[n] for the block, then per warp Lx[n], x[n].
__global__ void one_opt_kernel(const double* __restrict__ PL, int n, int* __restrict__ xs, int count,
                               double* __restrict__ cost_out, int* __restrict__ status)
{
    extern __shared__ __align__(16) double sm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nv = (n + 1) & ~1;
    double* d = sm;
    for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = PL[i + (size_t)i * n];
    __syncthreads();
    const int h = blockIdx.x * nw + warp;
    if (h >= count) return;
    double* Lx = sm + nv + (size_t)warp * 2 * nv;
    int* x = (int*)(Lx + nv);
    int* xg = xs + (size_t)h * n;
    for (int i = lane; i < n; i += 32) x[i] = xg[i];
    __syncwarp();
    double part = 0.0;
    for (int i = lane; i < n; i += 32) {
        double acc = 0.0;
        for (int j = 0; j < n; ++j) acc += PL[i + (size_t)j * n] * (double)x[j];
        Lx[i] = acc;
        part += (double)x[i] * acc;
    }
    double cost = warp_sum(part);
    __syncwarp();
    const int cap = 10 * n + 100;
    int flips = 0;
    while (true) {
        double best = -1e300;
        int idx = 0x7fffffff;
        for (int i = lane; i < n; i += 32) {
            const double dl = d[i] - (double)x[i] * Lx[i];
            if (dl > best) {
                best = dl;
                idx = i;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
            if (ob > best || (ob == best && oi < idx)) {
                best = ob;
                idx = oi;
            }
        }
        if (!(best > 0.001)) break;
        if (++flips > cap) {
            if (lane == 0) atomicOr(status, 2);
            break;
        }
        const double sgn = (x[idx] > 0) ? -2.0 : 2.0;
        const double* col = PL + (size_t)idx * n;
        __syncwarp();
        for (int j = lane; j < n; j += 32) {
            const double lv = col[j];
            if (fabs(lv) > 0.001) Lx[j] += sgn * lv;
        }
        if (lane == 0) x[idx] = -x[idx];
        cost += 4 * best;
        __syncwarp();
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32) xg[i] = x[i];
    if (lane == 0 && cost_out) cost_out[h] = cost;
}

// One block per cut: lift to the original 0/1 vector and evaluate.
// fix: [0, N) flags, [N, 2N) node values, [2N, 3N) rank among free vertices.
__global__ void eval_kernel(const double* __restrict__ P0L, int N0, const int* __restrict__ xs, int n,
                            const int* __restrict__ fix, int* __restrict__ sols, double* __restrict__ vals,
                            int from_x)
{
    __shared__ double red[64];
    const int h = blockIdx.x;
    const int N = N0 - 1;
    int* s = sols + (size_t)h * N;
    if (from_x) {
        const int* x = xs + (size_t)h * n;
        for (int i = threadIdx.x; i < N; i += blockDim.x)
            s[i] = fix[i] ? fix[N + i] : (x[fix[2 * N + i]] + 1) / 2;
        __syncthreads();
    }
    double part = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        if (!s[i]) continue;
        const double* Li = P0L + (size_t)i * N0;
        double r = 0.0;
        for (int j = 0; j < N; ++j)
            if (s[j]) r += Li[j];
        part += r;
    }
    const double v = block_sum(part, red);
    if (threadIdx.x == 0) vals[h] = v;
}

__global__ void select_kernel(const double* __restrict__ vals, int count, const int* __restrict__ sols,
                              int N, int* __restrict__ best, double* __restrict__ bestval)
{
    __shared__ int hbest;
    if (threadIdx.x == 0) {
        double b = -1e9;   // -BIG_NUMBER, src/heuristic.c:135
        int hb = 0;
        for (int h = 0; h < count; ++h)
            if (b < vals[h]) {
                b = vals[h];
                hb = h;
            }
        hbest = hb;
        best[0] = hb;
        *bestval = b;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += blockDim.x) best[1 + i] = sols[(size_t)hbest * N + i];
}

}  // namespace

void potrf_device(double* dZ, int n, int* dstatus, cudaStream_t s)
{
    const size_t need = ((size_t)((n + 1) & ~1) + (size_t)n * n) * sizeof(double);
    const int in_smem = need <= rt().smem_optin ? 1 : 0;
    const size_t bytes = in_smem ? need : (size_t)((n + 1) & ~1) * sizeof(double);
    BQB_SMEM_LIMIT(potrf_kernel, bytes);
    potrf_kernel<<<1, POTRF_THREADS, bytes, s>>>(dZ, n, dstatus, in_smem);
    BQB_COUNT_LAUNCH();
    check_launch("potrf_kernel");
}

void remix_device(double* dZ, const double* dX, const double* dxh, double c, int n, cudaStream_t s)
{
    const size_t nn = (size_t)n * n;
    remix_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(dZ, dX, dxh, c, n);
    BQB_COUNT_LAUNCH();
    check_launch("remix_kernel");
}

static size_t one_opt_smem(int n, int warps)
{
    const size_t nv = (size_t)((n + 1) & ~1);
    return (nv + (size_t)warps * 2 * nv) * sizeof(double);
}

void one_opt_device(HeurState& st, const double* dPL, int n, int count, cudaStream_t s)
{
    const int warps = 4;
    const size_t bytes = one_opt_smem(n, warps);
    BQB_SMEM_LIMIT(one_opt_kernel, bytes);
    one_opt_kernel<<<(count + warps - 1) / warps, warps * 32, bytes, s>>>(dPL, n, st.x.p, count, st.vals.p,
                                                                         st.status.p);
    BQB_COUNT_LAUNCH();
    check_launch("one_opt_kernel");
}

void evaluate_device(HeurState& st, const double* dP0L, int N0, int count, cudaStream_t s)
{
    eval_kernel<<<count, 128, 0, s>>>(dP0L, N0, nullptr, 0, st.fixed.p, st.sols.p, st.vals.p, 0);
    BQB_COUNT_LAUNCH();
    check_launch("eval_kernel");
}

void gw_round_device(HeurState& st, const double* dPL, int n, const double* dP0L, int N0, int num,
                     cudaStream_t s)
{
    dim3 pg((n + 127) / 128, num);
    gw_project_kernel<<<pg, 128, 0, s>>>(st.Z.p, st.V.p, n, st.x.p);
    BQB_COUNT_LAUNCH();
    gw_round_finish(st, dPL, n, dP0L, N0, num, s);
}

void gw_round_finish(HeurState& st, const double* dPL, int n, const double* dP0L, int N0, int num, cudaStream_t s)
{
    one_opt_device(st, dPL, n, num, s);
    eval_kernel<<<num, 128, 0, s>>>(dP0L, N0, st.x.p, n, st.fixed.p, st.sols.p, st.vals.p, 1);
    BQB_COUNT_LAUNCH();
    select_kernel<<<1, 256, 0, s>>>(st.vals.p, num, st.sols.p, N0 - 1, st.best.p, st.bestval.p);
    BQB_COUNT_LAUNCH();
    check_launch("gw_round");
}

}  // namespace bqb
