// Triangle separation (src/cutting_planes.c:20-127) on the GPU.
//
// The reference scans type = 1..4, i = 0..n-1, j < i, k < j in that order,
// evaluates value = +-X_ij +-X_ik +-X_jk - 1 (src/cutting_planes.c:24-36;
// summed in the order the reference build uses, see tri_values),
// tracks the maximum, and keeps a streaming list of at most TriIneq cuts
// with value > violated_TriIneq: the first TriIneq fill the list, later ones
// replace the first-found minimum when strictly larger (:70-116).
//
// GPU form, three steps:
//  1. scan: one warp per (i, j) pair, lanes over k, all four types from the
//     same three X entries (X read as columns of its transpose, so lanes
//     load contiguous doubles).  Pass 1 counts violated cuts per (type,
//     pair) and reduces the maximum; an exclusive scan gives each (type,
//     pair) its place; pass 2 writes the candidates in exactly the
//     reference's scan order (ballot + popc inside each warp).
//  2. replay: one warp replays the streaming top-K over the ordered
//     candidates with a (value, slot) min-heap in shared memory.  The heap
//     top is the reference's "first-found minimum" (lowest slot among equal
//     minima), so the final list, including slot order, is the reference's.
//     Lanes test 32 candidates at a time against the current minimum and
//     only the few that beat it are inserted one by one.
//  3. the host reads back at most TriIneq records.
#include <math.h>

#include "trisep.cuh"

namespace bqb {
namespace {

constexpr double BIG_NUMBER = 1e9;   // src/biqbin.h:35

__global__ void transpose_kernel(const double* __restrict__ X, double* __restrict__ XT, int n)
{
    __shared__ double tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int row = by + r, col = bx + threadIdx.x;
        if (row < n && col < n) tile[r][threadIdx.x] = X[row + (size_t)col * n];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int col = by + threadIdx.x, row = bx + r;   // XT(row, col) = X(col, row)
        if (row < n && col < n) XT[row + (size_t)col * n] = tile[threadIdx.x][r];
    }
}

__device__ __forceinline__ void pair_decode(long long p, int* i, int* j)
{
    int ii = (int)floor((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
    while ((long long)ii * (ii - 1) / 2 > p) --ii;
    while ((long long)(ii + 1) * ii / 2 <= p) ++ii;
    *i = ii;
    *j = (int)(p - (long long)ii * (ii - 1) / 2);
}

template <bool WRITE>
__global__ void __launch_bounds__(256) tri_scan_kernel(const double* __restrict__ X,
                                                       const double* __restrict__ XT, int n,
                                                       long long P, double thr,
                                                       uint32_t* __restrict__ cnt,
                                                       TriCand* __restrict__ cand,
                                                       unsigned long long* __restrict__ gmax)
{
    const int lane = threadIdx.x & 31;
    const long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (p >= P) return;
    int i, j;
    pair_decode(p, &i, &j);
    const double a = X[i + (size_t)j * n];
    const double* Bi = XT + (size_t)i * n;   // X[i + k n]
    const double* Bj = XT + (size_t)j * n;   // X[j + k n]
    uint32_t c4[4] = {0u, 0u, 0u, 0u};
    uint32_t base[4] = {0u, 0u, 0u, 0u};
    if (WRITE) {
#pragma unroll
        for (int t = 0; t < 4; ++t) base[t] = cnt[t * P + p];
    }
    double vmax = -BIG_NUMBER;
    const unsigned lt = (1u << lane) - 1u;
    for (int k0 = 0; k0 < j; k0 += 32) {
        const int k = k0 + lane;
        const bool valid = k < j;
        const double b = valid ? Bi[k] : 0.0;
        const double c = valid ? Bj[k] : 0.0;
        double v[4];
        tri_values(a, b, c, v);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const bool hit = valid && v[t] > thr;
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (!WRITE) {
                if (valid) vmax = fmax(vmax, v[t]);
            } else if (hit) {
                TriCand cd;
                cd.value = v[t];
                cd.code = tri_code(t + 1, i, j, k);
                cd.pad_ = 0u;
                cand[base[t] + c4[t] + __popc(m & lt)] = cd;
            }
            c4[t] += __popc(m);
        }
    }
    if (!WRITE) {
        vmax = warp_max(vmax);
        if (lane == 0) {
#pragma unroll
            for (int t = 0; t < 4; ++t) cnt[t * P + p] = c4[t];
            atomicMax(gmax, dbl_to_ordered(vmax));
        }
    }
}

// Exclusive scan of N counts in place (single block); total -> *total.
__global__ void __launch_bounds__(1024) scan_kernel(uint32_t* __restrict__ a, long long N,
                                                    unsigned long long* __restrict__ total)
{
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned long long carry_s;
    constexpr int ITEMS = 8;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) carry_s = 0;
    __syncthreads();
    for (long long base = 0; base < N; base += 1024LL * ITEMS) {
        uint32_t v[ITEMS];
        unsigned long long s = 0;
        const long long off = base + (long long)tid * ITEMS;
#pragma unroll
        for (int q = 0; q < ITEMS; ++q) {
            v[q] = (off + q < N) ? a[off + q] : 0u;
            s += v[q];
        }
        unsigned long long incl = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            unsigned long long w = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        unsigned long long run = carry_s + (warp ? wsum[warp - 1] : 0ull) + incl - s;
#pragma unroll
        for (int q = 0; q < ITEMS; ++q) {
            if (off + q < N) a[off + q] = (uint32_t)run;
            run += v[q];
        }
        __syncthreads();
        if (tid == 0) carry_s += wsum[31];
        __syncthreads();
    }
    if (tid == 0) *total = carry_s;
}

__device__ __forceinline__ bool heap_less(const double* hv, const int* hs, int a, int b)
{
    return hv[a] < hv[b] || (hv[a] == hv[b] && hs[a] < hs[b]);
}

__device__ void heap_sift_down(double* hv, int* hs, int T, int i)
{
    while (true) {
        const int l = 2 * i + 1, r = l + 1;
        int m = i;
        if (l < T && heap_less(hv, hs, l, m)) m = l;
        if (r < T && heap_less(hv, hs, r, m)) m = r;
        if (m == i) return;
        const double tv = hv[i];
        hv[i] = hv[m];
        hv[m] = tv;
        const int ts = hs[i];
        hs[i] = hs[m];
        hs[m] = ts;
        i = m;
    }
}

// One warp.  Streaming top-T replay (src/cutting_planes.c:70-116).
__global__ void tri_replay_kernel(const TriCand* __restrict__ cand,
                                  const unsigned long long* __restrict__ misc, int T,
                                  TriCand* __restrict__ list, int* __restrict__ out_size)
{
    extern __shared__ __align__(16) double hsm[];
    const int lane = threadIdx.x;
    const long long V = (long long)misc[1];
    if (T <= 0) {
        if (lane == 0) *out_size = 0;
        return;
    }
    if (V <= T) {
        for (long long q = lane; q < V; q += 32) list[q] = cand[q];
        if (lane == 0) *out_size = (int)V;
        return;
    }
    double* hv = hsm;
    int* hs = (int*)(hv + T);
    for (int q = lane; q < T; q += 32) {
        const TriCand c = cand[q];
        list[q] = c;
        hv[q] = c.value;
        hs[q] = q;
    }
    __syncwarp();
    if (lane == 0)
        for (int q = T / 2 - 1; q >= 0; --q) heap_sift_down(hv, hs, T, q);
    __syncwarp();
    for (long long base = T; base < V; base += 32) {
        const long long idx = base + lane;
        const double v = idx < V ? cand[idx].value : -INFINITY;
        double thr = hv[0];
        unsigned mask = __ballot_sync(0xffffffffu, v > thr);
        while (mask) {
            const int l = __ffs(mask) - 1;
            const double vl = __shfl_sync(0xffffffffu, v, l);
            __syncwarp();
            if (lane == 0) {
                const int slot = hs[0];
                list[slot] = cand[base + l];
                hv[0] = vl;
                heap_sift_down(hv, hs, T, 0);
            }
            __syncwarp();
            thr = hv[0];
            mask = __ballot_sync(0xffffffffu, lane > l && v > thr);
        }
    }
    if (lane == 0) *out_size = T;
}

}  // namespace

double trisep_device(TriSepState& st, const double* dX, int n, int tri_ineq, double violated,
                     int* list_size, cudaStream_t s)
{
    const long long P = (long long)n * (n - 1) / 2;
    const long long ncand_max = n >= 3 ? 4LL * n * (n - 1) * (n - 2) / 6 : 0;
    unsigned long long* misc = st.misc.ensure(4);
    // misc[0]: running maximum as an order-preserving integer, starting at
    // -BIG_NUMBER (the reference's initial maxAllIneq); misc[1]: candidate
    // count; misc[2]: list size.
    unsigned long long negbig;
    {
        const double d = -BIG_NUMBER;
        unsigned long long u;
        memcpy(&u, &d, sizeof u);
        negbig = (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
    }
    const unsigned long long h0[4] = {negbig, 0ull, 0ull, 0ull};
    unsigned long long* hm = st.hmisc.ensure(4);
    memcpy(hm, h0, sizeof h0);
    BQB_CUDA(cudaMemcpyAsync(misc, hm, 4 * sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
    if (P <= 0 || n < 3) {
        BQB_CUDA(cudaStreamSynchronize(s));
        *list_size = 0;
        return -BIG_NUMBER;
    }
    double* XT = st.XT.ensure((size_t)n * n);
    uint32_t* cnt = st.cnt.ensure((size_t)(4 * P));
    TriCand* cand = st.cand.ensure((size_t)ncand_max);
    TriCand* list = st.list.ensure((size_t)(tri_ineq > 0 ? tri_ineq : 1));
    TriCand* hlist = st.hlist.ensure((size_t)(tri_ineq > 0 ? tri_ineq : 1));
    int* dsize = (int*)(misc + 2);

    dim3 tb(32, 8), tg((n + 31) / 32, (n + 31) / 32);
    transpose_kernel<<<tg, tb, 0, s>>>(dX, XT, n);
    BQB_COUNT_LAUNCH();
    const long long threads = P * 32;
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    tri_scan_kernel<false><<<blocks, 256, 0, s>>>(dX, XT, n, P, violated, cnt, nullptr, misc);
    BQB_COUNT_LAUNCH();
    scan_kernel<<<1, 1024, 0, s>>>(cnt, 4 * P, misc + 1);
    BQB_COUNT_LAUNCH();
    tri_scan_kernel<true><<<blocks, 256, 0, s>>>(dX, XT, n, P, violated, cnt, cand, misc);
    BQB_COUNT_LAUNCH();
    const size_t heap_bytes = (size_t)(tri_ineq > 0 ? tri_ineq : 1) * (sizeof(double) + sizeof(int));
    BQB_SMEM_LIMIT(tri_replay_kernel, heap_bytes);
    tri_replay_kernel<<<1, 32, heap_bytes, s>>>(cand, misc, tri_ineq, list, dsize);
    BQB_COUNT_LAUNCH();
    check_launch("trisep");
    BQB_CUDA(cudaMemcpyAsync(hm, misc, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    const int size = *(int*)(hm + 2);
    if (size > 0) {
        BQB_CUDA(cudaMemcpyAsync(hlist, list, (size_t)size * sizeof(TriCand), cudaMemcpyDeviceToHost, s));
        BQB_CUDA(cudaStreamSynchronize(s));
    }
    *list_size = size;
    return ordered_to_dbl(hm[0]);
}

}  // namespace bqb
