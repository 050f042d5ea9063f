// Shared device helpers and runtime plumbing for the B200 bounding path.
#pragma once
#include <atomic>

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

namespace bqb {

// ---------------------------------------------------------------------------
// Error handling.  Every CUDA call goes through BQB_CUDA; a failure records
// the message (bqb_last_error) and calls the abort hook, which by default
// exits with code 10 like the reference's MPI_Abort(MPI_COMM_WORLD, 10).
// ---------------------------------------------------------------------------
void fatal(const char* where, const char* msg);
void set_error(const char* where, const char* msg);

#define BQB_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t _e = (call);                                              \
        if (_e != cudaSuccess) ::bqb::fatal(#call, cudaGetErrorString(_e));   \
    } while (0)

// ---------------------------------------------------------------------------
// Warp / block reductions (deterministic fixed trees).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum over the block; every thread gets the result.  `red` needs 33 doubles
// of shared memory.  Contains three __syncthreads().
__device__ __forceinline__ double block_sum(double v, double* red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double r = lane < nw ? red[lane] : 0.0;
        r = warp_sum(r);
        if (lane == 0) red[32] = r;
    }
    __syncthreads();
    double r = red[32];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double block_max(double v, double* red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_max(v);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double r = lane < nw ? red[lane] : -1e300;
        r = warp_max(r);
        if (lane == 0) red[32] = r;
    }
    __syncthreads();
    double r = red[32];
    __syncthreads();
    return r;
}

// Order-preserving map double -> uint64 (for atomicMax on doubles).
__device__ __forceinline__ unsigned long long dbl_to_ordered(double x)
{
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ inline double ordered_to_dbl(unsigned long long u)
{
    unsigned long long v = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
    double d;
    memcpy(&d, &v, sizeof d);
    return d;
}

// ---------------------------------------------------------------------------
// Growable device / pinned-host buffers.
// ---------------------------------------------------------------------------
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    T* ensure(size_t n)
    {
        if (n <= cap) return p;
        if (p) BQB_CUDA(cudaFree(p));
        size_t c = n < 64 ? 64 : n;
        BQB_CUDA(cudaMalloc(&p, c * sizeof(T)));
        cap = c;
        return p;
    }
    // grow keeping the first `keep` elements
    T* grow_keep(size_t n, size_t keep, cudaStream_t s)
    {
        if (n <= cap) return p;
        T* q = nullptr;
        size_t c = n + n / 2;
        BQB_CUDA(cudaMalloc(&q, c * sizeof(T)));
        if (p && keep) BQB_CUDA(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s));
        if (p) {
            BQB_CUDA(cudaStreamSynchronize(s));
            BQB_CUDA(cudaFree(p));
        }
        p = q;
        cap = c;
        return p;
    }
};

template <class T>
struct HostBuf {
    T* p = nullptr;
    size_t cap = 0;
    T* ensure(size_t n)
    {
        if (n <= cap) return p;
        if (p) BQB_CUDA(cudaFreeHost(p));
        size_t c = n < 64 ? 64 : n;
        BQB_CUDA(cudaMallocHost(&p, c * sizeof(T)));
        cap = c;
        return p;
    }
};

// Process-wide runtime: one device and the library stream the drop-in entry
// points use (the reference is single-threaded and so are they); concurrent
// bounding runs on engines with streams of their own.
struct Runtime {
    int device = -1;
    int num_sms = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
};
Runtime& rt();

// Kernel-launch counter (reported by bench.py as gpu_launches).
extern std::atomic<unsigned long long> g_launches;
#define BQB_COUNT_LAUNCH() (++::bqb::g_launches)

// Raise a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`.  The limit is a per-(device, function) setting shared by
// every host thread, so it only ever grows (a thread lowering it could invalidate another thread's launch
// in flight between its own raise and launch).  Allocation-free.
cudaError_t raise_smem_limit(const void* fn, size_t bytes);

// Set on the bounding pool's worker threads (a fatal error there ends the
// process with _exit rather than exit).
extern thread_local bool t_pool_worker;
#define BQB_SMEM_LIMIT(fn, bytes) BQB_CUDA(::bqb::raise_smem_limit((const void*)(fn), (size_t)(bytes)))

inline void check_launch(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fatal(what, cudaGetErrorString(e));
}

}  // namespace bqb
