// Annealing chains of the k-gonal separation, one chain per warp
// (src/qap_simulated_annealing.c:12-190 restated per chain; the warp
// evaluates the moves of its chain speculatively, kgon_chain_warp).
//
// Layout: the chains of a CTA share the matrix X, staged in shared memory
// when it fits, and each warp keeps its chain's permutation in shared
// memory.  The sum that sets the starting temperature is taken by one thread
// in the reference's order, so every chain's arithmetic is the sequential
// arithmetic of the restatement it is checked against (IEEE double, no
// reassociation).
#include <math.h>

#include "kgon_sa.cuh"

namespace bqb {

namespace {

constexpr int SA_WARPS = 8;   // chains per CTA

__global__ void __launch_bounds__(SA_WARPS * 32)
kgon_sa_kernel(const double* __restrict__ X, int n, int K, int types, int chains, unsigned long long seed,
               int x_in_smem, double* __restrict__ cost_out, int* __restrict__ perm_out, int* __restrict__ status)
{
    extern __shared__ __align__(16) double sa_smem[];
    const int tid = threadIdx.x, w = tid >> 5;
    const size_t nn = (size_t)n * n;
    double* sX = sa_smem;
    double* sT = sa_smem + (x_in_smem ? nn : 0);
    unsigned short* P = (unsigned short*)(sT + 2) + (size_t)w * n;
    if (x_in_smem)
        for (size_t e = tid; e < nn; e += blockDim.x) sX[e] = X[e];
    __syncthreads();
    const double* Xs = x_in_smem ? sX : X;
    if (tid == 0) sT[0] = kgon_temperature(Xs, n, K);
    __syncthreads();
    const int c = blockIdx.x * SA_WARPS + w;
    if (c >= chains) return;
    kgon_chain_warp(Xs, n, K, types, c, seed, sT[0], P, cost_out, perm_out, status);
}

}  // namespace

void kgon_sa_device(KgonSaState& st, const double* dX, int n, int k, int types, int chains, uint64_t seed,
                    cudaStream_t s)
{
    if (chains <= 0) return;
    st.cost.ensure(chains);
    st.perm.ensure((size_t)chains * 7);
    st.status.ensure(1);
    st.hcost.ensure(chains);
    st.hperm.ensure((size_t)chains * 7);
    st.hstat.ensure(1);
    const size_t perm_bytes = (size_t)n * SA_WARPS * sizeof(unsigned short);
    const size_t fixed = 2 * sizeof(double) + perm_bytes;
    const size_t xbytes = (size_t)n * n * sizeof(double);
    const int x_in_smem = fixed + xbytes <= rt().smem_optin ? 1 : 0;
    const size_t bytes = fixed + (x_in_smem ? xbytes : 0);
    BQB_SMEM_LIMIT(kgon_sa_kernel, bytes);
    BQB_CUDA(cudaMemsetAsync(st.status.p, 0, sizeof(int), s));
    const int grid = (chains + SA_WARPS - 1) / SA_WARPS;
    kgon_sa_kernel<<<grid, SA_WARPS * 32, bytes, s>>>(dX, n, k, types, chains, (unsigned long long)seed,
                                                         x_in_smem, st.cost.p, st.perm.p, st.status.p);
    BQB_COUNT_LAUNCH();
    check_launch("kgon_sa_kernel");
    BQB_CUDA(cudaMemcpyAsync(st.hcost.p, st.cost.p, chains * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(st.hperm.p, st.perm.p, (size_t)chains * 7 * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(st.hstat.p, st.status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace bqb
