// Annealing chains of the k-gonal separation, one chain per thread
// (src/qap_simulated_annealing.c:12-190 restated per chain).
//
// Layout: the chains of a CTA share the matrix X, staged in shared memory
// when it fits (n <= 158 for 64 chains), and keep their permutations in
// shared memory interleaved by chain (perm entry i of chain t at
// i * SA_CHAINS_PER_CTA + t) so that the threads of a warp touching the same
// position hit different banks.  The sum that sets the starting temperature
// is taken by one thread in the reference's order, so every chain's
// arithmetic is the sequential arithmetic of the restatement it is checked
// against (IEEE double, no reassociation).
#include <math.h>

#include "kgon_sa.cuh"

namespace bqb {

namespace {

__global__ void __launch_bounds__(SA_CHAINS_PER_CTA)
kgon_sa_kernel(const double* __restrict__ X, int n, int K, int types, int chains, unsigned long long seed,
               int x_in_smem, double* __restrict__ cost_out, int* __restrict__ perm_out, int* __restrict__ status)
{
    extern __shared__ __align__(16) double sa_smem[];
    const int tid = threadIdx.x;
    const size_t nn = (size_t)n * n;
    double* sX = sa_smem;
    double* sT = sa_smem + (x_in_smem ? nn : 0);
    unsigned short* P = (unsigned short*)(sT + 2);
    if (x_in_smem)
        for (size_t e = tid; e < nn; e += blockDim.x) sX[e] = X[e];
    __syncthreads();
    const double* Xs = x_in_smem ? sX : X;
    if (tid == 0) sT[0] = kgon_temperature(Xs, n, K);
    __syncthreads();
    const int c = blockIdx.x * SA_CHAINS_PER_CTA + tid;
    if (c >= chains) return;
    kgon_chain(Xs, n, K, types, c, seed, sT[0], P, SA_CHAINS_PER_CTA, tid, cost_out, perm_out, status);
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
    const size_t perm_bytes = (size_t)n * SA_CHAINS_PER_CTA * sizeof(unsigned short);
    const size_t fixed = 2 * sizeof(double) + perm_bytes;
    const size_t xbytes = (size_t)n * n * sizeof(double);
    const int x_in_smem = fixed + xbytes <= rt().smem_optin ? 1 : 0;
    const size_t bytes = fixed + (x_in_smem ? xbytes : 0);
    BQB_SMEM_LIMIT(kgon_sa_kernel, bytes);
    BQB_CUDA(cudaMemsetAsync(st.status.p, 0, sizeof(int), s));
    const int grid = (chains + SA_CHAINS_PER_CTA - 1) / SA_CHAINS_PER_CTA;
    kgon_sa_kernel<<<grid, SA_CHAINS_PER_CTA, bytes, s>>>(dX, n, k, types, chains, (unsigned long long)seed,
                                                         x_in_smem, st.cost.p, st.perm.p, st.status.p);
    BQB_COUNT_LAUNCH();
    check_launch("kgon_sa_kernel");
    BQB_CUDA(cudaMemcpyAsync(st.hcost.p, st.cost.p, chains * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(st.hperm.p, st.perm.p, (size_t)chains * 7 * sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(st.hstat.p, st.status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace bqb
