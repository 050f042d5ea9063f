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

__device__ __forceinline__ uint32_t sa_next(uint64_t& state)
{
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (uint32_t)(z >> 33);
}

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
    if (tid == 0) {
        // starting temperature k^2 * (n + sum_{i<j} 2|X_ij|) / (n (n-1))
        double sumX = n;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) sumX = __dadd_rn(sumX, __dmul_rn(2.0, fabs(Xs[j + (size_t)i * n])));
        double t = (double)(K * K);
        t = __dmul_rn(t, sumX);
        t = __ddiv_rn(t, (double)(n * (n - 1)));
        sT[0] = t;
    }
    __syncthreads();
    const int c = blockIdx.x * SA_CHAINS_PER_CTA + tid;
    if (c >= chains) return;
    const int type = c % types + 1;
    // H(a, b) = e_a e_b with e_a = -1 for a < type - 1, else +1
    auto e = [&](int a) { return a < type - 1 ? -1 : 1; };
    auto PA = [&](int i) -> unsigned short& { return P[(size_t)i * SA_CHAINS_PER_CTA + tid]; };
    auto XA = [&](int a, int b) { return Xs[a + (size_t)n * b]; };

    uint64_t rs = seed + (uint64_t)(c + 1) * SA_CHAIN_STRIDE;
    for (int i = 0; i < n; ++i) PA(i) = (unsigned short)i;
    for (int i = n - 1; i > 0; --i) {
        const int r = (int)(sa_next(rs) % (uint32_t)i);
        const unsigned short tmp = PA(i);
        PA(i) = PA(r);
        PA(r) = tmp;
    }
    double t1 = sT[0];
    int m1 = n;
    double sol = K;
    for (int i = 0; i < K; ++i)
        for (int j = i + 1; j < K; ++j)
            sol = __dadd_rn(sol, __dmul_rn((double)(2 * e(j) * e(i)), XA(PA(j), PA(i))));
    double cost = 1e9;
    int best[7] = {0, 0, 0, 0, 0, 0, 0};
    int not_done = 1, rounds = 0;
    while (not_done > 0 && rounds < SA_MAX_ROUNDS) {
        not_done = 0;
        for (int it = 0; it < m1; ++it) {
            int i1 = (int)(sa_next(rs) % (uint32_t)K);
            int i2 = (int)(sa_next(rs) % (uint32_t)n);
            if (i2 < i1) {
                const int tmp = i1;
                i1 = i2;
                i2 = tmp;
            }
            const int p1 = PA(i1), p2 = PA(i2);
            double delta = 0.0;
            for (int i = 0; i < K; ++i) {
                const int pi = PA(i);
                const double d = __dsub_rn(XA(pi, p2), XA(pi, p1));
                delta = __dadd_rn(delta, e(i) * e(i1) > 0 ? d : -d);
            }
            if (i2 < K)
                for (int i = 0; i < K; ++i) {
                    const int pi = PA(i);
                    const double d = __dsub_rn(XA(pi, p1), XA(pi, p2));
                    delta = __dadd_rn(delta, e(i) * e(i2) > 0 ? d : -d);
                }
            delta = __dmul_rn(delta, 2.0);
            const double tv1 = __dsub_rn(2.0, __dmul_rn(2.0, XA(p2, p1)));
            double tv2 = 1.0;
            if (i2 < K) tv2 = __dadd_rn(tv2, __dadd_rn((double)(-2 * e(i1) * e(i2)), 1.0));
            delta = __dadd_rn(delta, __dmul_rn(tv1, tv2));
            const double sol_temp = __dadd_rn(sol, delta);
            int accept;
            if (delta > 0) {
                const double dt1 = __ddiv_rn(delta, t1);
                if (dt1 > 5)
                    accept = 0;
                else
                    accept = __ddiv_rn((double)sa_next(rs), (double)SA_RAND_MAX) < exp(-dt1) ? 1 : 0;
            } else {
                accept = 1;
            }
            if (accept) {
                if (fabs(delta) > 0.001) not_done = 1;
                PA(i1) = (unsigned short)p2;
                PA(i2) = (unsigned short)p1;
                sol = sol_temp;
                if (sol < cost) {
                    cost = sol;
#pragma unroll
                    for (int a = 0; a < 7; ++a)
                        if (a < K) best[a] = PA(a);
                }
            }
        }
        t1 = __dmul_rn(t1, 0.6);
        m1 = (int)round(__dmul_rn((double)m1, 1.1));
        ++rounds;
    }
    if (not_done > 0) atomicOr(status, 1);
    cost_out[c] = cost;
#pragma unroll
    for (int a = 0; a < 7; ++a) perm_out[(size_t)c * 7 + a] = a < K ? best[a] : 0;
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
