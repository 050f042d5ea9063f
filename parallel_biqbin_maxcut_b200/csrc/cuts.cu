// op_B (gather) and op_Bt (symmetric scatter) on the GPU.
//
// op_B restates src/operators.c:51-132: y[c] -= scale * (sum of +-X entries),
// summed over index pairs in lexicographic order of the stored tuple exactly
// as the reference writes each bracket, so results are bit-identical to a
// reference build that keeps source order.  One thread per (cut, matrix):
// one 16-byte vector load for the cut record, then k(k-1)/2 gathers from X
// (L2 resident).
//
// op_Bt restates src/operators.c:140-481: X -= B^T(t) adds +-temp to both
// X[p_a + p_b n] and X[p_b + p_a n] for every pair of every cut, with
// temp = t/2, t/4, t/6 per kind.  The reference applies the contributions to
// one entry in cut order; the GPU form is a deterministic gather: one thread
// per touched pair walks that pair's contributions (CSR built when the cut
// list changes) in cut order, so no atomics and the same rounding sequence.
#include <algorithm>

#include "cuts.cuh"

namespace bqb {

void PairCSR::build(const std::vector<CutRec>& cuts)
{
    struct E { uint32_t key, code; };
    std::vector<E> ent;
    ent.reserve(cuts.size() * 3);
    for (size_t c = 0; c < cuts.size(); ++c) {
        const CutRec& r = cuts[c];
        const unsigned p[7] = {r.x & 0xffffu, r.x >> 16, r.y & 0xffffu, r.y >> 16,
                               r.z & 0xffffu, r.z >> 16, r.w & 0xffffu};
        const int k = (int)((r.w >> 16) & 0xffu);
        const unsigned neg = (r.w >> 24) & 0x7fu;
        for (int a = 0; a < k; ++a)
            for (int b = a + 1; b < k; ++b) {
                const unsigned u = std::min(p[a], p[b]), v = std::max(p[a], p[b]);
                const unsigned sneg = ((neg >> a) ^ (neg >> b)) & 1u;   // e_a e_b = -1
                ent.push_back({u | (v << 16), (uint32_t)(c << 1) | sneg});
            }
    }
    std::stable_sort(ent.begin(), ent.end(), [](const E& a, const E& b) { return a.key < b.key; });
    pair_uv.clear();
    offsets.clear();
    contrib.clear();
    contrib.reserve(ent.size());
    for (size_t i = 0; i < ent.size(); ++i) {
        if (i == 0 || ent[i].key != ent[i - 1].key) {
            pair_uv.push_back(ent[i].key);
            offsets.push_back((uint32_t)i);
        }
        contrib.push_back(ent[i].code);
    }
    offsets.push_back((uint32_t)ent.size());
}

void DevCuts::upload(const std::vector<CutRec>& cuts, int mt, int mp, int mh, cudaStream_t s)
{
    m = (int)cuts.size();
    m_tri = mt;
    m_pent = mp;
    m_hept = mh;
    PairCSR csr;
    csr.build(cuts);
    npairs = (int)csr.pair_uv.size();
    if (m) {
        rec.ensure(m);
        BQB_CUDA(cudaMemcpyAsync(rec.p, cuts.data(), m * sizeof(CutRec), cudaMemcpyHostToDevice, s));
    }
    if (npairs) {
        pair_uv.ensure(npairs);
        offsets.ensure(npairs + 1);
        contrib.ensure(csr.contrib.size());
        BQB_CUDA(cudaMemcpyAsync(pair_uv.p, csr.pair_uv.data(), npairs * 4, cudaMemcpyHostToDevice, s));
        BQB_CUDA(cudaMemcpyAsync(offsets.p, csr.offsets.data(), (npairs + 1) * 4, cudaMemcpyHostToDevice, s));
        BQB_CUDA(cudaMemcpyAsync(contrib.p, csr.contrib.data(), csr.contrib.size() * 4,
                                 cudaMemcpyHostToDevice, s));
    }
    // host vectors die here: make the copies complete before returning
    BQB_CUDA(cudaStreamSynchronize(s));
}

namespace {

__global__ void __launch_bounds__(256) opB_kernel(const CutRec* __restrict__ cuts, int m,
                                                  const double* __restrict__ Xbase, size_t ldx_mat,
                                                  const int* __restrict__ slot, int n,
                                                  double* __restrict__ Y, size_t ldy, int init_one)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (c >= m) return;
    const double* X = Xbase + (size_t)(slot ? slot[j] : j) * ldx_mat;
    double* y = Y + c + (size_t)(slot ? slot[j] : j) * ldy;
    *y = cut_apply(cuts[c], X, n, init_one ? 1.0 : *y);
}

__global__ void __launch_bounds__(256) opBt_kernel(const uint32_t* __restrict__ pair_uv,
                                                   const uint32_t* __restrict__ offsets,
                                                   const uint32_t* __restrict__ contrib, int npairs,
                                                   int m_tri, int m_tp, double* __restrict__ X, int n,
                                                   const double* __restrict__ t)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npairs) return;
    const unsigned uv = pair_uv[q];
    const unsigned u = uv & 0xffffu, v = uv >> 16;
    const size_t e1 = u + (size_t)v * n, e2 = v + (size_t)u * n;
    double x1 = X[e1], x2 = X[e2];
    pair_apply(contrib, offsets[q], offsets[q + 1], m_tri, m_tp, t, &x1, &x2);
    X[e1] = x1;
    X[e2] = x2;
}

}  // namespace

void opB_launch(const DevCuts& dc, const double* Xbase, size_t ldx_mat, const int* slot, int ncols,
                int n, double* Y, size_t ldy, bool init_one, cudaStream_t s)
{
    if (dc.m <= 0 || ncols <= 0) return;
    dim3 grid((dc.m + 255) / 256, ncols);
    opB_kernel<<<grid, 256, 0, s>>>(dc.rec.p, dc.m, Xbase, ldx_mat, slot, n, Y, ldy, init_one ? 1 : 0);
    BQB_COUNT_LAUNCH();
    check_launch("opB_kernel");
}

void opBt_launch(const DevCuts& dc, double* X, int n, const double* t, cudaStream_t s)
{
    if (dc.npairs <= 0) return;
    opBt_kernel<<<(dc.npairs + 255) / 256, 256, 0, s>>>(dc.pair_uv.p, dc.offsets.p, dc.contrib.p,
                                                        dc.npairs, dc.m_tri, dc.m_tri + dc.m_pent, X, n, t);
    BQB_COUNT_LAUNCH();
    check_launch("opBt_kernel");
}

}  // namespace bqb
