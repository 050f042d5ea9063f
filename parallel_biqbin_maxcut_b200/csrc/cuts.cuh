// Cut operators B (gather) and B^T (symmetric scatter) over packed cut lists.
#pragma once
#include <vector>

#include "bqb_common.cuh"

namespace bqb {

// One cut = one 16-byte record (uint4), read with a single vector load:
//   x = p0 | p1 << 16, y = p2 | p3 << 16, z = p4 | p5 << 16,
//   w = p6 | k << 16 | negmask << 24
// k in {3, 5, 7} is the number of indices; bit a of negmask is set when the
// sign e_a is -1.  The cut is B_c(X) <= 1 with
//   B_c(X) = -scale_k * sum_{a<b} e_a e_b X[p_a + p_b * n],
// scale_3 = 1, scale_5 = 1/2, scale_7 = 1/3 (src/operators.c:51-132).
// Records are stored in dual-vector order [tri | pent | hept].
typedef uint4 CutRec;

// Sign masks per kind and type, from the sign vectors the reference encodes
// in its switch statements (src/operators.c:64-129) and H matrices
// (src/cutting_planes.c:239-244, 431-438).
__host__ __device__ inline unsigned tri_negmask(int type)
{
    // type 1: (1,1,1); 2: (1,1,-1); 3: (1,-1,1); 4: (-1,1,1)
    return type == 1 ? 0u : (type == 2 ? 4u : (type == 3 ? 2u : 1u));
}

__host__ __device__ inline unsigned pent_negmask(int type)
{
    // H1 = ee', e = 1; H2: e0 = -1; H3: e0 = e1 = -1
    return type == 1 ? 0u : (type == 2 ? 1u : 3u);
}

__host__ __device__ inline unsigned hept_negmask(int type)
{
    // H1: none; H2: e0; H3: e0, e1; H4: e0, e1, e2
    return type == 1 ? 0u : (type == 2 ? 1u : (type == 3 ? 3u : 7u));
}

__host__ __device__ inline CutRec pack_cut(int k, const int* p, unsigned negmask)
{
    unsigned q[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int a = 0; a < k; ++a) q[a] = (unsigned)p[a] & 0xffffu;
    CutRec r;
    r.x = q[0] | (q[1] << 16);
    r.y = q[2] | (q[3] << 16);
    r.z = q[4] | (q[5] << 16);
    r.w = q[6] | ((unsigned)k << 16) | ((negmask & 0x7fu) << 24);
    return r;
}

// One cut's entry of y0 - B(X) (op_B, src/operators.c:51-132): y0 - scale *
// (sum of -e_a e_b X[p_a + p_b n] over a < b in tuple order).
__host__ __device__ inline double cut_apply(const CutRec& r, const double* X, int n, double y0)
{
    const unsigned p[7] = {r.x & 0xffffu, r.x >> 16, r.y & 0xffffu, r.y >> 16,
                           r.z & 0xffffu, r.z >> 16, r.w & 0xffffu};
    const int k = (int)((r.w >> 16) & 0xffu);
    const unsigned neg = (r.w >> 24) & 0x7fu;
    double acc = 0.0;
    bool first = true;
    for (int a = 0; a < k; ++a) {
        for (int b = a + 1; b < k; ++b) {
            // coefficient inside the bracket is -e_a e_b
            const bool plus = ((neg >> a) ^ (neg >> b)) & 1u;
            const double x = X[p[a] + (size_t)p[b] * n];
            if (first) {
                acc = plus ? x : -x;
                first = false;
            } else {
                acc = plus ? acc + x : acc - x;
            }
        }
    }
    if (k == 3) return y0 - acc;
    if (k == 5) return y0 - 0.5 * acc;
    return y0 - (1.0 / 3.0) * acc;
}

// One pair's B^T update (op_Bt, src/operators.c:140-481): the pair's
// contributions (cut << 1 | negative) applied in cut order to x1 = X_uv and
// x2 = X_vu, with temp = t/2, t/4, t/6 for triangle / pentagonal /
// heptagonal cuts.
__host__ __device__ inline void pair_apply(const uint32_t* contrib, unsigned b, unsigned e, int m_tri, int m_tp,
                                           const double* t, double* x1, double* x2)
{
    double a1 = *x1, a2 = *x2;
    for (unsigned i = b; i < e; ++i) {
        const unsigned code = contrib[i];
        const int c = (int)(code >> 1);
        const double tc = t[c];
        const double temp = c < m_tri ? 0.5 * tc : (c < m_tp ? 0.25 * tc : (1.0 / 6.0) * tc);
        // X -= B^T(t): coefficient of X_uv in B is -scale e_u e_v, so the
        // entry moves by +e_u e_v * temp
        if (code & 1u) {
            a1 -= temp;
            a2 -= temp;
        } else {
            a1 += temp;
            a2 += temp;
        }
    }
    *x1 = a1;
    *x2 = a2;
}

// CSR over the index pairs touched by a cut list, for the deterministic
// gather form of B^T: every touched unordered pair {u < v} owns the list of
// (cut id << 1 | negative) contributions in cut order.
struct PairCSR {
    std::vector<uint32_t> pair_uv;    // u | v << 16
    std::vector<uint32_t> offsets;    // size npairs + 1
    std::vector<uint32_t> contrib;    // cut << 1 | neg
    void build(const std::vector<CutRec>& cuts);
};

// Device-resident copy of one cut list and its pair CSR.
struct DevCuts {
    int m = 0, m_tri = 0, m_pent = 0, m_hept = 0;
    int npairs = 0;
    DevBuf<CutRec> rec;
    DevBuf<uint32_t> pair_uv, offsets, contrib;
    void upload(const std::vector<CutRec>& cuts, int mt, int mp, int mh, cudaStream_t s);
};

// Y[c + s_j*ldy] = (init_one ? 1 : Y[c + s_j*ldy]) - B_c(X_j) for every cut
// c and every matrix j < ncols; X_j = Xbase + s_j * ldx_mat with
// s_j = slot[j] (slot may be null: s_j = j).  ld of every X_j is n.  The
// slot array lets the bundle address its physical matrix/column slots.
void opB_launch(const DevCuts& dc, const double* Xbase, size_t ldx_mat, const int* slot, int ncols,
                int n, double* Y, size_t ldy, bool init_one, cudaStream_t s);

// X[u + v n], X[v + u n] -= B^T(t) contributions, for every touched pair.
void opBt_launch(const DevCuts& dc, double* X, int n, const double* t, cudaStream_t s);

}  // namespace bqb
