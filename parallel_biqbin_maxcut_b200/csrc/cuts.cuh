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
unsigned tri_negmask(int type);
unsigned pent_negmask(int type);
unsigned hept_negmask(int type);

CutRec pack_cut(int k, const int* p, unsigned negmask);

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
