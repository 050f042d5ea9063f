// Triangle-inequality separation on the GPU.
#pragma once
#include "bqb_common.cuh"

namespace bqb {

// One separated cut: type 1..4, indices i > j > k, value = B(X) - 1.
struct TriCand {
    double value;
    uint32_t code;   // type-1 << 30 | i << 20 | j << 10 | k
    uint32_t pad_;
};

__host__ __device__ inline uint32_t tri_code(int type, int i, int j, int k)
{
    return ((uint32_t)(type - 1) << 30) | ((uint32_t)i << 20) | ((uint32_t)j << 10) | (uint32_t)k;
}
__host__ __device__ inline void tri_decode(uint32_t c, int* type, int* i, int* j, int* k)
{
    *type = (int)(c >> 30) + 1;
    *i = (int)((c >> 20) & 1023u);
    *j = (int)((c >> 10) & 1023u);
    *k = (int)(c & 1023u);
}

// The four triangle values B(X) - 1 for a = X_ij, b = X_ik, c = X_jk
// (src/cutting_planes.c:24-36).  The reference is built with -ffast-math
// (reference Makefile:17), under which gcc evaluates each 4-term sum in a
// reassociated order; these are the orders that reproduce the reference
// build's values bit for bit (matched on every triple of several X), so
// thresholds, ties and the streaming top-K see exactly the reference's
// numbers.  Negation is exact, so x - y is written as x + (-y).
__host__ __device__ inline void tri_values(double a, double b, double c, double* v)
{
    v[0] = (-a - 1.0) + (-b - c);   // -X_ij - X_ik - X_jk - 1
    v[1] = (-a - 1.0) + (b + c);    // -X_ij + X_ik + X_jk - 1
    v[2] = (a - b) + (c - 1.0);     //  X_ij - X_ik + X_jk - 1
    v[3] = (a - c) + (b - 1.0);     //  X_ij + X_ik - X_jk - 1
}

struct TriSepState {
    DevBuf<double> XT;
    DevBuf<uint32_t> cnt;            // per (type, pair) counts, then offsets
    DevBuf<unsigned long long> misc; // [0] ordered max, [1] total count
    DevBuf<TriCand> cand;
    DevBuf<TriCand> list;            // separated list in slot order (<= T)
    HostBuf<unsigned long long> hmisc;
    HostBuf<TriCand> hlist;
};

// Separate on device X (n x n, column-major).  Fills st.list (device) and
// st.hlist (host, pinned) with *list_size entries in the reference's slot
// order and returns the maximum violation over all 4*C(n,3) cuts
// (src/cutting_planes.c:48-127).  Synchronises the stream.
double trisep_device(TriSepState& st, const double* dX, int n, int tri_ineq, double violated,
                     int* list_size, cudaStream_t s);

}  // namespace bqb
