// Device bodies of the learned warm start (warm.h), shared by its kernels
// (warm.cu) and the fused node kernel (nodek.cu) so both compute the same
// features and the same proposal.
#pragma once
#include <cuda_bf16.h>
#include <math.h>

#include "warm.h"

namespace bqb {

__device__ __forceinline__ float warm_softplus(float z) { return z > 20.f ? z : log1pf(expf(z)); }

// Features of the triangle cut (type, i, j, k), whose inequality is
// s_ij X_ij + s_ik X_ik + s_jk X_jk <= 1 with the type's signs
// (src/cutting_planes.c:20-39): its violation v, v relative to the largest
// violation viol3, viol3, the three signed X entries (sorted), the signed
// objective entries s L / scale (sorted), n / 128, log(1 + m) / 10,
// log(1 + gap / scale), and from the parent node: the multiplier the same
// cut ended with in the parent's final list / scale and 1 (pg >= 0), or 0
// and 0 when the parent did not hold the cut (pg < 0; also every cut of a
// node bounded without its parent's list).
__device__ inline void warm_cut_features(int type, int i, int j, int k, double v, const double* X,
                                         const double* L, int n, int m, double viol3, double gap, double sc,
                                         double pg, float* f)
{
    const double sij = (type == 3 || type == 4) ? 1.0 : -1.0;
    const double sik = (type == 2 || type == 4) ? 1.0 : -1.0;
    const double sjk = (type == 2 || type == 3) ? 1.0 : -1.0;
    const size_t eij = i + (size_t)j * n, eik = i + (size_t)k * n, ejk = j + (size_t)k * n;
    double x0 = sij * X[eij], x1 = sik * X[eik], x2 = sjk * X[ejk];
    double l0 = sij * L[eij] / sc, l1 = sik * L[eik] / sc, l2 = sjk * L[ejk] / sc;
    auto sort3 = [](double& a, double& b, double& d) {
        double t;
        if (a > b) t = a, a = b, b = t;
        if (b > d) t = b, b = d, d = t;
        if (a > b) t = a, a = b, b = t;
    };
    sort3(x0, x1, x2);
    sort3(l0, l1, l2);
    f[0] = (float)v;
    f[1] = (float)(viol3 > 1e-12 ? v / viol3 : 0.0);
    f[2] = (float)viol3;
    f[3] = (float)x0;
    f[4] = (float)x1;
    f[5] = (float)x2;
    f[6] = (float)l0;
    f[7] = (float)l1;
    f[8] = (float)l2;
    f[9] = (float)(n / 128.0);
    f[10] = (float)(log1p((double)m) / 10.0);
    f[11] = (float)log1p(fmax(gap, 0.0) / sc);
    f[12] = pg >= 0.0 ? (float)(pg / sc) : 0.f;
    f[13] = pg >= 0.0 ? 1.f : 0.f;
}

// The network on one feature row, BF16 weights, FP32 arithmetic; returns
// softplus of the output (the multiplier in units of the objective scale).
__device__ inline float warm_mlp_bf16(const float* xf, const __nv_bfloat16* __restrict__ P)
{
    float h1[WARM_H];
#pragma unroll
    for (int h = 0; h < WARM_H; ++h) {
        float a = __bfloat162float(P[WARM_OFF_B1 + h]);
#pragma unroll
        for (int i = 0; i < WARM_F; ++i) a = fmaf(xf[i], __bfloat162float(P[WARM_OFF_W1 + i * WARM_H + h]), a);
        h1[h] = fmaxf(a, 0.f);
    }
    float z = __bfloat162float(P[WARM_OFF_B3]);
    for (int h2 = 0; h2 < WARM_H; ++h2) {
        float a = __bfloat162float(P[WARM_OFF_B2 + h2]);
#pragma unroll
        for (int h = 0; h < WARM_H; ++h) a = fmaf(h1[h], __bfloat162float(P[WARM_OFF_W2 + h * WARM_H + h2]), a);
        z = fmaf(fmaxf(a, 0.f), __bfloat162float(P[WARM_OFF_W3 + h2]), z);
    }
    return warm_softplus(z);
}

}  // namespace bqb
