// Device bodies of the proximal bundle method (src/bundle.c), shared by the
// bundle kernels (bundle.cu) and the fused node kernel (nodek.cu).
#pragma once
#include <math.h>

#include "bundle.cuh"

namespace bqb {

constexpr double BQB_BUNDLE_BIG = 1e9;   // BIG_NUMBER, src/biqbin.h:35
// Threads of the bundle CTAs (lambda_eta, step, F value): the fused node
// kernel runs the same bodies with its IPM_THREADS threads, and the block
// reductions' order depends on the thread count.
constexpr int LE_THREADS = 512;
constexpr int QP_SMEM_K = 90;   // k up to this keeps Q and the KKT factor in shared memory

__device__ __forceinline__ double Qat(const double* Q, int k, int a, int b)
{
    return a >= b ? Q[a + (size_t)b * k] : Q[b + (size_t)a * k];
}

// Doubles of the QP workspace's matrix region for bundle size k: the
// register form (k <= 32) uses a 32 x 32 broadcast buffer.
__host__ __device__ constexpr size_t qp_a_doubles(int k) { return k <= 32 ? 1024 : (size_t)k * k; }

// Step J of the Cholesky factorisation of the QP's matrix A = Q + Diag(z ./
// lambda) held in registers (lane p < KP holds row p in s[], columns <= p;
// rows and columns from k to KP - 1 are the identity's).  The same
// operations in the same order as the shared-memory form below: the pivot's
// reciprocal square root rj, the column scaled by it, then every entry
// (p, r), J < r <= p, less l_pJ l_rJ (a rounded product, then a rounded
// difference).  Column J goes to the warp through Lc (one store per lane,
// then broadcast reads).  Instantiated for every J so that s[] stays in
// registers.  After a non-positive pivot the steps go on with a unit pivot
// and pd is false.
template <int KP, int J>
__device__ __forceinline__ void qp_chol_step(double (&s)[KP], int p, bool& pd, double& rdiag, double* Lc)
{
    if constexpr (J < KP) {
        double d = __shfl_sync(0xffffffffu, s[J], J);
        if (!(d > 0.0)) {
            pd = false;
            d = 1.0;
        }
        const double rj = rsqrt(d);
        const double l = p == J ? __dmul_rn(d, rj) : __dmul_rn(s[J], rj);
        if (p == J) rdiag = rj;
        s[J] = l;
        if (p < KP) Lc[J * KP + p] = l;
        __syncwarp();
#pragma unroll
        for (int r = J + 1; r < KP; ++r)
            if (r <= p) s[r] = __dsub_rn(s[r], __dmul_rn(l, Lc[J * KP + r]));
        __syncwarp();
        qp_chol_step<KP, J + 1>(s, p, pd, rdiag, Lc);
    }
}

// Forward substitution step J for u and w together (lane p holds u_p, w_p
// and row p of the factor; R: the factor's diagonal reciprocals in shared
// memory): u_J *= 1/L_JJ, then u_p -= L_pJ u_J below.
template <int KP, int J>
__device__ __forceinline__ void qp_fwd_step(const double (&s)[KP], int p, const double* R, double& u, double& w)
{
    if constexpr (J < KP) {
        const double rj = R[J];
        const double uj = __dmul_rn(__shfl_sync(0xffffffffu, u, J), rj);
        const double wj = __dmul_rn(__shfl_sync(0xffffffffu, w, J), rj);
        if (p == J) {
            u = uj;
            w = wj;
        } else if (p > J) {
            u = __dsub_rn(u, __dmul_rn(s[J], uj));
            w = __dsub_rn(w, __dmul_rn(s[J], wj));
        }
        qp_fwd_step<KP, J + 1>(s, p, R, u, w);
    }
}

// Backward substitution step J (from KP - 1 down): u_J *= 1/L_JJ, then
// u_p -= L_Jp u_J above; Lr holds the factor by rows.
template <int KP, int J>
__device__ __forceinline__ void qp_bwd_step(const double* Lr, int p, const double* R, double& u, double& w)
{
    if constexpr (J >= 0) {
        const double rj = R[J];
        const double uj = __dmul_rn(__shfl_sync(0xffffffffu, u, J), rj);
        const double wj = __dmul_rn(__shfl_sync(0xffffffffu, w, J), rj);
        if (p == J) {
            u = uj;
            w = wj;
        } else if (p < J) {
            const double l = Lr[J * KP + p];
            u = __dsub_rn(u, __dmul_rn(l, uj));
            w = __dsub_rn(w, __dmul_rn(l, wj));
        }
        qp_bwd_step<KP, J - 1>(Lr, p, R, u, w);
    }
}

// warp_qp for k <= KP (8, 12 or 16): lane a < k keeps the QP's entry a of
// lambda, z, Q lambda, c, u, w and row a of A = Q + Diag(z ./ lambda) in
// registers; ws holds the factor's column broadcasts, then its rows (KP x KP
// doubles), then its diagonal reciprocals (KP).  The arithmetic is warp_qp's below, operation for operation
// (the same sums in the same order, the same warp reductions), so both
// forms return the same bits; this one has no shared-memory loop per row.
template <int KP>
__device__ __noinline__ bool warp_qp_reg(int k, const double* Q, const double* c, double* lam, double* ws)
{
    const int lane = threadIdx.x & 31;
    const bool own = lane < k;
    double la = 1.0 / k;
    if (own) lam[lane] = la;
    __syncwarp();
    double qla = 0.0, ca = 0.0, za = 0.0;
    if (own) {
        ca = c[lane];
        double acc = 0.0;
        for (int b = 0; b < k; ++b) acc += Qat(Q, k, lane, b) * lam[b];
        qla = acc;
        za = acc + ca;
    }
    double mintmp = own ? za : BQB_BUNDLE_BIG;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mintmp = fmin(mintmp, __shfl_xor_sync(0xffffffffu, mintmp, o));
    double y;
    if (mintmp > 1) {
        y = 0.0;
    } else {
        y = mintmp - 1.0;
        if (own) za = za - y;
    }
    // (each lane's partial starts at 0.0, as the loop form's does)
    double s1 = own ? 0.0 + za * la : 0.0, s2 = own ? 0.0 + la : 0.0;
    double s3 = own ? 0.0 + la * qla : 0.0, s4 = own ? 0.0 + la * ca : 0.0;
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    s3 = warp_sum(s3);
    s4 = warp_sum(s4);
    double mu = 0.5 * (s1 / k);
    double res_p = 1.0 - s2;
    double gap = (s4 + 0.5 * s3) - (y - 0.5 * s3);
    int cnt = 0;
    double* L = ws;             // KP x KP
    double* R = ws + KP * KP;   // KP
    while (fabs(gap) > 1e-5) {
        ++cnt;
        // A = Q + Diag(z ./ lambda) (lower, padded with the identity), r = c - y + Qlam
        // (an own lane's entries b <= lane are Q's lower triangle: Q[lane + b k])
        double a[KP];
        const double dg = own ? za / la : 0.0;
#pragma unroll
        for (int b = 0; b < KP; ++b) {
            double v = b == lane ? 1.0 : 0.0;
            if (own && b <= lane) {
                v = Q[lane + (size_t)b * k];
                if (b == lane) v += dg;
            }
            a[b] = v;
        }
        double u = own ? 1.0 : 0.0;
        double w = own ? c[lane] - y + qla : 0.0;
        bool pd = true;
        double rdiag = 1.0;
        qp_chol_step<KP, 0>(a, lane, pd, rdiag, L);
        if (!pd) return false;
        if (lane < KP) {
#pragma unroll
            for (int r = 0; r < KP; ++r) L[lane * KP + r] = r <= lane ? a[r] : 0.0;
            R[lane] = rdiag;
        }
        __syncwarp();
        qp_fwd_step<KP, 0>(a, lane, R, u, w);
        qp_bwd_step<KP, KP - 1>(L, lane, R, u, w);
        const double su = warp_sum(own ? 0.0 + u : 0.0), sw = warp_sum(own ? 0.0 + w : 0.0);
        const double dy = (res_p + sw) / su;
        double ap = -BQB_BUNDLE_BIG, ad = -BQB_BUNDLE_BIG;
        double dl = 0.0, dz = 0.0;
        if (own) {
            dl = u * dy - w;
            dz = 1.0 / la * (mu - la * za - za * dl);
            ap = -dl / la;
            ad = -dz / za;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ap = fmax(ap, __shfl_xor_sync(0xffffffffu, ap, o));
            ad = fmax(ad, __shfl_xor_sync(0xffffffffu, ad, o));
        }
        ap = (ap > 0) ? ((0.99 / ap < 1.0) ? 0.99 / ap : 1.0) : 1.0;
        ad = (ad > 0) ? ((0.99 / ad < 1.0) ? 0.99 / ad : 1.0) : 1.0;
        y += ad * dy;
        if (own) {
            la = fma(ap, dl, la);
            za = fma(ad, dz, za);
            lam[lane] = la;
        }
        __syncwarp();
        double t1 = 0.0, t2 = 0.0, t3 = 0.0, t4 = 0.0;
        if (own) {
            double acc = 0.0;
            for (int b = 0; b < k; ++b) acc += Qat(Q, k, lane, b) * lam[b];
            qla = acc;
            t1 = 0.0 + la;
            t2 = 0.0 + la * za;
            t3 = 0.0 + la * acc;
            t4 = 0.0 + la * ca;
        }
        t1 = warp_sum(t1);
        t2 = warp_sum(t2);
        t3 = warp_sum(t3);
        t4 = warp_sum(t4);
        __syncwarp();
        res_p = 1 - t1;
        mu = (t2 / k) * 0.4;
        if (ap + ad > 1.8) mu *= 0.2;
        gap = (t4 + 0.5 * t3) - (y - 0.5 * t3);
        if (cnt > 30) break;
    }
    return true;
}

// One warp.  Q: k x k (lower triangle read), c: k, lam: k (out).
// ws: A[k*k], then six k-vectors (Q lambda, z, dlambda, u, w, and the
// reciprocals of the factor's diagonal).  Returns false on a non-PD A.
// Bundles of up to 16 go to the register form above (same results).
__device__ inline bool warp_qp(int k, const double* Q, const double* c, double* lam, double* ws)
{
    if (k <= 8) return warp_qp_reg<8>(k, Q, c, lam, ws);
    if (k <= 12) return warp_qp_reg<12>(k, Q, c, lam, ws);
    if (k <= 16) return warp_qp_reg<16>(k, Q, c, lam, ws);
    const int lane = threadIdx.x & 31;
    double* A = ws;
    double* Qlam = A + (size_t)k * k;
    double* z = Qlam + k;
    double* dlam = z + k;
    double* u = dlam + k;
    double* w = u + k;
    double* dinv = w + k;   // reciprocals of the factor's diagonal

    for (int b = lane; b < k; b += 32) lam[b] = 1.0 / k;
    __syncwarp();
    double part_min = BQB_BUNDLE_BIG;
    for (int a = lane; a < k; a += 32) {
        double acc = 0.0;
        for (int b = 0; b < k; ++b) acc += Qat(Q, k, a, b) * lam[b];
        Qlam[a] = acc;
        const double tv = acc + c[a];
        z[a] = tv;
        part_min = fmin(part_min, tv);
    }
    double mintmp = part_min;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mintmp = fmin(mintmp, __shfl_xor_sync(0xffffffffu, mintmp, o));
    double y;
    __syncwarp();
    if (mintmp > 1) {
        y = 0.0;
    } else {
        y = mintmp - 1.0;
        for (int a = lane; a < k; a += 32) z[a] = z[a] - y;
    }
    __syncwarp();
    double s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
    for (int a = lane; a < k; a += 32) {
        s1 += z[a] * lam[a];
        s2 += lam[a];
        s3 += lam[a] * Qlam[a];
        s4 += lam[a] * c[a];
    }
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    s3 = warp_sum(s3);
    s4 = warp_sum(s4);
    double mu = 0.5 * (s1 / k);
    double res_p = 1.0 - s2;
    double gap = (s4 + 0.5 * s3) - (y - 0.5 * s3);
    int cnt = 0;
    while (fabs(gap) > 1e-5) {
        ++cnt;
        // A = Q + Diag(z ./ lambda) (lower), r = c - y + Qlam
        for (int a = lane; a < k; a += 32) {
            for (int b = 0; b <= a; ++b) A[a + (size_t)b * k] = Qat(Q, k, a, b);
            A[a + (size_t)a * k] += z[a] / lam[a];
            u[a] = 1.0;
            w[a] = c[a] - y + Qlam[a];
        }
        __syncwarp();
        // Cholesky of A; one reciprocal square root per pivot, the column and
        // the substitutions below multiply by it
        for (int j = 0; j < k; ++j) {
            const double d = A[j + (size_t)j * k];
            if (!(d > 0.0)) return false;
            const double rj = rsqrt(d);
            __syncwarp();
            for (int i = j + 1 + lane; i < k; i += 32) A[i + (size_t)j * k] *= rj;
            if (lane == 0) {
                A[j + (size_t)j * k] = d * rj;
                dinv[j] = rj;
            }
            __syncwarp();
            for (int i = j + 1 + lane; i < k; i += 32) {
                const double lij = A[i + (size_t)j * k];
                for (int cc = j + 1; cc <= i; ++cc) A[i + (size_t)cc * k] -= lij * A[cc + (size_t)j * k];
            }
            __syncwarp();
        }
        // forward and backward substitution for u and w together
        for (int j = 0; j < k; ++j) {
            const double rj = dinv[j];
            const double uj = u[j] * rj, wj = w[j] * rj;
            __syncwarp();
            if (lane == 0) {
                u[j] = uj;
                w[j] = wj;
            }
            for (int i = j + 1 + lane; i < k; i += 32) {
                const double l = A[i + (size_t)j * k];
                u[i] -= l * uj;
                w[i] -= l * wj;
            }
            __syncwarp();
        }
        for (int j = k - 1; j >= 0; --j) {
            const double rj = dinv[j];
            const double uj = u[j] * rj, wj = w[j] * rj;
            __syncwarp();
            if (lane == 0) {
                u[j] = uj;
                w[j] = wj;
            }
            for (int i = lane; i < j; i += 32) {
                const double l = A[j + (size_t)i * k];
                u[i] -= l * uj;
                w[i] -= l * wj;
            }
            __syncwarp();
        }
        double su = 0.0, sw = 0.0;
        for (int a = lane; a < k; a += 32) {
            su += u[a];
            sw += w[a];
        }
        su = warp_sum(su);
        sw = warp_sum(sw);
        const double dy = (res_p + sw) / su;
        double ap = -BQB_BUNDLE_BIG, ad = -BQB_BUNDLE_BIG;
        for (int a = lane; a < k; a += 32) {
            const double dl = u[a] * dy - w[a];
            dlam[a] = dl;
            const double dz = 1.0 / lam[a] * (mu - lam[a] * z[a] - z[a] * dl);
            u[a] = dz;   // u now holds dz
            ap = fmax(ap, -dl / lam[a]);
            ad = fmax(ad, -dz / z[a]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ap = fmax(ap, __shfl_xor_sync(0xffffffffu, ap, o));
            ad = fmax(ad, __shfl_xor_sync(0xffffffffu, ad, o));
        }
        ap = (ap > 0) ? ((0.99 / ap < 1.0) ? 0.99 / ap : 1.0) : 1.0;
        ad = (ad > 0) ? ((0.99 / ad < 1.0) ? 0.99 / ad : 1.0) : 1.0;
        y += ad * dy;
        __syncwarp();
        for (int a = lane; a < k; a += 32) {
            lam[a] = fma(ap, dlam[a], lam[a]);
            z[a] = fma(ad, u[a], z[a]);
        }
        __syncwarp();
        double t1 = 0.0, t2 = 0.0, t3 = 0.0, t4 = 0.0;
        for (int a = lane; a < k; a += 32) {
            double acc = 0.0;
            for (int b = 0; b < k; ++b) acc += Qat(Q, k, a, b) * lam[b];
            Qlam[a] = acc;
            t1 += lam[a];
            t2 += lam[a] * z[a];
            t3 += lam[a] * acc;
            t4 += lam[a] * c[a];
        }
        t1 = warp_sum(t1);
        t2 = warp_sum(t2);
        t3 = warp_sum(t3);
        t4 = warp_sum(t4);
        __syncwarp();
        res_p = 1 - t1;
        mu = (t2 / k) * 0.4;
        if (ap + ad > 1.8) mu *= 0.2;
        gap = (t4 + 0.5 * t3) - (y - 0.5 * t3);
        if (cnt > 30) break;
    }
    return true;
}

__device__ __forceinline__ const double* gcol(const double* G, int ldg, const int* slot, int b)
{
    return G + (size_t)(slot ? slot[b] : b) * ldg;
}

struct LeArgs {
    const double* G;
    int ldg;
    const int* slot;
    int m;
    const double* zeta_in;
    const double* Fv;
    const double* gam;
    double* lam;
    double* eta;
    double* dgam;
    double* gtest;
    double* dstate;
    int* istate;
    double* qp_ws_global;
    int k_fixed;   // >= 0: use this k instead of istate[BI_K]
    unsigned long long* prof = nullptr;   // (profiling) calls, rounds, sum of k, QP cycles, cycles, sum of m
};

// sm: dynamic shared memory of le_smem_bytes(min(k, QP_SMEM_K)) bytes (at
// least 3k doubles when k > QP_SMEM_K).
__device__ inline void lambda_eta_body(const LeArgs& a, double* sm)
{
    __shared__ double red[64];
    __shared__ int flag;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int k = a.k_fixed >= 0 ? a.k_fixed : a.istate[BI_K];
    const int m = a.m;
    double t = a.dstate[BD_T];
    const bool qp_in_smem = k <= QP_SMEM_K;
    double* zeta = sm;
    double* c = zeta + k;
    double* lam = c + k;
    double* Q = qp_in_smem ? lam + k : a.qp_ws_global;
    double* qpws = qp_in_smem ? Q + (size_t)k * k : a.qp_ws_global + (size_t)k * k;

    // zeta
    for (int b = warp; b < k; b += nw) {
        if (a.zeta_in) {
            if (lane == 0) zeta[b] = a.zeta_in[b];
            continue;
        }
        const double* Gb = gcol(a.G, a.ldg, a.slot, b);
        double acc = 0.0;
        for (int i = lane; i < m; i += 32) acc = fma(Gb[i], a.gam[i], acc);
        acc = warp_sum(acc);
        if (lane == 0) zeta[b] = -a.Fv[b] - acc;
    }
    // Q = t G'G (lower)
    for (int p = warp; p < k * (k + 1) / 2; p += nw) {
        int r = (int)((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
        while (r * (r + 1) / 2 > p) --r;
        while ((r + 1) * (r + 2) / 2 <= p) ++r;
        const int col = p - r * (r + 1) / 2;
        const double* Gr = gcol(a.G, a.ldg, a.slot, r);
        const double* Gc = gcol(a.G, a.ldg, a.slot, col);
        double acc = 0.0;
        for (int i = lane; i < m; i += 32) acc = fma(Gr[i], Gc[i], acc);
        acc = warp_sum(acc);
        if (lane == 0) Q[r + (size_t)col * k] = t * acc;
    }
    for (int i = tid; i < m; i += blockDim.x) a.eta[i] = 0.0;
    if (tid == 0) flag = 0;
    __syncthreads();

    double dir_prev = 0.0;
    int cnt = 0;
    const long long c_start = a.prof ? clock64() : 0;
    long long c_qp = 0;
    while (true) {
        ++cnt;
        for (int b = warp; b < k; b += nw) {
            const double* Gb = gcol(a.G, a.ldg, a.slot, b);
            double acc = 0.0;
            for (int i = lane; i < m; i += 32) acc = fma(Gb[i], a.eta[i], acc);
            acc = warp_sum(acc);
            if (lane == 0) c[b] = zeta[b] + (-t) * acc;
        }
        __syncthreads();
        const long long c0 = a.prof ? clock64() : 0;
        if (warp == 0) {
            const bool ok = warp_qp(k, Q, c, lam, qpws);
            if (!ok && lane == 0) flag = 1;
        }
        __syncthreads();
        if (a.prof) c_qp += clock64() - c0;
        if (flag) break;
        double acc2 = 0.0;
        for (int i = tid; i < m; i += blockDim.x) {
            double tmp = 0.0;
            for (int b = 0; b < k; ++b) tmp = fma(gcol(a.G, a.ldg, a.slot, b)[i], lam[b], tmp);
            double e = -a.gam[i] / t + tmp;
            e = (e > 0) ? e : 0;
            a.eta[i] = e;
            const double dg = t * (e - tmp);
            a.dgam[i] = dg;
            acc2 += dg * dg;
        }
        const double dir_curr = sqrt(block_sum(acc2, red));
        bool done = fabs(dir_curr - dir_prev) / (1.0 + dir_curr) < 1e-5;
        if (cnt >= 50) {
            done = true;
            t *= 0.95;
        }
        dir_prev = dir_curr;
        if (done) break;
    }
    if (flag) {
        if (tid == 0) atomicOr(&a.istate[BI_ERR], 2);
        return;
    }
    if (a.prof && tid == 0) {
        atomicAdd(a.prof + 0, 1ull);
        atomicAdd(a.prof + 1, (unsigned long long)cnt);
        atomicAdd(a.prof + 2, (unsigned long long)k);
        atomicAdd(a.prof + 3, (unsigned long long)c_qp);
        atomicAdd(a.prof + 4, (unsigned long long)(clock64() - c_start));
        atomicAdd(a.prof + 5, (unsigned long long)m);
    }
    for (int b = tid; b < k; b += blockDim.x) a.lam[b] = lam[b];
    if (a.gtest)
        for (int i = tid; i < m; i += blockDim.x) a.gtest[i] = a.gam[i] + a.dgam[i];
    if (tid == 0) a.dstate[BD_T] = t;
}

__device__ inline void solve_lambda_body(int k, const double* Q, const double* c, double* lam, int* err,
                                         double* ws_global, double* sm)
{
    const bool in_smem = k <= QP_SMEM_K;
    double* cl = sm;
    double* ll = cl + k;
    double* ws = in_smem ? ll + k : ws_global;
    for (int b = threadIdx.x; b < k; b += 32) cl[b] = c[b];
    __syncwarp();
    const bool ok = warp_qp(k, Q, cl, ll, ws);
    __syncwarp();
    for (int b = threadIdx.x; b < k; b += 32) lam[b] = ll[b];
    if (threadIdx.x == 0) *err = ok ? 0 : 1;
}

struct StepArgs {
    const double* G;
    int ldg;
    int m;
    int n;
    int cap;
    const double* L;
    const double* Xb;
    const double* phi_out;
    double* Fv;
    int* slot;
    int* slot_old;
    const double* lam;
    double* gam;
    const double* gtest;
    double* dstate;
    int* istate;
};

__device__ inline void bundle_step_body(const StepArgs& a)
{
    __shared__ double red[64];
    __shared__ int s_serious;
    __shared__ unsigned char used[BQB_MAX_BUNDLE + 8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int k = a.istate[BI_K];
    const int next = a.istate[BI_NEXT];
    const int n = a.n;
    const double f = a.dstate[BD_F];
    double t = a.dstate[BD_T];
    const double phi = a.phi_out[0];
    if ((int)a.phi_out[2] != 0 && tid == 0) atomicOr(&a.istate[BI_ERR], 4);

    // f_test = phi + sum(gamma_test)
    double sg = 0.0;
    for (int i = tid; i < a.m; i += blockDim.x) sg += a.gtest[i];
    const double ftest = phi + block_sum(sg, red);
    // del = f - (F + G'gamma_test)'lambda
    __syncthreads();
    double dl = 0.0;
    for (int b = warp; b < k; b += nw) {
        const double* Gb = a.G + (size_t)a.slot[b] * a.ldg;
        double acc = 0.0;
        for (int i = lane; i < a.m; i += 32) acc = fma(Gb[i], a.gtest[i], acc);
        acc = warp_sum(acc);
        if (lane == 0) dl += (a.Fv[b] + acc) * a.lam[b];
    }
    const double del = f - block_sum(dl, red);
    // F of the new element: <L, X_test> over the upper triangle, 2x off-diagonal
    const double* Xt = a.Xb + (size_t)next * n * n;
    double fv = 0.0;
    for (int i = warp; i < n; i += nw) {
        for (int j = i + lane; j < n; j += 32) {
            const size_t e = j + (size_t)i * n;
            fv += (i == j) ? a.L[e] * Xt[e] : 2 * a.L[e] * Xt[e];
        }
    }
    const double Fnew = block_sum(fv, red);

    if (tid == 0) {
        double lmax = -BQB_BUNDLE_BIG;
        for (int b = 0; b < k; ++b) lmax = (a.lam[b] > lmax) ? a.lam[b] : lmax;
        const bool serious = (f - ftest > 0.05 * del);
        s_serious = serious ? 1 : 0;
        for (int b = 0; b < k; ++b) a.slot_old[b] = a.slot[b];
        int kept = 0;
        const int scan = serious ? k : k - 1;
        for (int b = 0; b < scan; ++b) {
            if (a.lam[b] < 0.01 * lmax) continue;
            a.slot[kept] = a.slot_old[b];
            a.Fv[kept] = a.Fv[b];
            ++kept;
        }
        int bundle;
        if (serious) {
            bundle = kept;
            if (bundle == BQB_MAX_BUNDLE) a.istate[BI_ERR] |= 1;
            a.slot[bundle] = next;
            a.Fv[bundle] = Fnew;
            ++bundle;
            a.dstate[BD_F] = ftest;
            t *= 1.01;
        } else {
            const double Flast = a.Fv[k - 1];
            const int slast = a.slot_old[k - 1];
            bundle = kept + 1;   // PP->bundle -= subtracted
            if (bundle == BQB_MAX_BUNDLE) a.istate[BI_ERR] |= 1;
            a.slot[bundle] = slast;
            a.Fv[bundle] = Flast;
            a.slot[bundle - 1] = next;
            a.Fv[bundle - 1] = Fnew;
            ++bundle;
            t /= 1.01;
        }
        for (int q = 0; q < a.cap; ++q) used[q] = 0;
        for (int b = 0; b < bundle; ++b) used[a.slot[b]] = 1;
        int nf = -1;
        for (int q = 0; q < a.cap; ++q)
            if (!used[q]) {
                nf = q;
                break;
            }
        if (nf < 0) {
            a.istate[BI_ERR] |= 8;
            nf = next;
        }
        a.istate[BI_KOLD] = k;
        a.istate[BI_K] = bundle;
        a.istate[BI_SERIOUS] = serious ? 1 : 0;
        a.istate[BI_LAST] = next;
        a.istate[BI_NEXT] = nf;
        a.dstate[BD_T] = t;
        a.dstate[BD_FTEST] = ftest;
        a.dstate[BD_DEL] = del;
    }
    __syncthreads();
    if (s_serious)
        for (int i = tid; i < a.m; i += blockDim.x) a.gam[i] = a.gtest[i];
}

// Entries start, start + stride, ... of X (every entry is one fixed-order
// sum, so the result does not depend on how the entries are split).
__device__ inline void bundle_xcomb_body(const double* __restrict__ Xb, const int* __restrict__ slot_old,
                                         const double* __restrict__ lam, const int* __restrict__ istate,
                                         double* __restrict__ X, size_t nn, size_t start, size_t stride)
{
    if (!istate[BI_SERIOUS]) return;
    const int k = istate[BI_KOLD];
    for (size_t e = start; e < nn; e += stride) {
        double acc = 0.0;
        for (int b = 0; b < k; ++b) acc = fma(Xb[(size_t)slot_old[b] * nn + e], lam[b], acc);
        X[e] = acc;
    }
}

__device__ inline void bundle_fval_body(const double* __restrict__ L, const double* __restrict__ Xb, int n,
                                        const int* __restrict__ slot_ptr, const int* __restrict__ pos_ptr,
                                        double* __restrict__ Fv)
{
    __shared__ double red[64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double* Xt = Xb + (size_t)(*slot_ptr) * n * n;
    double fv = 0.0;
    for (int i = warp; i < n; i += nw)
        for (int j = i + lane; j < n; j += 32) {
            const size_t e = j + (size_t)i * n;
            fv += (i == j) ? L[e] * Xt[e] : 2 * L[e] * Xt[e];
        }
    const double s = block_sum(fv, red);
    if (threadIdx.x == 0) Fv[*pos_ptr] = s;
}

// Append the element evaluated into slot NEXT at bundle position K
// (src/bounding.c:291-318: overflow test, then ++bundle), pick the next
// free slot.
__device__ inline void bundle_append_body(int* __restrict__ slot, int* __restrict__ istate, int cap)
{
    __shared__ unsigned char used[BQB_MAX_BUNDLE + 8];
    if (threadIdx.x != 0) return;
    const int k = istate[BI_K];
    const int next = istate[BI_NEXT];
    if (k == BQB_MAX_BUNDLE) istate[BI_ERR] |= 1;
    slot[k] = next;
    istate[BI_LAST] = next;
    istate[BI_K] = k + 1;
    for (int q = 0; q < cap; ++q) used[q] = 0;
    for (int b = 0; b <= k; ++b) used[slot[b]] = 1;
    int nf = -1;
    for (int q = 0; q < cap; ++q)
        if (!used[q]) {
            nf = q;
            break;
        }
    if (nf < 0) {
        istate[BI_ERR] |= 8;
        nf = next;
    }
    istate[BI_NEXT] = nf;
}

__host__ __device__ inline size_t le_smem_bytes(int k)
{
    const size_t base = 3 * (size_t)k;
    if (k <= QP_SMEM_K) return (base + (size_t)k * k + qp_a_doubles(k) + 6 * (size_t)k) * sizeof(double);
    return base * sizeof(double);
}


}  // namespace bqb
