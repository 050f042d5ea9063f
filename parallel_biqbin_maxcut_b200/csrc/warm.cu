// Learned warm start of the bundle multipliers: feature, inference and
// training kernels, the recorder of training pairs, and the C entry points.
// The method is described in warm.h.
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <random>
#include <tuple>
#include <vector>

#include "internal.h"
#include "warm.h"
#include "warm_body.cuh"

namespace bqb {

namespace {

constexpr int WT = 128;   // threads per block of the warm-start kernels

__device__ __forceinline__ float warm_sigmoid(float z) { return 1.f / (1.f + expf(-z)); }

// Scale of the node's objective: the mean |L_ij| over i != j (1 when
// n < 2 or L vanishes).  One block.
__global__ void warm_scale_kernel(const double* __restrict__ L, int n, double* __restrict__ scale)
{
    __shared__ double red[WT];
    double a = 0.0;
    const size_t nn = (size_t)n * n;
    for (size_t e = threadIdx.x; e < nn; e += blockDim.x)
        if (e % n != e / n) a += fabs(L[e]);
    red[threadIdx.x] = a;
    __syncthreads();
    for (int o = WT / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double v = n > 1 ? red[0] / ((double)n * (n - 1)) : 0.0;
        *scale = v > 0.0 ? v : 1.0;
    }
}

// Features of each cut (warm_cut_features), one thread per cut.
__global__ void warm_feat_kernel(const int4* __restrict__ cut, const double* __restrict__ val, int m,
                                 const double* __restrict__ X, const double* __restrict__ L, int n, double viol3,
                                 double gap, const double* __restrict__ scale, const double* __restrict__ pgam,
                                 float* __restrict__ F)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    const int4 q = cut[c];
    double v = val[c];
    if (isnan(v)) {   // a cut the separation did not evaluate: its violation at X (src/cutting_planes.c:20-39)
        const double xij = X[q.y + (size_t)q.z * n], xik = X[q.y + (size_t)q.w * n], xjk = X[q.z + (size_t)q.w * n];
        v = q.x == 1 ? -xij - xik - xjk - 1.0
            : q.x == 2 ? -xij + xik + xjk - 1.0
            : q.x == 3 ? xij - xik + xjk - 1.0
                       : xij + xik - xjk - 1.0;
    }
    warm_cut_features(q.x, q.y, q.z, q.w, v, X, L, n, m, viol3, gap, *scale, pgam ? pgam[c] : -1.0,
                      F + (size_t)c * WARM_F);
}

// Inference with BF16 weights, FP32 arithmetic; one thread per cut.  The
// network predicts the multiplier in units of the objective's scale.
__global__ void warm_infer_kernel(const float* __restrict__ F, int m, const __nv_bfloat16* __restrict__ P,
                                  const double* __restrict__ scale, double* __restrict__ gam)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    float xf[WARM_F];
#pragma unroll
    for (int i = 0; i < WARM_F; ++i) xf[i] = F[(size_t)c * WARM_F + i];
    gam[c] = (scale ? *scale : 1.0) * (double)warm_mlp_bf16(xf, P);
}

__global__ void warm_to_bf16_kernel(const float* __restrict__ P, __nv_bfloat16* __restrict__ Q, int count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) Q[i] = __float2bfloat16_rn(P[i]);
}

// ---- training (FP32) --------------------------------------------------
// Loss: mean over the batch of (softplus(z) - y)^2.

// Forward for sample b = dataset row idx[b]: hidden activations (after
// ReLU) into H1, H2; dz[b] = d loss / d z; lossb[b] = squared error.
__global__ void warm_fwd_kernel(const float* __restrict__ Xd, const float* __restrict__ Yd, const int* __restrict__ idx,
                                int B, const float* __restrict__ P, float* __restrict__ H1, float* __restrict__ H2,
                                float* __restrict__ dz, float* __restrict__ lossb)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const int r = idx ? idx[b] : b;
    const float* x = Xd + (size_t)r * WARM_F;
    float h1[WARM_H];
#pragma unroll
    for (int h = 0; h < WARM_H; ++h) {
        float a = P[WARM_OFF_B1 + h];
#pragma unroll
        for (int i = 0; i < WARM_F; ++i) a = fmaf(x[i], P[WARM_OFF_W1 + i * WARM_H + h], a);
        h1[h] = fmaxf(a, 0.f);
        H1[(size_t)b * WARM_H + h] = h1[h];
    }
    float z = P[WARM_OFF_B3];
    for (int h2 = 0; h2 < WARM_H; ++h2) {
        float a = P[WARM_OFF_B2 + h2];
#pragma unroll
        for (int h = 0; h < WARM_H; ++h) a = fmaf(h1[h], P[WARM_OFF_W2 + h * WARM_H + h2], a);
        a = fmaxf(a, 0.f);
        H2[(size_t)b * WARM_H + h2] = a;
        z = fmaf(a, P[WARM_OFF_W3 + h2], z);
    }
    const float e = warm_softplus(z) - Yd[r];
    dz[b] = 2.f * e / (float)B * warm_sigmoid(z);
    lossb[b] = e * e;
}

// Back through the hidden layers, one thread per (sample, unit):
// dH2 = dz w3 (H2 > 0); dH1 = (W2 dH2) (H1 > 0).
__global__ void warm_bwd_hidden_kernel(int B, const float* __restrict__ P, const float* __restrict__ H1,
                                       const float* __restrict__ H2, const float* __restrict__ dz,
                                       float* __restrict__ dH1, float* __restrict__ dH2)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= B * WARM_H) return;
    const int b = e / WARM_H, h = e % WARM_H;
    const float g = dz[b];
    const float* h2 = H2 + (size_t)b * WARM_H;
    dH2[e] = h2[h] > 0.f ? g * P[WARM_OFF_W3 + h] : 0.f;
    float a = 0.f;
    for (int k = 0; k < WARM_H; ++k)
        if (h2[k] > 0.f) a = fmaf(g * P[WARM_OFF_W3 + k], P[WARM_OFF_W2 + h * WARM_H + k], a);
    dH1[e] = H1[e] > 0.f ? a : 0.f;
}

// Gradient of one parameter, summed over the batch in sample order (one
// thread per parameter: deterministic).
__global__ void warm_param_grad_kernel(const float* __restrict__ Xd, const int* __restrict__ idx, int B,
                                       const float* __restrict__ H1, const float* __restrict__ H2,
                                       const float* __restrict__ dz, const float* __restrict__ dH1,
                                       const float* __restrict__ dH2, float* __restrict__ grad)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= WARM_NPARAM) return;
    float s = 0.f;
    if (p < WARM_OFF_B1) {
        const int i = p / WARM_H, h = p % WARM_H;
        for (int b = 0; b < B; ++b) s = fmaf(Xd[(size_t)(idx ? idx[b] : b) * WARM_F + i], dH1[(size_t)b * WARM_H + h], s);
    } else if (p < WARM_OFF_W2) {
        const int h = p - WARM_OFF_B1;
        for (int b = 0; b < B; ++b) s += dH1[(size_t)b * WARM_H + h];
    } else if (p < WARM_OFF_B2) {
        const int q = p - WARM_OFF_W2, h = q / WARM_H, k = q % WARM_H;
        for (int b = 0; b < B; ++b) s = fmaf(H1[(size_t)b * WARM_H + h], dH2[(size_t)b * WARM_H + k], s);
    } else if (p < WARM_OFF_W3) {
        const int k = p - WARM_OFF_B2;
        for (int b = 0; b < B; ++b) s += dH2[(size_t)b * WARM_H + k];
    } else if (p < WARM_OFF_B3) {
        const int h = p - WARM_OFF_W3;
        for (int b = 0; b < B; ++b) s = fmaf(dz[b], H2[(size_t)b * WARM_H + h], s);
    } else {
        for (int b = 0; b < B; ++b) s += dz[b];
    }
    grad[p] = s;
}

// Adam (Kingma and Ba, 2015), bias-corrected step sizes from the host.
__global__ void warm_adam_kernel(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m1,
                                 float* __restrict__ m2, float lr_t, float b1, float b2, float eps_t)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= WARM_NPARAM) return;
    const float gp = g[p];
    const float a = b1 * m1[p] + (1.f - b1) * gp;
    const float v = b2 * m2[p] + (1.f - b2) * gp * gp;
    m1[p] = a;
    m2[p] = v;
    P[p] -= lr_t * a / (sqrtf(v) + eps_t);
}

}  // namespace

// ---- host side ---------------------------------------------------------

namespace {

struct WarmGlobal {
    std::mutex mu;                      // model load, dataset, training buffers
    DevBuf<__nv_bfloat16> pb;           // inference weights
    bool loaded = false;
    std::atomic<bool> enabled{false};
    std::atomic<bool> recording{false};
    std::vector<float> feats, targets;  // recorded training pairs
    std::atomic<long long> kept{0}, rejected{0};
    DevBuf<unsigned long long> dstats;  // the fused kernel's {kept, rejected}
    // training buffers
    DevBuf<float> X, Y, P, G, M1, M2, H1, H2, dz, dH1, dH2, lossb, pf;
    DevBuf<int> idx;
};

WarmGlobal& wg()
{
    static WarmGlobal g;
    return g;
}

unsigned blocks(long long count) { return (unsigned)((count + WT - 1) / WT); }

// Forward and backward over `B` samples (rows idx[0..B), or 0..B when idx
// is null) of the dataset in g.X / g.Y at parameters g.P; gradient into g.G.
void train_pass(WarmGlobal& g, const int* idx, int B, cudaStream_t s)
{
    warm_fwd_kernel<<<blocks(B), WT, 0, s>>>(g.X.p, g.Y.p, idx, B, g.P.p, g.H1.p, g.H2.p, g.dz.p, g.lossb.p);
    BQB_COUNT_LAUNCH();
    warm_bwd_hidden_kernel<<<blocks((long long)B * WARM_H), WT, 0, s>>>(B, g.P.p, g.H1.p, g.H2.p, g.dz.p, g.dH1.p,
                                                                        g.dH2.p);
    BQB_COUNT_LAUNCH();
    warm_param_grad_kernel<<<blocks(WARM_NPARAM), WT, 0, s>>>(g.X.p, idx, B, g.H1.p, g.H2.p, g.dz.p, g.dH1.p, g.dH2.p,
                                                              g.G.p);
    BQB_COUNT_LAUNCH();
    check_launch("warm training pass");
}

void upload_dataset(WarmGlobal& g, const float* feats, const float* targets, int N, int B, cudaStream_t s)
{
    g.X.ensure((size_t)N * WARM_F);
    g.Y.ensure((size_t)N);
    g.P.ensure(WARM_NPARAM);
    g.G.ensure(WARM_NPARAM);
    g.H1.ensure((size_t)B * WARM_H);
    g.H2.ensure((size_t)B * WARM_H);
    g.dH1.ensure((size_t)B * WARM_H);
    g.dH2.ensure((size_t)B * WARM_H);
    g.dz.ensure((size_t)B);
    g.lossb.ensure((size_t)B);
    BQB_CUDA(cudaMemcpyAsync(g.X.p, feats, (size_t)N * WARM_F * sizeof(float), cudaMemcpyHostToDevice, s));
    if (targets) BQB_CUDA(cudaMemcpyAsync(g.Y.p, targets, (size_t)N * sizeof(float), cudaMemcpyHostToDevice, s));
}

float batch_loss(WarmGlobal& g, int B, cudaStream_t s)
{
    std::vector<float> l(B);
    BQB_CUDA(cudaMemcpyAsync(l.data(), g.lossb.p, (size_t)B * sizeof(float), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    double t = 0.0;
    for (float v : l) t += v;
    return (float)(t / B);
}

}  // namespace

bool warm_active() { return wg().enabled.load() && wg().loaded; }
bool warm_recording() { return wg().recording.load(); }

void warm_features(WarmDev& w, const Triangle_Inequality* cuts, int m, const double* dX, const double* dL, int n,
                   double viol3, double gap, cudaStream_t s, const double* parent_gam)
{
    if (m <= 0) return;
    int4* hc = w.hcut.ensure(m);
    double* hv = w.hval.ensure(m);
    for (int c = 0; c < m; ++c) {
        hc[c] = make_int4(cuts[c].type, cuts[c].i, cuts[c].j, cuts[c].k);
        hv[c] = cuts[c].value;
    }
    int4* dc = w.cut.ensure(m);
    double* dv = w.val.ensure(m);
    float* df = w.feat.ensure((size_t)m * WARM_F);
    BQB_CUDA(cudaMemcpyAsync(dc, hc, (size_t)m * sizeof(int4), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemcpyAsync(dv, hv, (size_t)m * sizeof(double), cudaMemcpyHostToDevice, s));
    double* dpg = nullptr;
    if (parent_gam) {
        dpg = w.pgam.ensure(m);
        BQB_CUDA(cudaMemcpyAsync(dpg, parent_gam, (size_t)m * sizeof(double), cudaMemcpyHostToDevice, s));
        BQB_CUDA(cudaStreamSynchronize(s));   // the caller's host array may go away
    }
    double* dsc = w.scale.ensure(1);
    warm_scale_kernel<<<1, WT, 0, s>>>(dL, n, dsc);
    BQB_COUNT_LAUNCH();
    warm_feat_kernel<<<blocks(m), WT, 0, s>>>(dc, dv, m, dX, dL, n, viol3, gap, dsc, dpg, df);
    BQB_COUNT_LAUNCH();
    check_launch("warm_feat_kernel");
}

void warm_infer(WarmDev& w, int m, cudaStream_t s)
{
    if (m <= 0) return;
    double* dg = w.gam.ensure(m);
    warm_infer_kernel<<<blocks(m), WT, 0, s>>>(w.feat.p, m, wg().pb.p, w.scale.p, dg);
    BQB_COUNT_LAUNCH();
    check_launch("warm_infer_kernel");
}

double warm_fetch_features(WarmDev& w, int m, std::vector<float>& out, cudaStream_t s)
{
    out.resize((size_t)m * WARM_F);
    if (m <= 0) return 1.0;
    double* hs = w.hscale.ensure(1);
    BQB_CUDA(cudaMemcpyAsync(out.data(), w.feat.p, out.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaMemcpyAsync(hs, w.scale.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    return hs[0];
}

void warm_record(const std::vector<float>& feats, double scale, const Triangle_Inequality* first, int m_first,
                 const Triangle_Inequality* final_cuts, const double* final_gamma, int m_final)
{
    std::map<std::tuple<int, int, int, int>, double> fin;
    for (int c = 0; c < m_final; ++c)
        fin[std::make_tuple(final_cuts[c].type, final_cuts[c].i, final_cuts[c].j, final_cuts[c].k)] = final_gamma[c];
    WarmGlobal& g = wg();
    std::lock_guard<std::mutex> lock(g.mu);
    for (int c = 0; c < m_first; ++c) {
        auto it = fin.find(std::make_tuple(first[c].type, first[c].i, first[c].j, first[c].k));
        g.feats.insert(g.feats.end(), feats.begin() + (size_t)c * WARM_F, feats.begin() + (size_t)(c + 1) * WARM_F);
        // the bundle's multipliers can end a rounding error below 0
        g.targets.push_back(it == fin.end() ? 0.f : (float)(fmax(it->second, 0.0) / scale));
    }
}

void warm_count(bool kept) { (kept ? wg().kept : wg().rejected).fetch_add(1); }

const void* warm_device_params() { return warm_active() ? (const void*)wg().pb.p : nullptr; }

unsigned long long* warm_device_stats()
{
    WarmGlobal& g = wg();
    std::lock_guard<std::mutex> lock(g.mu);
    if (!g.dstats.p) {
        g.dstats.ensure(2);
        BQB_CUDA(cudaMemset(g.dstats.p, 0, 2 * sizeof(unsigned long long)));
    }
    return g.dstats.p;
}

}  // namespace bqb

using namespace bqb;

// Train the warm-start network on (feats[N x WARM_F], targets[N]) with Adam
// on minibatches of `batch` rows (a seeded shuffle per epoch), `steps`
// steps from the parameters in params[WARM_NPARAM], which receive the
// result; losses[steps] (may be null) receives each minibatch's loss.
BQB_API int bqb_warm_train(const float* feats, const float* targets, int N, int steps, int batch, float lr,
                           unsigned seed, float* params, float* losses)
{
    if (!feats || !targets || !params || N <= 0 || steps < 0 || batch <= 0) return -1;
    const int B = std::min(batch, N);
    WarmGlobal& g = wg();
    std::lock_guard<std::mutex> lock(g.mu);
    cudaStream_t s = rt().stream;
    upload_dataset(g, feats, targets, N, B, s);
    g.M1.ensure(WARM_NPARAM);
    g.M2.ensure(WARM_NPARAM);
    int* didx = g.idx.ensure((size_t)B);
    BQB_CUDA(cudaMemcpyAsync(g.P.p, params, WARM_NPARAM * sizeof(float), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemsetAsync(g.M1.p, 0, WARM_NPARAM * sizeof(float), s));
    BQB_CUDA(cudaMemsetAsync(g.M2.p, 0, WARM_NPARAM * sizeof(float), s));
    std::mt19937 rng(seed);
    std::vector<int> order(N);
    for (int i = 0; i < N; ++i) order[i] = i;
    std::vector<int> hidx(B);
    int pos = N;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int t = 1; t <= steps; ++t) {
        for (int b = 0; b < B; ++b) {
            if (pos >= N) {
                std::shuffle(order.begin(), order.end(), rng);
                pos = 0;
            }
            hidx[b] = order[pos++];
        }
        BQB_CUDA(cudaMemcpyAsync(didx, hidx.data(), (size_t)B * sizeof(int), cudaMemcpyHostToDevice, s));
        train_pass(g, didx, B, s);
        const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
        warm_adam_kernel<<<blocks(WARM_NPARAM), WT, 0, s>>>(g.P.p, g.G.p, g.M1.p, g.M2.p, lr * sqrtf(c2) / c1, b1,
                                                            b2, eps * sqrtf(c2));
        BQB_COUNT_LAUNCH();
        check_launch("warm_adam_kernel");
        if (losses) losses[t - 1] = batch_loss(g, B, s);   // synchronises the host thread (hidx reuse)
        else BQB_CUDA(cudaStreamSynchronize(s));
    }
    BQB_CUDA(cudaMemcpyAsync(params, g.P.p, WARM_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    return 0;
}

// Loss and its gradient over all N rows at `params` (the training kernels'
// forward and backward pass, one batch of N): grad[WARM_NPARAM], *loss.
BQB_API int bqb_warm_grad(const float* params, const float* feats, const float* targets, int N, float* grad,
                          float* loss)
{
    if (!params || !feats || !targets || !grad || N <= 0) return -1;
    WarmGlobal& g = wg();
    std::lock_guard<std::mutex> lock(g.mu);
    cudaStream_t s = rt().stream;
    upload_dataset(g, feats, targets, N, N, s);
    BQB_CUDA(cudaMemcpyAsync(g.P.p, params, WARM_NPARAM * sizeof(float), cudaMemcpyHostToDevice, s));
    train_pass(g, nullptr, N, s);
    BQB_CUDA(cudaMemcpyAsync(grad, g.G.p, WARM_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, s));
    const float l = batch_loss(g, N, s);
    if (loss) *loss = l;
    return 0;
}

// The inference path (BF16 weights, FP32 arithmetic) on N feature rows:
// out[N] = proposed multipliers.
BQB_API int bqb_warm_predict(const float* params, const float* feats, int N, double* out)
{
    if (!params || !feats || !out || N <= 0) return -1;
    WarmGlobal& g = wg();
    std::lock_guard<std::mutex> lock(g.mu);
    cudaStream_t s = rt().stream;
    upload_dataset(g, feats, nullptr, N, 1, s);
    float* pf = g.pf.ensure(WARM_NPARAM);
    static DevBuf<__nv_bfloat16> qb;
    static DevBuf<double> dout;
    BQB_CUDA(cudaMemcpyAsync(pf, params, WARM_NPARAM * sizeof(float), cudaMemcpyHostToDevice, s));
    warm_to_bf16_kernel<<<blocks(WARM_NPARAM), WT, 0, s>>>(pf, qb.ensure(WARM_NPARAM), WARM_NPARAM);
    BQB_COUNT_LAUNCH();
    warm_infer_kernel<<<blocks(N), WT, 0, s>>>(g.X.p, N, qb.p, nullptr, dout.ensure(N));
    BQB_COUNT_LAUNCH();
    check_launch("warm_infer_kernel");
    BQB_CUDA(cudaMemcpyAsync(out, dout.p, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, s));
    BQB_CUDA(cudaStreamSynchronize(s));
    return 0;
}

// Load the model SDPbound's warm start uses (params[WARM_NPARAM], stored as
// BF16); null unloads it.  Call before bounding starts, not during.
BQB_API int bqb_warm_set_model(const float* params)
{
    WarmGlobal& g = wg();
    std::lock_guard<std::mutex> lock(g.mu);
    if (!params) {
        g.loaded = false;
        return 0;
    }
    cudaStream_t s = rt().stream;
    float* pf = g.pf.ensure(WARM_NPARAM);
    BQB_CUDA(cudaMemcpyAsync(pf, params, WARM_NPARAM * sizeof(float), cudaMemcpyHostToDevice, s));
    warm_to_bf16_kernel<<<blocks(WARM_NPARAM), WT, 0, s>>>(pf, g.pb.ensure(WARM_NPARAM), WARM_NPARAM);
    BQB_COUNT_LAUNCH();
    check_launch("warm_to_bf16_kernel");
    BQB_CUDA(cudaStreamSynchronize(s));
    g.loaded = true;
    return 0;
}

// Switch the warm start on (a model must be loaded) or off (the default).
BQB_API void bqb_warm_enable(int on) { wg().enabled.store(on != 0); }

// Switch the recording of training pairs on or off (off by default).
BQB_API void bqb_warm_record(int on) { wg().recording.store(on != 0); }

// Recorded training pairs: copies min(count, cap) rows into feats
// (WARM_F floats each) and targets; returns the number recorded.
BQB_API long long bqb_warm_dataset(float* feats, float* targets, long long cap)
{
    WarmGlobal& g = wg();
    std::lock_guard<std::mutex> lock(g.mu);
    const long long count = (long long)g.targets.size();
    const long long k = std::min(count, cap < 0 ? 0LL : cap);
    if (k > 0 && feats && targets) {
        memcpy(feats, g.feats.data(), (size_t)k * WARM_F * sizeof(float));
        memcpy(targets, g.targets.data(), (size_t)k * sizeof(float));
    }
    return count;
}

BQB_API void bqb_warm_dataset_clear(void)
{
    WarmGlobal& g = wg();
    std::lock_guard<std::mutex> lock(g.mu);
    g.feats.clear();
    g.targets.clear();
}

// out[2] = {proposals kept, proposals rejected} since the last reset (the
// engines' and the fused kernel's).
BQB_API void bqb_warm_stats(long long* out, int reset)
{
    WarmGlobal& g = wg();
    out[0] = reset ? g.kept.exchange(0) : g.kept.load();
    out[1] = reset ? g.rejected.exchange(0) : g.rejected.load();
    std::lock_guard<std::mutex> lock(g.mu);
    if (g.dstats.p) {
        unsigned long long d[2];
        BQB_CUDA(cudaDeviceSynchronize());
        BQB_CUDA(cudaMemcpy(d, g.dstats.p, sizeof d, cudaMemcpyDeviceToHost));
        out[0] += (long long)d[0];
        out[1] += (long long)d[1];
        if (reset) BQB_CUDA(cudaMemset(g.dstats.p, 0, sizeof d));
    }
}

// Sizes of the network: out[3] = {features, hidden units, parameters}.
BQB_API void bqb_warm_dims(int* out)
{
    out[0] = WARM_F;
    out[1] = WARM_H;
    out[2] = WARM_NPARAM;
}

// The warm start's features of m triangle cuts (cuts: m x {type, i, j, k};
// values: their violations) at X and the objective L (n x n, column-major,
// host); parent_gamma (m entries, may be NULL): the parent's final
// multiplier of each cut, -1 for one the parent did not hold; out: m x
// WARM_F floats.  For tests against the oracle.
BQB_API int bqb_warm_features(const double* Xh, const double* Lh, int n, const int* cuts, const double* values,
                              int m, double viol3, double gap, const double* parent_gamma, float* out)
{
    if (!Xh || !Lh || !cuts || !values || !out || n <= 0 || m <= 0) return -1;
    static WarmDev w;
    static DevBuf<double> dX, dL;
    WarmGlobal& g = wg();
    std::lock_guard<std::mutex> lock(g.mu);
    cudaStream_t s = rt().stream;
    const size_t nn = (size_t)n * n;
    BQB_CUDA(cudaMemcpyAsync(dX.ensure(nn), Xh, nn * sizeof(double), cudaMemcpyHostToDevice, s));
    BQB_CUDA(cudaMemcpyAsync(dL.ensure(nn), Lh, nn * sizeof(double), cudaMemcpyHostToDevice, s));
    std::vector<Triangle_Inequality> t(m);
    for (int c = 0; c < m; ++c) {
        t[c].type = cuts[4 * c];
        t[c].i = cuts[4 * c + 1];
        t[c].j = cuts[4 * c + 2];
        t[c].k = cuts[4 * c + 3];
        t[c].value = values[c];
        t[c].y = 0.0;
        if (t[c].type < 1 || t[c].type > 4 || t[c].i < 0 || t[c].i >= n || t[c].j < 0 || t[c].j >= n || t[c].k < 0 ||
            t[c].k >= n)
            return -1;
    }
    warm_features(w, t.data(), m, dX.p, dL.p, n, viol3, gap, s, parent_gamma);
    std::vector<float> f;
    warm_fetch_features(w, m, f, s);
    memcpy(out, f.data(), f.size() * sizeof(float));
    return 0;
}
