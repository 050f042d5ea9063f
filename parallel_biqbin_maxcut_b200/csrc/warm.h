// Learned warm start of the bundle multipliers.
//
// After a node's first triangle separation, SDPbound starts its bundle from
// gamma = 0 (src/bounding.c:121-131).  A small network proposes gamma >= 0
// for those cuts instead, from per-cut features of the node's X.  Any
// gamma >= 0 gives a valid bound (the dual function of the cut-augmented
// SDP is an upper bound at every nonnegative gamma), so the proposal only
// changes where the bundle starts: the proposal is evaluated once (one IPM
// on L - B^T(gamma)) and kept only if its dual value is below the plain
// start's; then the plain bundle runs to its own stopping rules.
//
// Network: features (WARM_F) -> WARM_H ReLU -> WARM_H ReLU -> 1, softplus
// output.  Training runs on the GPU (FP32, Adam) with this library's own
// forward and backward kernels; inference uses BF16 weights with FP32
// arithmetic.  Training pairs (features of the first-separation cuts, the
// multipliers those cuts hold when the plain bound ends; 0 for cuts purged
// on the way) are recorded by the plain method itself.
#pragma once
#include <cuda_runtime.h>
#include <vector_types.h>

#include <memory>
#include <unordered_map>
#include <vector>

#include "bqb_common.cuh"
#include "globals.h"

namespace bqb {

constexpr int WARM_F = 14;   // features per cut
constexpr int WARM_H = 32;   // hidden units per layer
// parameter layout (float): W1[F][H], b1[H], W2[H][H], b2[H], w3[H], b3
constexpr int WARM_OFF_W1 = 0;
constexpr int WARM_OFF_B1 = WARM_OFF_W1 + WARM_F * WARM_H;
constexpr int WARM_OFF_W2 = WARM_OFF_B1 + WARM_H;
constexpr int WARM_OFF_B2 = WARM_OFF_W2 + WARM_H * WARM_H;
constexpr int WARM_OFF_W3 = WARM_OFF_B2 + WARM_H;
constexpr int WARM_OFF_B3 = WARM_OFF_W3 + WARM_H;
constexpr int WARM_NPARAM = WARM_OFF_B3 + 1;
static_assert(WARM_NPARAM == BQB_WARM_NPARAM, "the public header's parameter count");

// Per-engine device buffers of the warm start.
struct WarmDev {
    DevBuf<int4> cut;       // (type, i, j, k) per cut
    DevBuf<double> val;     // the cut's violation at X
    DevBuf<float> feat;     // m x WARM_F
    DevBuf<double> gam;     // proposed multipliers
    DevBuf<double> X;       // the IPM solution at the proposal
    DevBuf<double> scale;   // the node's objective scale (mean |L_ij|, i != j)
    DevBuf<double> pgam;    // per cut: the parent's final multiplier (-1: not in the parent's list)
    HostBuf<double> hscale;
    HostBuf<int4> hcut;
    HostBuf<double> hval;
    HostBuf<float> hfeat;
    HostBuf<double> hgam;
};

// A node's final triangle cuts in the original problem's vertex numbering
// (the subproblem's free vertices in order, then the last vertex), with
// the multipliers they end with: what a child node inherits.  A triangle
// keeps its orientation (i > j > k) and its type under this numbering, so
// the same key names the same inequality in parent and child.
// A node's final pentagonal / heptagonal cut in original vertex numbers
// (v[0..k-1]) with its final multiplier.
struct ParentKgon {
    int type;
    int v[7];
    double gam;
};
struct ParentCuts {
    std::vector<uint64_t> key;     // triangle cuts (orig_cut_key) ...
    std::vector<double> gam;       // ... and their final multipliers
    std::unordered_map<uint64_t, double> index;
    std::vector<ParentKgon> pent, hept;
};
inline uint64_t orig_cut_key(int type, int a, int b, int c)
{
    return ((uint64_t)type << 48) | ((uint64_t)a << 32) | ((uint64_t)b << 16) | (uint64_t)c;
}
// Parent cuts whose predicted multiplier (in units of the objective's scale)
// reaches this value join the child's first cut list (the shortlist).
constexpr double WARM_SHORTLIST_MIN = 0.01;

// A model is loaded and warm starts are switched on.
bool warm_active();
// Training pairs are being recorded.
bool warm_recording();

// Features of the m triangle cuts at the device matrices dX and dL (the
// node's objective), n x n, on stream s into w.feat (and the objective's
// scale into w.scale).  viol3: the separation's largest violation; gap:
// the node's bound minus the incumbent; parent_gam (host, m entries, may be
// null): the multiplier each cut ended with in the parent node's final cut
// list, -1 for a cut the parent did not hold.
void warm_features(WarmDev& w, const Triangle_Inequality* cuts, int m, const double* dX, const double* dL, int n,
                   double viol3, double gap, cudaStream_t s, const double* parent_gam = nullptr);
// The proposal for the m cuts whose features are in w.feat, into w.gam.
void warm_infer(WarmDev& w, int m, cudaStream_t s);
// The features of the last warm_features call (m cuts), copied to the
// host; returns the objective's scale.
double warm_fetch_features(WarmDev& w, int m, std::vector<float>& out, cudaStream_t s);
// Record one node's training pairs: the features of its first-separation
// cuts and, per such cut, the multiplier it holds in the final list
// (final_cuts / final_gamma, m_final entries; 0 when it was purged) in units
// of the objective's scale.
void warm_record(const std::vector<float>& feats, double scale, const Triangle_Inequality* first, int m_first,
                 const Triangle_Inequality* final_cuts, const double* final_gamma, int m_final);
// Counters: proposals kept and proposals rejected (worse than the plain start).
void warm_count(bool kept);
// For the fused node kernel: the loaded model's device weights (BF16) when
// the warm start is on, else null; device counters {kept, rejected}.
const void* warm_device_params();
unsigned long long* warm_device_stats();

}  // namespace bqb
