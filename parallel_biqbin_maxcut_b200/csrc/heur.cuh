// Goemans-Williamson rounding + 1-opt on the GPU.
#pragma once
#include "bqb_common.cuh"

namespace bqb {

// Device state of one heuristic call (grown on demand).
struct HeurState {
    DevBuf<double> Z;          // n x n: X, then its Cholesky factor (lower)
    DevBuf<double> V;          // num x n hyperplanes (row h = hyperplane h)
    DevBuf<int> x;             // num x n  +-1 cuts of the subproblem
    DevBuf<int> sols;          // num x (N0-1) lifted 0/1 solutions
    DevBuf<double> vals;       // num values
    DevBuf<int> best;          // [0] = best index, [1..] = best solution
    DevBuf<double> bestval;    // [0]
    DevBuf<int> fixed;         // 2 x (N0-1): xfixed, sol
    DevBuf<int> status;        // [0] potrf status, [1] 1-opt overflow
    DevBuf<double> P0L, PL, Xs; // staging for host-pointer entry points
    DevBuf<float> Vf;          // batched rounding: FP32 factor and hyperplanes
    DevBuf<int> tcerr;         // batched rounding: the tensor-core kernel's error word
    HostBuf<double> hV;
    HostBuf<int> hbest;
    HostBuf<double> hval;
    HostBuf<int> hstat;
};

// Z <- lower Cholesky factor of Z (n x n) in place; *dstatus = 0 ok, 1 not PD.
void potrf_device(double* dZ, int n, int* dstatus, cudaStream_t s);

// Z = (1 - c) X + c xh xh^T on the lower triangle (src/heuristic.c:105-110).
void remix_device(double* dZ, const double* dX, const double* dxh, double c, int n, cudaStream_t s);

// One GW round (src/heuristic.c:119-186) with the factor already in st.Z and
// the hyperplanes in st.V:  sign(L v) per hyperplane, 1-opt on P_L, lift with
// the node's fixed variables, evaluate on P0_L, keep the first best.
// Results: st.best (device), st.bestval (device).
void gw_round_device(HeurState& st, const double* dPL, int n, const double* dP0L, int N0, int num,
                     cudaStream_t s);

// The steps of a GW round after the projection (cuts already in st.x):
// 1-opt, lift, evaluate, keep the first best.
void gw_round_finish(HeurState& st, const double* dPL, int n, const double* dP0L, int N0, int num, cudaStream_t s);

// Batched rounding on the tensor cores (csrc/gw_tc.cu): x[h * n + i] =
// sign((Lf v_h)_i) for H hyperplanes drawn on the device from `seed`, Lf the
// lower factor in st.Z.
cudaError_t gw_project_tf32(const double* Lf, int n, int H, unsigned long long seed, int* x, DevBuf<float>& ws,
                            DevBuf<int>& err, cudaStream_t s);

// 1-opt alone on `count` cuts stored as rows of st.x (n ints each); writes
// the final cost of cut h to st.vals[h].
void one_opt_device(HeurState& st, const double* dPL, int n, int count, cudaStream_t s);

// Value of the 0/1 vectors in st.sols rows 0..count-1 on P0_L
// (src/bab_functions.c:96-107) into st.vals.
void evaluate_device(HeurState& st, const double* dP0L, int N0, int count, cudaStream_t s);

}  // namespace bqb
