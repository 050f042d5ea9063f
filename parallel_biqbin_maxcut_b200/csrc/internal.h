// Internal (non-exported) device-level API shared by the C entry points
// and the device-resident bounding driver.
#pragma once
#include <atomic>
#include <vector>

#include "bqb_common.cuh"
#include "cuts.cuh"
#include "globals.h"
#include "heur.cuh"
#include "rng.h"

namespace bqb {

// Basic SDP bound of one n x n problem already on the device (one launch).
// ws: the caller's IPM scratch (grown as needed).  dout: 4 doubles (phi,
// iterations, status, <L,X>).  xslot (optional, device): write X into
// dX + (*xslot) * n * n.  yout (optional, device): y of the last iterate.
void ipm_device(DevBuf<double>& ws, const double* dL, double* dX, int n, double* dout, cudaStream_t s,
                const int* xslot = nullptr, double* yout = nullptr);

// Largest n of the register-resident IPM body (RM_NMAX in reg_linalg.cuh);
// ipm_device hands larger problems to ipm_large.
constexpr int IPM_REG_NMAX = 128;

// ipm_mc_pk for n > IPM_REG_NMAX as one cooperative multi-CTA launch
// (csrc/ipm_large.cu); same arguments and results as ipm_device.
void ipm_large(DevBuf<double>& ws, const double* dL, double* dX, int n, double* dout, cudaStream_t s,
               const int* xslot, double* yout = nullptr);
// Engines bounding nodes with n > IPM_REG_NMAX at the moment: ipm_large
// divides the co-resident CTAs among them (csrc/ipm_large.cu).
extern std::atomic<int> g_large_share;

// FP64 certificate of the basic SDP bound of dL from the dual vector dy (both
// device): dout[0..3] = certified bound, lower bound on lambda_min(Diag(y) -
// L), shift used, status (csrc/certificate.cu).  ws: n x n scratch.
void sdp_certificate(DevBuf<double>& ws, const double* dL, const double* dy, int n, double* dout, cudaStream_t s);

// The lambda_eta counters' device address while the engines' phase profile
// is on, else null (csrc/bundle.cu).
unsigned long long* le_prof_device();

// Raise the reference's fatal error for a non-zero IPM status word.
void check_ipm_status_host(const double* out);

// Pack cut lists into device records (dual-vector order tri | pent | hept).
std::vector<CutRec> pack_cuts(const Triangle_Inequality* c, int mt, const Pentagonal_Inequality* p, int mp,
                              const Heptagonal_Inequality* h, int mh);
// The same for the reference's global cut arrays with P's counts.
std::vector<CutRec> pack_global_cuts(const Problem* P);

// runHeuristic_unpacked (src/heuristic.c:19-115) with device X, P_L and
// P0_L, device state st and random stream rng.  x: host, length N0 - 1.
double heuristic_device(HeurState& st, Rng& rng, const double* dX, const double* dPL, int n, const double* dP0L,
                        int N0, const int* xfixed, const int* sol, int* x, cudaStream_t s, int hyperplanes = 0);

// Hyperplanes per GW round of the engines' heuristic (bqb_set_gw_hyperplanes;
// 0: the reference's count N0 with host draws in rand() order).
int gw_hyperplanes();

}  // namespace bqb
