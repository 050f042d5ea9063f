// Internal (non-exported) device-level API shared by the C entry points
// and the device-resident bounding driver.
#pragma once
#include <vector>

#include "bqb_common.cuh"
#include "cuts.cuh"
#include "globals.h"

namespace bqb {

// Basic SDP bound of one n x n problem already on the device (one launch).
// dout: 4 doubles (phi, iterations, status, <L,X>).  xslot (optional,
// device): write X into dX + (*xslot) * n * n.
void ipm_device(const double* dL, double* dX, int n, double* dout, cudaStream_t s,
                const int* xslot = nullptr);

// Raise the reference's fatal error for a non-zero IPM status word.
void check_ipm_status_host(const double* out);

// Pack the reference's global cut arrays into device records.
std::vector<CutRec> pack_global_cuts(const Problem* P);

// runHeuristic_unpacked with device X, P_L and P0_L (capi_heur.cu).
double heuristic_device(const double* dX, const double* dPL, int n, const double* dP0L, int N0,
                        const int* xfixed, const int* sol, int* x, cudaStream_t s);

}  // namespace bqb
