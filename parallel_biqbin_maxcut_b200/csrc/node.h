// Device-resident state of the node being bounded, and the bounding driver.
#pragma once
#include "bundle.cuh"
#include "cuts.cuh"
#include "globals.h"

namespace bqb {

struct NodeDev {
    int n = 0;
    DevBuf<double> L;      // PP->L (n x n)
    DevBuf<double> L0;     // L - B^T(gamma) scratch
    DevBuf<double> X;      // the reference's global X (current primal matrix)
    DevBuf<double> out;    // IPM output words
    DevBuf<double> P0L;    // SP->L (N0 x N0)
    int P0N = 0;
    const double* P0L_src = nullptr;
    DevCuts cuts;
    BundleDev b;
    HostBuf<double> hs;    // pinned scratch for small reads
    HostBuf<int> hi;
};

NodeDev& node_dev();

// bdl_iter iterations of src/bundle.c:47-235 on the device-resident bundle;
// t in/out on the host.  Synchronises once at the end and returns f.
double bundle_iterations(NodeDev& nd, int bdl_iter, double* t, cudaStream_t s);

// Pack the current host cut lists (globals) and upload them with their
// pair CSR; resize the bundle's m-vectors.
void upload_cuts(NodeDev& nd, const Problem* P, cudaStream_t s);

// updateTriangleInequalities (src/cutting_planes.c:132-214) with the
// separation run on the device-resident X.
double tri_update_dev(NodeDev& nd, Problem* P, const double* y, int* added, int* subtracted, cudaStream_t s);

}  // namespace bqb
