// Basic SDP bound (the IPM kernel) with no device allocation at all.
//
// Who needs this: code that is not allowed to call cudaMalloc while it
// runs -- for example a solver embedded in a host application whose memory
// manager owns the whole GPU and hands out no extra device memory, or a
// latency-critical loop where a first-call cudaMalloc (which can
// synchronise the device and fail under memory pressure) is not acceptable.
// Such callers own their inputs and outputs; what they cannot provide is the
// IPM's scratch space.  Here that scratch is one fixed array in the
// module's static device memory, reserved when the library is loaded.
//
// Limits and rules:
//  * n <= BQB_IPM_NOALLOC_NMAX (128).  The scratch array holds 3 * 128^2
//    doubles (384 KiB): the IPM keeps dX and dX1 in global memory, plus Zi
//    when only the Cholesky workspace fits in shared memory (n > 118).
//    Every GPU that loads the library holds this array until the process
//    exits.
//  * The first call on a device resolves the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it; make
//    that first call before any stream capture.
//  * All calls share the one array and it keeps the previous call's
//    contents.  Nothing in it needs to start at zero: every scratch element
//    the kernel reads is written earlier in the same call.  Calls that
//    overlap on the GPU (different streams, or different host threads
//    without ordering) race on the array and give wrong results; order them.
#include <mutex>

#include "../../include/bqb_gpu.h"
#include "ipm.cuh"

namespace {

constexpr int NOALLOC_NMAX = BQB_IPM_NOALLOC_NMAX;
constexpr size_t NOALLOC_DOUBLES = 3 * (size_t)NOALLOC_NMAX * NOALLOC_NMAX;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

std::mutex g_mu;
double* g_scratch_ptr[MAX_DEVICES] = {nullptr};
size_t g_smem_optin[MAX_DEVICES] = {0};

}  // namespace

extern "C" __attribute__((visibility("default"))) int bqb_ipm_noalloc(const double* L, double* X, int n,
                                                                     double* out, void* stream)
{
    if (n < 1 || n > NOALLOC_NMAX) {
        char msg[128];
        snprintf(msg, sizeof msg, "n = %d outside 1..%d (the fixed scratch holds 3*%d^2 doubles)", n,
                 NOALLOC_NMAX, NOALLOC_NMAX);
        bqb::set_error("bqb_ipm_noalloc", msg);
        return 1;
    }
    if (!L || !X || !out) {
        bqb::set_error("bqb_ipm_noalloc", "null device pointer");
        return 1;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        bqb::set_error("bqb_ipm_noalloc", e != cudaSuccess ? cudaGetErrorString(e) : "device index too large");
        return 2;
    }
    double* ws = nullptr;
    size_t optin = 0;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch_ptr[dev]) {
            // set-up, once per device, with that device current
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) {
                bqb::set_error("bqb_ipm_noalloc", cudaGetErrorString(e));
                return 2;
            }
            int v = 0;
            e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
            if (e != cudaSuccess) {
                bqb::set_error("bqb_ipm_noalloc", cudaGetErrorString(e));
                return 2;
            }
            g_smem_optin[dev] = (size_t)v;
            g_scratch_ptr[dev] = (double*)p;
        }
        ws = g_scratch_ptr[dev];
        optin = g_smem_optin[dev];
    }
    size_t bytes = 0;
    const int place = bqb::ipm_place(n, optin, &bytes);
    if (bqb::ipm_ws_doubles(n, place) > NOALLOC_DOUBLES) {
        bqb::set_error("bqb_ipm_noalloc", "scratch too small for this placement");
        return 1;
    }
    const bqb::IpmDesc d{L, X, ws, out, nullptr, n, 0};
    e = bqb::ipm_launch_prepared(d, place, bytes, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        bqb::set_error("bqb_ipm_noalloc", cudaGetErrorString(e));
        return 2;
    }
    return 0;
}
