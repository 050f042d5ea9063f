// Process runtime: device binding, stream, error/abort plumbing, and the
// definitions of the reference's process globals (used when the host
// program does not define them itself).
#include <stdarg.h>
#include <string.h>
#include <unistd.h>

#include <mutex>

#include "../../include/bqb_gpu.h"
#include "bqb_common.cuh"

// ---- the reference's globals (src/global_var.h:1-48, src/heap.c:7-8) ----
// A host program that defines them (the reference's allocate_free.c and
// heap.c) takes precedence at dynamic link time; these copies serve
// standalone use of the library.
extern "C" {
__attribute__((visibility("default"))) BiqBinParameters params;
__attribute__((visibility("default"))) Problem* SP = nullptr;
__attribute__((visibility("default"))) Problem* PP = nullptr;
__attribute__((visibility("default"))) double* X = nullptr;
__attribute__((visibility("default"))) double* Z = nullptr;
__attribute__((visibility("default"))) double* X_bundle = nullptr;
__attribute__((visibility("default"))) double* X_test = nullptr;
__attribute__((visibility("default"))) double* dual_gamma = nullptr;
__attribute__((visibility("default"))) double* dgamma = nullptr;
__attribute__((visibility("default"))) double* gamma_test = nullptr;
__attribute__((visibility("default"))) double* lambda = nullptr;
__attribute__((visibility("default"))) double* eta = nullptr;
__attribute__((visibility("default"))) double* F = nullptr;
__attribute__((visibility("default"))) double* G = nullptr;
__attribute__((visibility("default"))) double* g = nullptr;
__attribute__((visibility("default"))) double f = 0.0;
__attribute__((visibility("default"))) Triangle_Inequality* Cuts = nullptr;
__attribute__((visibility("default"))) Triangle_Inequality* List = nullptr;
__attribute__((visibility("default"))) Pentagonal_Inequality* Pent_Cuts = nullptr;
__attribute__((visibility("default"))) Pentagonal_Inequality* Pent_List = nullptr;
__attribute__((visibility("default"))) Heptagonal_Inequality* Hepta_Cuts = nullptr;
__attribute__((visibility("default"))) Heptagonal_Inequality* Hepta_List = nullptr;
__attribute__((visibility("default"))) int BabPbSize = 0;
}

namespace bqb {

std::atomic<unsigned long long> g_launches{0};

static char g_last_error[512] = "";
static std::mutex g_error_mu;
static void (*g_abort_hook)(int) = nullptr;

void set_error(const char* where, const char* msg)
{
    std::lock_guard<std::mutex> lock(g_error_mu);
    snprintf(g_last_error, sizeof g_last_error, "%s: %s", where, msg);
}

thread_local bool t_pool_worker = false;

void fatal(const char* where, const char* msg)
{
    set_error(where, msg);
    fprintf(stderr, "bqb_gpu fatal: %s\n", g_last_error);
    fflush(stderr);
    if (g_abort_hook) {
        g_abort_hook(10);
        return;
    }
    if (t_pool_worker) {
        // exit() from a worker would run the process's destructors under the
        // feet of the other bounding threads: flush and leave at once
        fflush(nullptr);
        _exit(10);
    }
    exit(10);
}

cudaError_t raise_smem_limit(const void* fn, size_t bytes)
{
    // the attribute is a setting of the function on the current device:
    // one cached limit per (device, function)
    constexpr int kMax = 256;
    static std::mutex mu;
    static const void* fns[kMax];
    static int devs[kMax];
    static size_t limit[kMax];
    static int used = 0;
    int dev = 0;
    const cudaError_t ge = cudaGetDevice(&dev);
    if (ge != cudaSuccess) return ge;
    std::lock_guard<std::mutex> lock(mu);
    int i = 0;
    while (i < used && !(fns[i] == fn && devs[i] == dev)) ++i;
    if (i == used) {
        if (used == kMax) return cudaErrorInvalidValue;
        fns[used] = fn;
        devs[used] = dev;
        limit[used] = 0;
        ++used;
    }
    if (bytes <= limit[i]) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) limit[i] = bytes;
    return e;
}

static Runtime g_rt;
static std::once_flag g_once;

static void init_device(int dev)
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        fatal("bqb_init", e != cudaSuccess ? cudaGetErrorString(e) : "no CUDA device");
        return;
    }
    if (dev < 0 || dev >= count) dev = 0;
    BQB_CUDA(cudaSetDevice(dev));
    cudaDeviceProp prop;
    BQB_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) {
        char buf[384];
        snprintf(buf, sizeof buf, "device %s is sm_%d%d; libbqb_gpu is compiled for sm_100a", prop.name,
                 prop.major, prop.minor);
        fatal("bqb_init", buf);
        return;
    }
    // How host threads wait for the device: BQB_SYNC = spin | yield | block
    // (unset: the CUDA runtime's automatic choice).  With many bounding
    // threads on few cores, yield or block leaves the cores to host work.
    if (const char* sync = getenv("BQB_SYNC")) {
        unsigned flags = cudaDeviceScheduleAuto;
        if (!strcmp(sync, "spin")) flags = cudaDeviceScheduleSpin;
        if (!strcmp(sync, "yield")) flags = cudaDeviceScheduleYield;
        if (!strcmp(sync, "block")) flags = cudaDeviceScheduleBlockingSync;
        BQB_CUDA(cudaSetDeviceFlags(flags));
    }
    g_rt.device = dev;
    g_rt.num_sms = prop.multiProcessorCount;
    g_rt.smem_optin = prop.sharedMemPerBlockOptin;
    BQB_CUDA(cudaStreamCreateWithFlags(&g_rt.stream, cudaStreamNonBlocking));
}

Runtime& rt()
{
    std::call_once(g_once, [] {
        // Concurrent engines each launch on their own stream; the runtime
        // maps streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware queues
        // (8 unless set), and streams sharing a queue serialise.  Ask for
        // the maximum unless the host program chose (only effective before
        // the device's context exists).
        setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
        const char* env = getenv("BQB_DEVICE");
        init_device(env ? atoi(env) : 0);
    });
    return g_rt;
}

}  // namespace bqb

extern "C" {

__attribute__((visibility("default"))) int bqb_init(int device)
{
    if (device >= 0) {
        char buf[16];
        snprintf(buf, sizeof buf, "%d", device);
        setenv("BQB_DEVICE", buf, 0);
    }
    bqb::rt();
    return bqb::rt().device >= 0 ? 0 : 1;
}

__attribute__((visibility("default"))) const char* bqb_last_error(void)
{
    return bqb::g_last_error;
}

__attribute__((visibility("default"))) void bqb_set_abort_hook(void (*hook)(int))
{
    bqb::g_abort_hook = hook;
}

__attribute__((visibility("default"))) unsigned long long bqb_kernel_launches(void)
{
    return bqb::g_launches.load();
}

__attribute__((visibility("default"))) void bqb_synchronize(void)
{
    BQB_CUDA(cudaStreamSynchronize(bqb::rt().stream));
}

}  // extern "C"
