// Goemans-Williamson projection of many random hyperplanes at once on the
// 5th-generation tensor cores (tcgen05, TF32 operands, FP32 accumulation in
// tensor memory), with the sign taken in the epilogue.
//
// The reference projects one hyperplane v at a time, s = Lf v with Lf the
// lower Cholesky factor of Z (src/heuristic.c:119-186), and rounds
// x_i = (s_i < 0) ? -1 : +1.  For H hyperplanes at once that is the product
// S = Lf V (n x n times n x H); only the signs are kept.  The operands are
// FP32 copies of Lf (row-major, K contiguous: the K-major A operand) and of
// V (one hyperplane per row: the K-major B operand), padded with zeros to
// whole tiles.  A sign flipped by TF32 rounding only changes which random
// cut the 1-opt search starts from; every cut found is evaluated exactly
// afterwards.
//
// gw_tc_kernel, one CTA per 128 x 128 output tile, 128 threads:
//  * thread 0 streams K in chunks of 32 TF32 (128 bytes per row, the
//    128-byte swizzle) through STAGES shared-memory stages with TMA
//    (cp.async.bulk.tensor, this GPU's own memory, no multicast), each stage
//    tracked by a "full" mbarrier (transaction bytes) and an "empty"
//    mbarrier (freed by tcgen05.commit when the MMAs reading it are done);
//  * thread 32 issues the MMAs (tcgen05.mma kind::tf32, M = 128, N = 128,
//    K = 8; four per stage) into a 128-column TMEM accumulator and commits
//    the last one to a "done" mbarrier;
//  * all four warps read the accumulator back (tcgen05.ld 32x32b: warp w
//    owns TMEM lanes 32w..32w+31 = rows of the tile) and write either the
//    FP32 product or the signs.
// Every wait is bounded (1 s of globaltimer); a wait that runs out sets an
// error word, and the CTA waits (bounded) for its own copies in flight,
// frees its tensor memory and returns.
#include <cuda.h>
#include <math.h>

#include <mutex>

#include "bqb_common.cuh"
#include "globals.h"

namespace bqb {

namespace {

constexpr int TC_BM = 128;
constexpr int TC_BN = 128;
constexpr int TC_BK = 32;                      // TF32 elements per 128-byte row chunk
constexpr int TC_STAGES = 4;
constexpr int TC_THREADS = 128;
constexpr int TC_A_BYTES = TC_BM * TC_BK * 4;  // 16 KB
constexpr int TC_B_BYTES = TC_BN * TC_BK * 4;  // 16 KB
constexpr int TC_STAGE_BYTES = TC_A_BYTES + TC_B_BYTES;
constexpr int TC_SMEM = TC_STAGES * TC_STAGE_BYTES + 1024 /* alignment */ + 256 /* barriers */;
constexpr unsigned long long TC_TIMEOUT_NS = 1000000000ull;

__device__ __forceinline__ unsigned long long tc_now()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of an mbarrier, at most TC_TIMEOUT_NS.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = tc_now();
    while (!mbar_try_wait(bar, parity))
        if (tc_now() - t0 > TC_TIMEOUT_NS) return false;
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(dst), "l"((unsigned long long)map), "r"(bar), "r"(c0), "r"(c1)
        : "memory");
}

// Shared-memory matrix descriptor: K-major operand tile in the canonical
// 128-byte-swizzle layout (rows of 128 bytes, 8-row atoms 1024 bytes apart).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)1 << 16;                          // leading byte offset (unused with swizzle)
    d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                          // descriptor version (sm100)
    d |= (uint64_t)2 << 61;                          // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D FP32, A and B TF32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N)
{
    return (1u << 4)                      // D format F32
           | (2u << 7)                    // A format TF32
           | (2u << 10)                   // B format TF32
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// D = A B^T for A (M x K) and B (N x K), both given by tensor maps over
// their padded extents.  mode 0: out_f[i + j * ldo] = D(i, j) for i < M,
// j < N (column-major); mode 1: out_x[j * ldo + i] = (D(i, j) < 0) ? -1 : 1
// (hyperplane j's cut, row i).
__global__ void __launch_bounds__(TC_THREADS, 1)
    gw_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M, int N,
                 int K, int mode, float* __restrict__ out_f, int* __restrict__ out_x, int ldo, int* __restrict__ err)
{
    extern __shared__ __align__(16) unsigned char tc_smem_raw[];
    const uint32_t raw = smem_u32(tc_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;   // 1024-byte aligned stages
    unsigned char* gbase = tc_smem_raw + (base - raw);
    const uint32_t bars = base + TC_STAGES * TC_STAGE_BYTES;
    // barrier words: full[s], empty[s], done, then the TMEM address slot
    auto full_bar = [&](int s) { return bars + 8u * s; };
    auto empty_bar = [&](int s) { return bars + 8u * (TC_STAGES + s); };
    const uint32_t done_bar = bars + 8u * (2 * TC_STAGES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + TC_STAGES * TC_STAGE_BYTES + 8 * (2 * TC_STAGES + 1));
    __shared__ int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * TC_BN;
    const int KT = (K + TC_BK - 1) / TC_BK;

    if (tid == 0) {
        s_fail = 0;
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)&tmA) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((unsigned long long)&tmB) : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC_BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    int issued = 0;   // (thread 0) stages loaded
    if (tid == 0) {
        // producer: TMA loads of A (rows m0..) and B (rows n0..), K chunk kt
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % TC_STAGES;
            if (kt >= TC_STAGES && !mbar_wait(empty_bar(s), ((kt / TC_STAGES) - 1) & 1)) {
                s_fail = 1;
                break;
            }
            const uint32_t sa = base + s * TC_STAGE_BYTES, sb = sa + TC_A_BYTES;
            mbar_expect_tx(full_bar(s), TC_STAGE_BYTES);
            tma_load_2d(sa, &tmA, full_bar(s), kt * TC_BK, m0);
            tma_load_2d(sb, &tmB, full_bar(s), kt * TC_BK, n0);
            ++issued;
        }
    } else if (tid == 32) {
        // MMA issuer
        const uint32_t idesc = idesc_tf32(TC_BM, TC_BN);
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % TC_STAGES;
            if (!mbar_wait(full_bar(s), (kt / TC_STAGES) & 1)) {
                s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = base + s * TC_STAGE_BYTES, sb = sa + TC_A_BYTES;
#pragma unroll
            for (int kk = 0; kk < TC_BK / 8; ++kk) {
                // each K = 8 step is 32 bytes further along the 128-byte rows
                umma_tf32(tmem, umma_desc_sw128(sa + 32 * kk), umma_desc_sw128(sb + 32 * kk), idesc,
                          (kt > 0 || kk > 0) ? 1u : 0u);
            }
            umma_commit(empty_bar(s));
        }
        umma_commit(done_bar);   // arrives when every MMA issued above is complete
    }
    __syncwarp();
    // epilogue: every thread waits for the accumulator
    const bool got = mbar_wait(done_bar, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!got) s_fail = 1;
    __syncthreads();
    if (!s_fail) {
        const int row = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < TC_BN; c0 += 32) {
            uint32_t r[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            if (row < M) {
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    const int col = n0 + c0 + q;
                    if (col >= N) continue;
                    const float v = __uint_as_float(r[q]);
                    if (mode == 0) out_f[row + (size_t)col * ldo] = v;
                    else out_x[(size_t)col * ldo + row] = v < 0.f ? -1 : 1;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (s_fail && tid == 0) {
        atomicOr(err, 1);
        // the copies this CTA started land before its shared memory goes away
        for (int kt = 0; kt < issued; ++kt) mbar_wait(full_bar(kt % TC_STAGES), (kt / TC_STAGES) & 1);
    }
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_BN) : "memory");
    }
}

// Lf (n x n, column-major FP64, lower triangle read) -> A (Mp x Kp FP32,
// row-major, zero above the diagonal and in the padding).
__global__ void gw_pack_factor_kernel(const double* __restrict__ Lf, int n, int Mp, int Kp, float* __restrict__ A)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)Mp * Kp) return;
    const int i = (int)(e / Kp), j = (int)(e % Kp);
    A[e] = (i < n && j < n && j <= i) ? (float)Lf[i + (size_t)j * n] : 0.f;
}

// Output `ctr` of the SplitMix64 stream at `seed` (a counter-based draw).
__device__ __forceinline__ unsigned long long gw_draw(unsigned long long seed, unsigned long long ctr)
{
    unsigned long long z = seed + (ctr + 1ull) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// V (H x Kp FP32): hyperplane h, entry j < n uniform in [-0.5, 0.5) from
// draw h * n + j of the stream at `seed`; zero in the padding.
__global__ void gw_hyperplanes_kernel(unsigned long long seed, int n, int H, int Kp, float* __restrict__ V)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)H * Kp) return;
    const int h = (int)(e / Kp), j = (int)(e % Kp);
    float v = 0.f;
    if (j < n) {
        const unsigned long long z = gw_draw(seed, (unsigned long long)h * n + j);
        v = (float)((double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5);
    }
    V[e] = v;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

// Tensor map of a row-major FP32 matrix (rows x cols, row pitch `pitch`
// floats, a multiple of 4) with 128-byte-swizzled boxes of box_rows x 32.
bool make_map(CUtensorMap* map, const float* p, int rows, int cols, int pitch, int box_rows)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)pitch * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(p), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

// D = A B^T on the tensor cores (see gw_tc_kernel).  A: M x K, B: N x K,
// row-major FP32 with row pitch Kp (a multiple of 32, padding zero), both
// 16-byte aligned device pointers.  Returns cudaErrorInvalidValue for bad
// sizes and cudaErrorNotSupported when the tensor-map encoder is missing.
cudaError_t tc_gemm_abt(const float* A, const float* B, int M, int N, int Kp, int mode, float* out_f, int* out_x,
                        int ldo, int* err_dev, cudaStream_t s)
{
    if (M < 1 || N < 1 || Kp < TC_BK || Kp % TC_BK || ((uintptr_t)A & 15) || ((uintptr_t)B & 15))
        return cudaErrorInvalidValue;
    CUtensorMap ta, tb;
    if (!make_map(&ta, A, M, Kp, Kp, TC_BM) || !make_map(&tb, B, N, Kp, Kp, TC_BN)) return cudaErrorNotSupported;
    cudaError_t e = raise_smem_limit((const void*)gw_tc_kernel, TC_SMEM);
    if (e != cudaSuccess) return e;
    const dim3 grid((M + TC_BM - 1) / TC_BM, (N + TC_BN - 1) / TC_BN);
    gw_tc_kernel<<<grid, TC_THREADS, TC_SMEM, s>>>(ta, tb, M, N, Kp, mode, out_f, out_x, ldo, err_dev);
    BQB_COUNT_LAUNCH();
    return cudaGetLastError();
}

// GW rounding of H hyperplanes at once: x[h * n + i] = sign((Lf v_h)_i) for
// the lower factor Lf (device, n x n column-major FP64) and hyperplanes drawn
// on the device from `seed`.  ws: grown as needed.
cudaError_t gw_project_tf32(const double* Lf, int n, int H, unsigned long long seed, int* x, DevBuf<float>& ws,
                            DevBuf<int>& err, cudaStream_t s)
{
    const int Kp = round_up(n, TC_BK), Mp = round_up(n, TC_BM), Hp = round_up(H, TC_BN);
    float* A = ws.ensure((size_t)Mp * Kp + (size_t)Hp * Kp);
    float* V = A + (size_t)Mp * Kp;
    int* e = err.ensure(1);
    BQB_CUDA(cudaMemsetAsync(e, 0, sizeof(int), s));
    gw_pack_factor_kernel<<<(unsigned)(((size_t)Mp * Kp + 255) / 256), 256, 0, s>>>(Lf, n, Mp, Kp, A);
    BQB_COUNT_LAUNCH();
    gw_hyperplanes_kernel<<<(unsigned)(((size_t)Hp * Kp + 255) / 256), 256, 0, s>>>(seed, n, Hp, Kp, V);
    BQB_COUNT_LAUNCH();
    return tc_gemm_abt(A, V, n, H, Kp, 1, nullptr, x, n, e, s);
}

}  // namespace bqb

using namespace bqb;

// D = A B^T in TF32 on the tensor cores, for tests and measurement: A (M x
// K) and B (N x K) row-major FP32 device arrays with row pitch Kp (a
// multiple of 32, zero beyond K), D (M x N, column-major, leading dimension
// M) FP32.  Synchronous.  Returns 0; 1 on bad arguments or a missing
// tensor-map encoder; 2 on a CUDA error or a kernel wait that ran out.
BQB_API int bqb_tc_gemm_tf32(const float* A, const float* B, float* D, int M, int N, int Kp)
{
    Runtime& R = rt();
    static DevBuf<int> err;
    int* e = err.ensure(1);
    BQB_CUDA(cudaMemsetAsync(e, 0, sizeof(int), R.stream));
    const cudaError_t c = tc_gemm_abt(A, B, M, N, Kp, 0, D, nullptr, M, e, R.stream);
    if (c == cudaErrorInvalidValue || c == cudaErrorNotSupported) {
        set_error("bqb_tc_gemm_tf32", cudaGetErrorString(c));
        return 1;
    }
    if (c != cudaSuccess) {
        set_error("bqb_tc_gemm_tf32", cudaGetErrorString(c));
        return 2;
    }
    int h = 0;
    BQB_CUDA(cudaMemcpyAsync(&h, e, sizeof(int), cudaMemcpyDeviceToHost, R.stream));
    BQB_CUDA(cudaStreamSynchronize(R.stream));
    if (h) {
        set_error("bqb_tc_gemm_tf32", "a bounded wait in the kernel ran out");
        return 2;
    }
    return 0;
}
