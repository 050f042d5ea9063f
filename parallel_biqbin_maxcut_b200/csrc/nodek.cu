// Fused node bounding: SDPbound (src/bounding.c:24-342) for a whole node in
// one CTA, many nodes at once.
//
// The engine path (node.cu) runs a node as a chain of small kernels driven
// by a host thread: one IPM CTA at a time per node, a host round trip at
// every decision, and at most ~32 nodes in flight (the hardware queues of
// independent streams).  Here a persistent kernel gives every SM one CTA
// (IPM_THREADS threads); each CTA pulls node indices from a counter and
// runs the complete bound on the device: subproblem construction
// (src/evaluate.c:38-138), the basic IPM, the GW heuristic with 1-opt,
// triangle separation and the cut-list updates, pentagonal / heptagonal
// separation by annealing chains, the bundle iterations and every prune /
// give-up test of the reference, in its order.  No host interaction until
// the batch is done.
//
// The phases run the same device code as the engine path where that code
// is a CTA body: the register-resident IPM (ipm_reg_body.cuh), lambda_eta
// and the bundle step (bundle_body.cuh), the cut operators (cuts.cuh) and
// the annealing chains (kgon_sa.cuh), with the same thread count, so the
// arithmetic is the same.  Triangle separation restates trisep.cu's passes
// as CTA loops and produces the same list.  Cut lists live on the device:
// purges and appends are ordered compactions, membership is a hash set of
// the kept triangle codes (a linear scan for the few k-gonal cuts), and the
// pair CSR for B^T is built by counting, filling and sorting every pair's
// short segment into cut order.
//
// Random numbers: the heuristic draws counter-based SplitMix64 values from
// a per-node stream (seed, node index), the annealing chains per call; the
// incumbent is a device word updated with atomicMax on order-preserving
// bits, read once per decision by thread 0 and broadcast.
//
// Nodes that exceed a slot's capacities (bundle size, cut counts) or meet a
// numerical failure are flagged; the host bounds them again on an engine.
#include <math.h>

#include "bundle_body.cuh"
#include "cuts.cuh"
#include "ipm_reg_body.cuh"
#include "kgon_sa.cuh"
#include "nodek.h"
#include "trisep.cuh"
#include "warm_body.cuh"

namespace bqb {

namespace {

constexpr int NKT = IPM_THREADS;
constexpr double NK_BIG = 1e9;          // BIG_NUMBER, src/biqbin.h:35
constexpr int NK_RAND_MAX = 2147483647;
constexpr int NK_MAX_GW_ROUNDS = 1000;  // rounds of one heuristic call (each improvement needs a larger cut value)

__shared__ int nk_si[8];
__shared__ unsigned long long nk_t0[NKP_COUNT];

__device__ __forceinline__ unsigned long long nk_now()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The kernel's dynamic shared memory.  Most phases below are separate
// functions (not inlined); they name this array instead of taking a pointer,
// so the compiler keeps shared-memory addressing across the call boundary.
extern __shared__ __align__(16) double nk_smem[];

// Phase timer: thread 0 adds the elapsed time of the enclosing scope to
// prof[phase] and counts the scope in prof[NKP_COUNT + phase].
struct NkTimer {
    unsigned long long* prof;
    int phase;
    unsigned long long t0;
    __device__ NkTimer(unsigned long long* p, int ph) : prof(p), phase(ph), t0(0)
    {
        if (threadIdx.x == 0 && prof) t0 = nk_now();
    }
    __device__ ~NkTimer()
    {
        if (threadIdx.x == 0 && prof) {
            atomicAdd(&prof[phase], nk_now() - t0);
            atomicAdd(&prof[NKP_COUNT + phase], 1ULL);
        }
    }
};
__shared__ double nk_sd[8];
__shared__ int nk_sw[40];
__shared__ double nk_red[64];

__device__ __forceinline__ int bcast_i(int v)
{
    if (threadIdx.x == 0) nk_si[0] = v;
    __syncthreads();
    const int r = nk_si[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double bcast_d(double v)
{
    if (threadIdx.x == 0) nk_sd[0] = v;
    __syncthreads();
    const double r = nk_sd[0];
    __syncthreads();
    return r;
}

// Counter-based draw: output `ctr` of the SplitMix64 stream at `seed`.
__device__ __forceinline__ uint32_t nk_rand(unsigned long long seed, unsigned long long ctr)
{
    uint64_t z = seed + (ctr + 1ull) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (uint32_t)(z >> 33);
}

__device__ __forceinline__ unsigned long long nk_mix(unsigned long long a, unsigned long long b)
{
    uint64_t z = a ^ (b * 0xD1B54A32D192ED03ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Exclusive scan of a[0..N) in place; returns the total (uniform).
__device__ unsigned long long cta_scan_u32(uint32_t* a, long long N)
{
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned long long carry_s;
    constexpr int ITEMS = 8;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nt = blockDim.x;
    if (tid == 0) carry_s = 0;
    __syncthreads();
    for (long long base = 0; base < N; base += (long long)nt * ITEMS) {
        uint32_t v[ITEMS];
        unsigned long long s = 0;
        const long long off = base + (long long)tid * ITEMS;
#pragma unroll
        for (int q = 0; q < ITEMS; ++q) {
            v[q] = (off + q < N) ? a[off + q] : 0u;
            s += v[q];
        }
        unsigned long long incl = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            unsigned long long w = lane < (nt >> 5) ? wsum[lane] : 0ull;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        unsigned long long run = carry_s + (warp ? wsum[warp - 1] : 0ull) + incl - s;
#pragma unroll
        for (int q = 0; q < ITEMS; ++q) {
            if (off + q < N) a[off + q] = (uint32_t)run;
            run += v[q];
        }
        __syncthreads();
        if (tid == 0) carry_s += wsum[(nt >> 5) - 1];
        __syncthreads();
    }
    const unsigned long long total = carry_s;
    __syncthreads();
    return total;
}

// Ordered compaction: for idx < N (in order) load(idx) -> v, keep(idx, v)
// selects, store(pos, v) writes the pos-th selected value.  All loads of a
// chunk precede its stores, and positions never pass the chunk, so the
// output may overwrite the input in place.  Returns the count (uniform).
template <class T, class Load, class Keep, class Store>
__device__ int cta_compact(int N, Load load, Keep keep, Store store)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    int total = 0;
    for (int base = 0; base < N; base += blockDim.x) {
        const int idx = base + tid;
        T v{};
        bool f = false;
        if (idx < N) {
            v = load(idx);
            f = keep(idx, v);
        }
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) nk_sw[warp] = __popc(m);
        __syncthreads();
        if (tid == 0) {
            int r = 0;
            for (int w = 0; w < nw; ++w) {
                const int c = nk_sw[w];
                nk_sw[w] = r;
                r += c;
            }
            nk_sw[32] = r;
        }
        __syncthreads();
        if (f) store(total + nk_sw[warp] + __popc(m & ((1u << lane) - 1u)), v);
        total += nk_sw[32];
        __syncthreads();
    }
    return total;
}

// ---------------------------------------------------------------------------
// Slot state
// ---------------------------------------------------------------------------
struct Nk {
    double *L, *L0, *X, *ws, *out, *Xb, *G, *Fv, *lam, *gam, *gtest, *dgam, *eta, *dstate, *qpws;
    int *slot, *slot_old, *istate;
    uint32_t* tricode;
    double* triy;
    unsigned long long* pentkey;
    double* penty;
    unsigned long long* heptkey;
    double* hepty;
    CutRec* rec;
    uint32_t *csroff, *csrcur, *contrib, *hash;
    uint32_t* tscnt;
    TriCand *tscand, *tslist;
    double* sacost;
    int* saperm;
    unsigned long long* klist;
    double* klistv;
    double* hz;
    double* hv;
    int* hx;
    double* hval;
    int* hsol;
    int* hbest;
    double* xh;
    int* freemap;
    int* fixedlist;

    int node, n, N0, N, nfix;
    const int *xf, *sx;
    double fixedvalue;
    int mt, mp, mh, ldg;
    unsigned long long hseed, hctr, saseed;
    unsigned sacalls;
    int status;
    double best_h;
};

template <class T>
__device__ __forceinline__ T* nk_arr(const FusedCfg& c, unsigned char* base, int id)
{
    return (T*)(base + c.off[id]);
}

__device__ void nk_bind(const FusedCfg& c, Nk& k, int slot_index)
{
    unsigned char* b = c.arena + (size_t)slot_index * c.slot_bytes;
    k.L = nk_arr<double>(c, b, NK_L);
    k.L0 = nk_arr<double>(c, b, NK_L0);
    k.X = nk_arr<double>(c, b, NK_X);
    k.ws = nk_arr<double>(c, b, NK_IPMWS);
    k.out = nk_arr<double>(c, b, NK_OUT);
    k.Xb = nk_arr<double>(c, b, NK_XB);
    k.G = nk_arr<double>(c, b, NK_G);
    k.Fv = nk_arr<double>(c, b, NK_FV);
    k.lam = nk_arr<double>(c, b, NK_LAM);
    k.gam = nk_arr<double>(c, b, NK_GAM);
    k.gtest = nk_arr<double>(c, b, NK_GTEST);
    k.dgam = nk_arr<double>(c, b, NK_DGAM);
    k.eta = nk_arr<double>(c, b, NK_ETA);
    k.dstate = nk_arr<double>(c, b, NK_DSTATE);
    k.qpws = nk_arr<double>(c, b, NK_QPWS);
    k.slot = nk_arr<int>(c, b, NK_SLOT);
    k.slot_old = nk_arr<int>(c, b, NK_SLOTOLD);
    k.istate = nk_arr<int>(c, b, NK_ISTATE);
    k.tricode = nk_arr<uint32_t>(c, b, NK_TRICODE);
    k.triy = nk_arr<double>(c, b, NK_TRIY);
    k.pentkey = nk_arr<unsigned long long>(c, b, NK_PENTKEY);
    k.penty = nk_arr<double>(c, b, NK_PENTY);
    k.heptkey = nk_arr<unsigned long long>(c, b, NK_HEPTKEY);
    k.hepty = nk_arr<double>(c, b, NK_HEPTY);
    k.rec = nk_arr<CutRec>(c, b, NK_REC);
    k.csroff = nk_arr<uint32_t>(c, b, NK_CSROFF);
    k.csrcur = nk_arr<uint32_t>(c, b, NK_CSRCUR);
    k.contrib = nk_arr<uint32_t>(c, b, NK_CONTRIB);
    k.hash = nk_arr<uint32_t>(c, b, NK_HASH);
    k.tscnt = nk_arr<uint32_t>(c, b, NK_TSCNT);
    k.tscand = nk_arr<TriCand>(c, b, NK_TSCAND);
    k.tslist = nk_arr<TriCand>(c, b, NK_TSLIST);
    k.sacost = nk_arr<double>(c, b, NK_SACOST);
    k.saperm = nk_arr<int>(c, b, NK_SAPERM);
    k.klist = nk_arr<unsigned long long>(c, b, NK_KLIST);
    k.klistv = nk_arr<double>(c, b, NK_KLISTV);
    k.hz = nk_arr<double>(c, b, NK_HZ);
    k.hv = nk_arr<double>(c, b, NK_HV);
    k.hx = nk_arr<int>(c, b, NK_HX);
    k.hval = nk_arr<double>(c, b, NK_HVAL);
    k.hsol = nk_arr<int>(c, b, NK_HSOL);
    k.hbest = nk_arr<int>(c, b, NK_HBEST);
    k.xh = nk_arr<double>(c, b, NK_XH);
    k.freemap = nk_arr<int>(c, b, NK_FREE);
    k.fixedlist = nk_arr<int>(c, b, NK_FIXED);
    k.ldg = c.mt_cap + c.mp_cap + c.mh_cap;
}

// The incumbent, read by thread 0 and broadcast (every thread takes the
// same decision even while other CTAs raise it).
__device__ double nk_lb(const FusedCfg& c)
{
    double v = 0.0;
    if (threadIdx.x == 0) v = ordered_to_dbl(*(volatile unsigned long long*)c.lb);
    return bcast_d(v);
}

// ---------------------------------------------------------------------------
// Subproblem (src/evaluate.c:38-138: createSubproblem, getFixedValue)
// ---------------------------------------------------------------------------
__device__ __noinline__ void nk_subproblem(const FusedCfg& c, Nk& k)
{
    NkTimer tm(c.prof, NKP_SUB);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int N = k.N, N0 = k.N0;
    const int* xf = k.xf;
    const int* sx = k.sx;
    if (tid == 0) {
        int r = 0, nf = 0;
        for (int i = 0; i < N; ++i) {
            if (xf[i]) {
                k.freemap[i] = -1;
                k.fixedlist[nf++] = i;
            } else {
                k.freemap[i] = r++;
            }
        }
        nk_si[1] = r + 1;
        nk_si[2] = nf;
    }
    __syncthreads();
    const int n = nk_si[1];
    k.nfix = nk_si[2];
    __syncthreads();
    k.n = n;
    double* L = k.L;
    double* fr = k.xh;   // fixedRow, by free rank
    for (int i = tid; i < N; i += nt) {
        if (xf[i]) continue;
        const int ri = k.freemap[i];
        double rs = 0.0;
        for (int j = 0; j < N; ++j) {
            if (xf[j]) continue;
            const double v = c.P0L[j + (size_t)i * N0];
            L[k.freemap[j] + (size_t)ri * n] = v;
            rs += v;
        }
        L[n - 1 + (size_t)ri * n] = rs;
        double f = 0.0;
        for (int q = 0; q < k.nfix; ++q) {
            const int a = k.fixedlist[q];
            if (sx[a] == 1) f += c.P0L[i + (size_t)a * N0];
        }
        fr[ri] = f;
    }
    __syncthreads();
    for (int i = tid; i < n - 1; i += nt) L[i + (size_t)(n - 1) * n] = L[n - 1 + (size_t)i * n];
    __syncthreads();
    for (int i = tid; i < n - 1; i += nt) {
        const double f2 = 2 * fr[i];
        L[i + (size_t)i * n] += f2;
        L[n - 1 + (size_t)i * n] += f2;
        L[i + (size_t)(n - 1) * n] += f2;
    }
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int i = 0; i < n - 1; ++i) s += L[i + (size_t)(n - 1) * n];
        L[n - 1 + (size_t)(n - 1) * n] = s;
        double v = 0.0;
        for (int qa = 0; qa < k.nfix; ++qa) {
            const int i = k.fixedlist[qa];
            for (int qb = 0; qb < k.nfix; ++qb) {
                const int j = k.fixedlist[qb];
                v += c.P0L[j + (size_t)i * N0] * sx[i] * sx[j];
            }
        }
        nk_sd[1] = v;
    }
    __syncthreads();
    k.fixedvalue = nk_sd[1];
    const size_t nn = (size_t)n * n;
    for (size_t e = tid; e < nn; e += nt) L[e] *= 0.25;
    __syncthreads();
}

// ---------------------------------------------------------------------------
// IPM (the engine's kernel body)
// ---------------------------------------------------------------------------
// Separate (not inlined) so the IPM body keeps the whole register budget.
// (The IPM body takes the shared memory as a generic pointer: measured
// faster here than naming nk_smem inside.)
__device__ __noinline__ void nk_ipm_call(IpmDesc d, double* smem, int zi, double* stats)
{
    ipm_body_reg(d, smem, zi, stats);
}

__device__ bool nk_ipm(const FusedCfg& c, Nk& k, const double* Lsrc, double* Xdst, const int* xslot)
{
    const int n = k.n;
    const size_t fixed = ipm_reg_fixed_smem_doubles(n) * sizeof(double);
    const size_t mat = (size_t)n * n * sizeof(double);
    const int zi = fixed + 2 * mat <= c.smem_bytes ? 1 : 0;
    IpmDesc d{Lsrc, Xdst, k.ws, k.out, xslot, n, 0};
    {
        NkTimer tm(c.prof, NKP_IPM);
        nk_ipm_call(d, nk_smem, zi, c.ipm_stats);
    }
    __syncthreads();
    if ((int)k.out[2] != IPM_OK) {
        k.status |= NKS_IPM;
        return false;
    }
    return true;
}

__device__ void nk_fracsol(const FusedCfg& c, Nk& k)
{
    const int n = k.n;
    double* fs = c.fracsol + (size_t)k.node * k.N;
    for (int i = threadIdx.x; i < k.N; i += blockDim.x)
        fs[i] = k.xf[i] ? (double)k.sx[i] : __dmul_rn(0.5, __dadd_rn(k.X[(size_t)(n - 1) * n + k.freemap[i]], 1.0));
    __syncthreads();
}

// Value of the 0/1 vector s (N entries) on SP->L: sum_ij L_ij s_i s_j
// (src/bab_functions.c:96-107), by the calling warp.  Integer data: exact.
__device__ double nk_eval_warp(const FusedCfg& c, const int* s, int N)
{
    const int lane = threadIdx.x & 31;
    double part = 0.0;
    for (int i = lane; i < N; i += 32) {
        if (!s[i]) continue;
        const double* Li = c.P0L + (size_t)i * c.N0;
        double r = 0.0;
        for (int j = 0; j < N; ++j)
            if (s[j]) r += Li[j];
        part += r;
    }
    return warp_sum(part);
}

// updateSolution (src/bab_functions.c:114-136) on the device: raise the
// incumbent and keep the node's best reported solution for the host.
__device__ void nk_report(const FusedCfg& c, Nk& k, double value, const int* x)
{
    const double lb = nk_lb(c);
    if (value > lb && threadIdx.x == 0) atomicMax(c.lb, dbl_to_ordered(value));
    if (value > k.best_h) {
        for (int i = threadIdx.x; i < k.N; i += blockDim.x) c.hsol[(size_t)k.node * k.N + i] = x[i];
        if (threadIdx.x == 0) c.hval[k.node] = value;
        k.best_h = value;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Heuristic (src/heuristic.c:19-115, 119-186, 197-290) with per-node
// counter-based random numbers.  Shared: Z (n^2), column buffer, 1-opt
// buffers.
// ---------------------------------------------------------------------------
__device__ __noinline__ double nk_heuristic(const FusedCfg& c, Nk& k)
{
    double* const smem = nk_smem;
    NkTimer tm(c.prof, NKP_HEUR);
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const int n = k.n, N = k.N, num = k.N0;
    const size_t nn = (size_t)n * n;
    const int nv = (n + 1) & ~1;
    double* Zs = smem;
    double* colb = Zs + nn;
    double* dg = colb + nv;
    double* wbuf = dg + nv;   // per warp: Lx[nv], x[nv] (as int)
    if (tid == 0) nk_si[5] = 0;

    for (int i = tid; i < n; i += nt) k.xh[i] = 2 * (int)(nk_rand(k.hseed, k.hctr + i) % 2u) - 1;
    k.hctr += n;
    __syncthreads();
    // fh: the random cut lifted with the fixed variables
    if (warp == 0) {
        for (int i = lane; i < N; i += 32)
            k.hbest[i] = k.xf[i] ? k.sx[i] : (int)((k.xh[k.freemap[i]] + 1) / 2.0);
        __syncwarp();
        const double v = nk_eval_warp(c, k.hbest, N);
        if (lane == 0) nk_sd[2] = v;
    }
    __syncthreads();
    double fh = nk_sd[2];
    __syncthreads();
    for (size_t e = tid; e < nn; e += nt) Zs[e] = k.X[e];
    for (int i = tid; i < n; i += nt) dg[i] = k.L[i + (size_t)i * n];
    __syncthreads();
    int done = 0, rounds = 0;
    double heur_val = -NK_BIG;
    while (done < 2 && rounds < NK_MAX_GW_ROUNDS) {
        ++done;
        ++rounds;
        if (!cta_potrf_lower(Zs, n, n, colb)) {
            k.status |= NKS_HEUR;
            __syncthreads();
            return heur_val;
        }
        __syncthreads();
        // hyperplanes v = rand/RAND_MAX - 0.5 and cuts x = sign(L v)
        const size_t nvh = (size_t)num * n;
        for (size_t q = tid; q < nvh; q += nt)
            k.hv[q] = __dsub_rn(__ddiv_rn((double)nk_rand(k.hseed, k.hctr + q), (double)NK_RAND_MAX), 0.5);
        k.hctr += nvh;
        __syncthreads();
        for (size_t q = tid; q < nvh; q += nt) {
            const int h = (int)(q / n), i = (int)(q % n);
            const double* v = k.hv + (size_t)h * n;
            double acc = 0.0;
            for (int j = 0; j <= i; ++j) acc = __dadd_rn(acc, __dmul_rn(v[j], Zs[i + (size_t)j * n]));
            k.hx[q] = (acc < 0) ? -1 : 1;
        }
        __syncthreads();
        // 1-opt on P_L, one warp per cut (src/heuristic.c:197-290)
        {
            double* Lx = wbuf + (size_t)warp * 2 * nv;
            int* x = (int*)(Lx + nv);
            for (int h = warp; h < num; h += nw) {
                int* xg = k.hx + (size_t)h * n;
                for (int i = lane; i < n; i += 32) x[i] = xg[i];
                __syncwarp();
                for (int i = lane; i < n; i += 32) {
                    double acc = 0.0;
                    for (int j = 0; j < n; ++j) acc += k.L[i + (size_t)j * n] * (double)x[j];
                    Lx[i] = acc;
                }
                __syncwarp();
                const int cap = 10 * n + 100;
                int flips = 0;
                while (true) {
                    double best = -1e300;
                    int idx = 0x7fffffff;
                    for (int i = lane; i < n; i += 32) {
                        const double dl = dg[i] - (double)x[i] * Lx[i];
                        if (dl > best) {
                            best = dl;
                            idx = i;
                        }
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
                        if (ob > best || (ob == best && oi < idx)) {
                            best = ob;
                            idx = oi;
                        }
                    }
                    if (!(best > 0.001)) break;
                    if (++flips > cap) {
                        if (lane == 0) atomicOr(&nk_si[5], 1);
                        break;
                    }
                    const double sgn = (x[idx] > 0) ? -2.0 : 2.0;
                    const double* col = k.L + (size_t)idx * n;
                    __syncwarp();
                    for (int j = lane; j < n; j += 32) {
                        const double lv = col[j];
                        if (fabs(lv) > 0.001) Lx[j] += sgn * lv;
                    }
                    if (lane == 0) x[idx] = -x[idx];
                    __syncwarp();
                }
                __syncwarp();
                for (int i = lane; i < n; i += 32) xg[i] = x[i];
                __syncwarp();
            }
        }
        __syncthreads();
        // lift with the fixed variables and evaluate on SP->L
        for (int h = warp; h < num; h += nw) {
            int* s = k.hsol + (size_t)h * N;
            const int* x = k.hx + (size_t)h * n;
            for (int i = lane; i < N; i += 32) s[i] = k.xf[i] ? k.sx[i] : (x[k.freemap[i]] + 1) / 2;
            __syncwarp();
            const double v = nk_eval_warp(c, s, N);
            if (lane == 0) k.hval[h] = v;
        }
        __syncthreads();
        if (tid == 0) {
            double b = -NK_BIG;
            int hb = 0;
            for (int h = 0; h < num; ++h)
                if (b < k.hval[h]) {
                    b = k.hval[h];
                    hb = h;
                }
            nk_sd[3] = b;
            nk_si[3] = hb;
        }
        __syncthreads();
        heur_val = nk_sd[3];
        const int hb = nk_si[3];
        for (int i = tid; i < N; i += nt) k.hbest[i] = k.hsol[(size_t)hb * N + i];
        __syncthreads();
        if (heur_val > fh) {
            done = 0;
            fh = heur_val;
            for (int i = tid; i < N; i += nt)
                if (!k.xf[i]) k.xh[k.freemap[i]] = 2 * k.hbest[i] - 1;
            if (tid == 0) k.xh[n - 1] = -1.0;
        }
        const double cc = 0.3 + 0.6 * ((double)nk_rand(k.hseed, k.hctr) / (double)NK_RAND_MAX);
        k.hctr += 1;
        __syncthreads();
        for (size_t e = tid; e < nn; e += nt) {
            const int i = (int)(e % n), j = (int)(e / n);
            const double a = (1.0 - cc) * k.X[e];
            Zs[e] = a + k.xh[i] * (cc * k.xh[j]);
        }
        __syncthreads();
    }
    if (nk_si[5]) k.status |= NKS_HEUR;
    __syncthreads();
    nk_report(c, k, heur_val, k.hbest);
    return heur_val;
}

// ---------------------------------------------------------------------------
// Triangle separation (src/cutting_planes.c:20-127): trisep.cu's passes as
// CTA loops.  X is staged transposed in shared memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void nk_pair_decode(long long p, int* i, int* j)
{
    int ii = (int)floor((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
    while ((long long)ii * (ii - 1) / 2 > p) --ii;
    while ((long long)(ii + 1) * ii / 2 <= p) ++ii;
    *i = ii;
    *j = (int)(p - (long long)ii * (ii - 1) / 2);
}

__device__ __forceinline__ bool nk_heap_less(const double* hv, const int* hs, int a, int b)
{
    return hv[a] < hv[b] || (hv[a] == hv[b] && hs[a] < hs[b]);
}

__device__ void nk_heap_down(double* hv, int* hs, int T, int i)
{
    while (true) {
        const int l = 2 * i + 1, r = l + 1;
        int m = i;
        if (l < T && nk_heap_less(hv, hs, l, m)) m = l;
        if (r < T && nk_heap_less(hv, hs, r, m)) m = r;
        if (m == i) return;
        const double tv = hv[i];
        hv[i] = hv[m];
        hv[m] = tv;
        const int ts = hs[i];
        hs[i] = hs[m];
        hs[m] = ts;
        i = m;
    }
}

// Returns the maximum violation; list in k.tslist, its size in *size.
__device__ __noinline__ double nk_trisep(const FusedCfg& c, Nk& k, const double* X, int* size)
{
    double* const smem = nk_smem;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const int n = k.n;
    const int T = c.TriIneq;
    const double thr = c.violated_TriIneq;
    const long long P = (long long)n * (n - 1) / 2;
    if (n < 3 || P <= 0) {
        *size = 0;
        return -NK_BIG;
    }
    double* XT = smem;   // XT[k + i n] = X[i + k n]
    const size_t nn = (size_t)n * n;
    for (size_t e = tid; e < nn; e += nt) {
        const int i = (int)(e % n), kk = (int)(e / n);
        XT[kk + (size_t)i * n] = X[e];
    }
    __syncthreads();
    uint32_t* cnt = k.tscnt;
    double vmax = -NK_BIG;
    const unsigned lt = (1u << lane) - 1u;
    for (int pass = 0; pass < 2; ++pass) {
        for (long long p = warp; p < P; p += nw) {
            int i, j;
            nk_pair_decode(p, &i, &j);
            const double a = XT[j + (size_t)i * n];
            const double* Bi = XT + (size_t)i * n;
            const double* Bj = XT + (size_t)j * n;
            uint32_t c4[4] = {0u, 0u, 0u, 0u};
            uint32_t base[4] = {0u, 0u, 0u, 0u};
            if (pass == 1) {
#pragma unroll
                for (int t = 0; t < 4; ++t) base[t] = cnt[t * P + p];
            }
            for (int k0 = 0; k0 < j; k0 += 32) {
                const int kk = k0 + lane;
                const bool valid = kk < j;
                const double b = valid ? Bi[kk] : 0.0;
                const double cv = valid ? Bj[kk] : 0.0;
                double v[4];
                tri_values(a, b, cv, v);
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const bool hit = valid && v[t] > thr;
                    const unsigned m = __ballot_sync(0xffffffffu, hit);
                    if (pass == 0) {
                        if (valid) vmax = fmax(vmax, v[t]);
                    } else if (hit) {
                        TriCand cd;
                        cd.value = v[t];
                        cd.code = tri_code(t + 1, i, j, kk);
                        cd.pad_ = 0u;
                        k.tscand[base[t] + c4[t] + __popc(m & lt)] = cd;
                    }
                    c4[t] += __popc(m);
                }
            }
            if (pass == 0 && lane == 0) {
#pragma unroll
                for (int t = 0; t < 4; ++t) cnt[t * P + p] = c4[t];
            }
        }
        __syncthreads();
        if (pass == 0) {
            vmax = block_max(vmax, nk_red);
            const unsigned long long V = cta_scan_u32(cnt, 4 * P);
            if (tid == 0) nk_si[4] = (int)V;
            __syncthreads();
        }
    }
    const long long V = nk_si[4];
    __syncthreads();
    // streaming top-T replay by warp 0 (trisep.cu tri_replay_kernel)
    double* hv = smem;   // XT is dead
    int* hs = (int*)(hv + (T > 0 ? T : 1));
    if (warp == 0) {
        if (T <= 0) {
            if (lane == 0) nk_si[6] = 0;
        } else if (V <= T) {
            for (long long q = lane; q < V; q += 32) k.tslist[q] = k.tscand[q];
            if (lane == 0) nk_si[6] = (int)V;
        } else {
            for (int q = lane; q < T; q += 32) {
                const TriCand cd = k.tscand[q];
                k.tslist[q] = cd;
                hv[q] = cd.value;
                hs[q] = q;
            }
            __syncwarp();
            if (lane == 0)
                for (int q = T / 2 - 1; q >= 0; --q) nk_heap_down(hv, hs, T, q);
            __syncwarp();
            for (long long base = T; base < V; base += 32) {
                const long long idx = base + lane;
                const double v = idx < V ? k.tscand[idx].value : -INFINITY;
                double th = hv[0];
                unsigned mask = __ballot_sync(0xffffffffu, v > th);
                while (mask) {
                    const int l = __ffs(mask) - 1;
                    const double vl = __shfl_sync(0xffffffffu, v, l);
                    __syncwarp();
                    if (lane == 0) {
                        const int sl = hs[0];
                        k.tslist[sl] = k.tscand[base + l];
                        hv[0] = vl;
                        nk_heap_down(hv, hs, T, 0);
                    }
                    __syncwarp();
                    th = hv[0];
                    mask = __ballot_sync(0xffffffffu, lane > l && v > th);
                }
            }
            if (lane == 0) nk_si[6] = T;
        }
    }
    __syncthreads();
    *size = nk_si[6];
    __syncthreads();
    return vmax;
}

// ---------------------------------------------------------------------------
// Cut lists (src/cutting_planes.c:144-206, 224-309, 416-503)
// ---------------------------------------------------------------------------
struct TriEnt {
    uint32_t code;
    double y;
};
struct KEnt {
    unsigned long long key;
    double y;
};

__device__ __forceinline__ unsigned long long kgon_key(int type, const int* perm, int K)
{
    unsigned long long key = (unsigned long long)type;
    for (int a = 0; a < K; ++a) key |= (unsigned long long)(perm[a] & 0xff) << (8 * (a + 1));
    return key;
}

__device__ __forceinline__ uint32_t nk_hash(uint32_t x, uint32_t mask)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x & mask;
}

// purge + separate + append for the triangle list.  y: current duals of
// the triangle cuts.  Returns the maximum violation (viol3).
__device__ __noinline__ double nk_tri_update(const FusedCfg& c, Nk& k, const double* y, int* added, int* subtracted)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int kept = cta_compact<TriEnt>(
        k.mt, [&](int i) { return TriEnt{k.tricode[i], y[i]}; },
        [&](int, const TriEnt& e) { return !(e.y < 1e-5); },
        [&](int pos, const TriEnt& e) {
            k.tricode[pos] = e.code;
            k.triy[pos] = e.y;
        });
    *subtracted = k.mt - kept;
    k.mt = kept;
    int size = 0;
    double mx;
    {
        NkTimer tm(c.prof, NKP_TRISEP);
        mx = nk_trisep(c, k, k.X, &size);
    }
    NkTimer tm2(c.prof, NKP_TRILIST);
    // membership among the kept cuts
    const uint32_t hmask = (uint32_t)c.hash_size - 1u;
    for (int q = tid; q < c.hash_size; q += nt) k.hash[q] = 0xffffffffu;
    __syncthreads();
    for (int q = tid; q < kept; q += nt) {
        const uint32_t code = k.tricode[q];
        uint32_t h = nk_hash(code, hmask);
        for (int probe = 0; probe < c.hash_size; ++probe) {
            const uint32_t old = atomicCAS(&k.hash[h], 0xffffffffu, code);
            if (old == 0xffffffffu || old == code) break;
            h = (h + 1) & hmask;
        }
    }
    __syncthreads();
    const int room = c.mt_cap - kept;
    const int add = cta_compact<uint32_t>(
        size, [&](int q) { return k.tslist[q].code; },
        [&](int, const uint32_t& code) {
            uint32_t h = nk_hash(code, hmask);
            for (int probe = 0; probe < c.hash_size; ++probe) {
                const uint32_t v = k.hash[h];
                if (v == code) return false;
                if (v == 0xffffffffu) return true;
                h = (h + 1) & hmask;
            }
            return true;
        },
        [&](int pos, const uint32_t& code) {
            if (pos < room) {
                k.tricode[kept + pos] = code;
                k.triy[kept + pos] = 0.0;
            }
        });
    if (add > room) k.status |= NKS_CUT_CAP;
    *added = add < room ? add : room;
    k.mt = kept + *added;
    __syncthreads();
    return mx;
}

// purge + separate (annealing chains) + append for the k-gonal list.
template <int K>
__device__ __noinline__ double nk_kgon_update(const FusedCfg& c, Nk& k, const double* y, int* added,
                                 int* subtracted)
{
    double* const smem = nk_smem;
    NkTimer tm(c.prof, NKP_KGON);
    const int tid = threadIdx.x, nt = blockDim.x;
    unsigned long long* keys = K == 5 ? k.pentkey : k.heptkey;
    double* ys = K == 5 ? k.penty : k.hepty;
    int& cnt = K == 5 ? k.mp : k.mh;
    const int capk = K == 5 ? c.mp_cap : c.mh_cap;
    const int kept = cta_compact<KEnt>(
        cnt, [&](int i) { return KEnt{keys[i], y[i]}; }, [&](int, const KEnt& e) { return !(e.y < 1e-5); },
        [&](int pos, const KEnt& e) {
            keys[pos] = e.key;
            ys[pos] = e.y;
        });
    *subtracted = cnt - kept;
    cnt = kept;
    const int n = k.n;
    const int types = K == 5 ? 3 : 4;
    const int trials = K == 5 ? c.Pent_Trials : c.Hepta_Trials;
    const int chains = trials > 0 ? trials * types : 0;
    double mn = NK_BIG;
    int size = 0;
    if (chains > 0 && n >= K) {
        // chains on X in shared memory; permutations interleaved by chain
        const size_t nn = (size_t)n * n;
        constexpr int PS = 256;   // chains per wave
        double* sX = smem;
        double* sT = sX + nn;
        unsigned short* P = (unsigned short*)(sT + 2);
        for (size_t e = tid; e < nn; e += nt) sX[e] = k.X[e];
        __syncthreads();
        if (tid == 0) sT[0] = kgon_temperature(sX, n, K);
        if (tid == 0) nk_si[7] = 0;
        __syncthreads();
        const unsigned long long seed = nk_mix(k.saseed, (unsigned long long)k.sacalls++);
        for (int w0 = 0; w0 < chains; w0 += PS) {
            const int ch = w0 + tid;
            if (tid < PS && ch < chains)
                kgon_chain(sX, n, K, types, ch, seed, sT[0], P, PS, tid, k.sacost, k.saperm, &nk_si[7]);
            __syncthreads();
        }
        // the reference's streaming list in (trial, type) order
        if (tid == 0) {
            int least = 0;
            double least_val = -NK_BIG;
            const int cap = K == 5 ? c.PentIneq : c.HeptaIneq;
            for (int ch = 0; ch < chains; ++ch) {
                const double v = k.sacost[ch];
                const int type = ch % types + 1;
                mn = v < mn ? v : mn;
                if (!(v < 1.0)) continue;
                const unsigned long long key = kgon_key(type, k.saperm + (size_t)ch * 7, K);
                if (size < cap) {
                    k.klist[size] = key;
                    k.klistv[size] = v;
                    if (size == 0 || v > least_val) {
                        least_val = v;
                        least = size;
                    }
                    ++size;
                } else if (v < least_val) {
                    k.klist[least] = key;
                    k.klistv[least] = v;
                    least_val = NK_BIG;
                    for (int q = 0; q < size; ++q)
                        if (k.klistv[q] > least_val) {
                            least_val = k.klistv[q];
                            least = q;
                        }
                }
            }
            nk_sd[4] = mn;
            nk_si[6] = size;
        }
        __syncthreads();
        mn = nk_sd[4];
        size = nk_si[6];
        __syncthreads();
    }
    const int room = capk - kept;
    const int add = cta_compact<unsigned long long>(
        size, [&](int q) { return k.klist[q]; },
        [&](int, const unsigned long long& key) {
            for (int q = 0; q < kept; ++q)
                if (keys[q] == key) return false;
            return true;
        },
        [&](int pos, const unsigned long long& key) {
            if (pos < room) {
                keys[kept + pos] = key;
                ys[kept + pos] = 0.0;
            }
        });
    if (add > room) k.status |= NKS_CUT_CAP;
    *added = add < room ? add : room;
    cnt = kept + *added;
    __syncthreads();
    return mn;
}

// Packed records [tri | pent | hept] and the pair CSR of B^T in cut order.
__device__ __noinline__ void nk_upload_cuts(const FusedCfg& c, Nk& k)
{
    NkTimer tm(c.prof, NKP_CUTS);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int m = k.mt + k.mp + k.mh;
    const int n = k.n;
    for (int q = tid; q < m; q += nt) {
        CutRec r;
        if (q < k.mt) {
            int t, i, j, kk;
            tri_decode(k.tricode[q], &t, &i, &j, &kk);
            const int p[3] = {i, j, kk};
            r = pack_cut(3, p, tri_negmask(t));
        } else {
            const bool pent = q < k.mt + k.mp;
            const unsigned long long key = pent ? k.pentkey[q - k.mt] : k.heptkey[q - k.mt - k.mp];
            const int K = pent ? 5 : 7;
            int p[7];
            for (int a = 0; a < K; ++a) p[a] = (int)((key >> (8 * (a + 1))) & 0xff);
            const int t = (int)(key & 0xff);
            r = pack_cut(K, p, pent ? pent_negmask(t) : hept_negmask(t));
        }
        k.rec[q] = r;
    }
    const long long P = (long long)n * (n - 1) / 2;
    for (long long q = tid; q <= P; q += nt) {
        k.csroff[q] = 0u;
        if (q < P) k.csrcur[q] = 0u;
    }
    __syncthreads();
    auto pidx = [](unsigned u, unsigned v) {
        const unsigned a = u < v ? u : v, b = u < v ? v : u;
        return (long long)b * (b - 1) / 2 + a;
    };
    for (int q = tid; q < m; q += nt) {
        const CutRec r = k.rec[q];
        const unsigned p[7] = {r.x & 0xffffu, r.x >> 16, r.y & 0xffffu, r.y >> 16, r.z & 0xffffu, r.z >> 16,
                               r.w & 0xffffu};
        const int K = (int)((r.w >> 16) & 0xffu);
        for (int a = 0; a < K; ++a)
            for (int b = a + 1; b < K; ++b) atomicAdd(&k.csroff[pidx(p[a], p[b])], 1u);
    }
    __syncthreads();
    cta_scan_u32(k.csroff, P + 1);
    for (int q = tid; q < m; q += nt) {
        const CutRec r = k.rec[q];
        const unsigned p[7] = {r.x & 0xffffu, r.x >> 16, r.y & 0xffffu, r.y >> 16, r.z & 0xffffu, r.z >> 16,
                               r.w & 0xffffu};
        const int K = (int)((r.w >> 16) & 0xffu);
        const unsigned neg = (r.w >> 24) & 0x7fu;
        for (int a = 0; a < K; ++a)
            for (int b = a + 1; b < K; ++b) {
                const long long pi = pidx(p[a], p[b]);
                const unsigned pos = atomicAdd(&k.csrcur[pi], 1u);
                const unsigned sneg = ((neg >> a) ^ (neg >> b)) & 1u;
                k.contrib[k.csroff[pi] + pos] = ((uint32_t)q << 1) | sneg;
            }
    }
    __syncthreads();
    // every pair's contributions into cut order (short segments)
    for (long long q = tid; q < P; q += nt) {
        const unsigned b = k.csroff[q], e = k.csroff[q + 1];
        for (unsigned i = b + 1; i < e; ++i) {
            const uint32_t v = k.contrib[i];
            unsigned j = i;
            while (j > b && k.contrib[j - 1] > v) {
                k.contrib[j] = k.contrib[j - 1];
                --j;
            }
            k.contrib[j] = v;
        }
    }
    __syncthreads();
}

// L0 = L - B^T(t)
__device__ __noinline__ void nk_opBt(const FusedCfg&, Nk& k, const double* t)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = k.n;
    const size_t nn = (size_t)n * n;
    for (size_t e = tid; e < nn; e += nt) k.L0[e] = k.L[e];
    __syncthreads();
    const long long P = (long long)n * (n - 1) / 2;
    const int m_tp = k.mt + k.mp;
    for (long long q = tid; q < P; q += nt) {
        const unsigned b = k.csroff[q], e = k.csroff[q + 1];
        if (b == e) continue;
        int v = (int)floor((1.0 + sqrt(1.0 + 8.0 * (double)q)) * 0.5);
        while ((long long)v * (v - 1) / 2 > q) --v;
        while ((long long)(v + 1) * v / 2 <= q) ++v;
        const int u = (int)(q - (long long)v * (v - 1) / 2);
        const size_t e1 = u + (size_t)v * n, e2 = v + (size_t)u * n;
        double x1 = k.L0[e1], x2 = k.L0[e2];
        pair_apply(k.contrib, b, e, k.mt, m_tp, t, &x1, &x2);
        k.L0[e1] = x1;
        k.L0[e2] = x2;
    }
    __syncthreads();
}

// G[:, s_j] = 1 - B(Xb[s_j]) for the slots s_j = slot[j] (or *slot_ptr).
__device__ __noinline__ void nk_opB(Nk& k, const int* slots, int ncols)
{
    const int m = k.mt + k.mp + k.mh;
    const size_t nn = (size_t)k.n * k.n;
    const long long tot = (long long)m * ncols;
    for (long long q = threadIdx.x; q < tot; q += blockDim.x) {
        const int cidx = (int)(q % m), j = (int)(q / m);
        const int s = slots[j];
        k.G[cidx + (size_t)s * k.ldg] = cut_apply(k.rec[cidx], k.Xb + (size_t)s * nn, k.n, 1.0);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Bundle (the engine's bodies)
// ---------------------------------------------------------------------------
__device__ __noinline__ void nk_lambda_eta(LeArgs a) { lambda_eta_body(a, nk_smem); }
__device__ __noinline__ void nk_step(StepArgs a) { bundle_step_body(a); }

__device__ void nk_bundle_iterations(const FusedCfg& c, Nk& k, int bdl_iter)
{
    const int m = k.mt + k.mp + k.mh;
    const size_t nn = (size_t)k.n * k.n;
    for (int it = 0; it < bdl_iter; ++it) {
        LeArgs a{k.G, k.ldg, k.slot, m, nullptr, k.Fv, k.gam, k.lam, k.eta, k.dgam, k.gtest, k.dstate, k.istate,
                 k.qpws, -1, c.le_prof};
        {
            NkTimer tm(c.prof, NKP_LAMBDA);
            nk_lambda_eta(a);
        }
        __syncthreads();
        {
            NkTimer tm(c.prof, NKP_OPBT);
            nk_opBt(c, k, k.gtest);
        }
        if (!nk_ipm(c, k, k.L0, k.Xb, k.istate + BI_NEXT)) return;
        if (m > 0) {
            NkTimer tm(c.prof, NKP_OPB);
            nk_opB(k, k.istate + BI_NEXT, 1);
        }
        NkTimer tms(c.prof, NKP_STEP);
        StepArgs s{k.G, k.ldg, m, k.n, c.bcap, k.L, k.Xb, k.out, k.Fv, k.slot, k.slot_old, k.lam, k.gam,
                   k.gtest, k.dstate, k.istate};
        nk_step(s);
        __syncthreads();
        bundle_xcomb_body(k.Xb, k.slot_old, k.lam, k.istate, k.X, nn, threadIdx.x, blockDim.x);
        __syncthreads();
        const int err = k.istate[BI_ERR];
        __syncthreads();
        if (err) {
            if (err & 2) k.status |= NKS_QP;
            if (err & (1 | 8)) k.status |= NKS_BUNDLE_CAP;
            if (err & 4) k.status |= NKS_IPM;
            return;
        }
    }
}

// ---------------------------------------------------------------------------
// Learned warm start (warm.h): the network's proposal for the first-
// separation cuts, evaluated once (L0 = L - B^T(gamma_w), one IPM into
// bundle slot 0); kept, as the bundle's starting multipliers and X, when its
// dual value is below f (the plain start's).  Returns the starting f.
// ---------------------------------------------------------------------------
__device__ __noinline__ double nk_warm(const FusedCfg& c, Nk& k, double viol3, double gap, double f)
{
    const __nv_bfloat16* P = (const __nv_bfloat16*)c.warm_p;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = k.n, m = k.mt;
    const size_t nn = (size_t)n * n;
    // the objective's scale: mean |L_ij| over i != j
    double a = 0.0;
    for (size_t e = tid; e < nn; e += nt)
        if (e % n != e / n) a += fabs(k.L[e]);
    a = block_sum(a, nk_red);
    const double sc = (n > 1 && a > 0.0) ? a / ((double)n * (n - 1)) : 1.0;
    double sg = 0.0;
    for (int q = tid; q < m; q += nt) {
        int type, i, j, kk;
        tri_decode(k.tricode[q], &type, &i, &j, &kk);
        const double xij = k.X[i + (size_t)j * n], xik = k.X[i + (size_t)kk * n], xjk = k.X[j + (size_t)kk * n];
        // the cut's violation as src/cutting_planes.c:20-39 evaluates it
        const double v = type == 1   ? -xij - xik - xjk - 1.0
                         : type == 2 ? -xij + xik + xjk - 1.0
                         : type == 3 ? xij - xik + xjk - 1.0
                                     : xij + xik - xjk - 1.0;
        float xf[WARM_F];
        warm_cut_features(type, i, j, kk, v, k.X, k.L, n, m, viol3, gap, sc, -1.0, xf);
        const double g = sc * (double)warm_mlp_bf16(xf, P);
        k.gtest[q] = g;
        sg += g;
    }
    sg = block_sum(sg, nk_red);
    nk_opBt(c, k, k.gtest);
    const int st0 = k.status;
    const bool ok = nk_ipm(c, k, k.L0, k.Xb, nullptr);
    const double fw = ok ? k.out[0] + sg : 0.0;
    __syncthreads();
    k.status = st0;   // a failed proposal is only rejected
    const bool keep = ok && fw < f;
    if (keep) {
        for (int q = tid; q < m; q += nt) k.gam[q] = k.gtest[q];
        for (size_t e = tid; e < nn; e += nt) k.X[e] = k.Xb[e];
    }
    __syncthreads();
    if (tid == 0 && c.warm_stats) atomicAdd(&c.warm_stats[keep ? 0 : 1], 1ull);
    return keep ? fw : f;
}

// ---------------------------------------------------------------------------
// One node: SDPbound (src/bounding.c:24-342)
// ---------------------------------------------------------------------------
__device__ double nk_bound(const FusedCfg& c, Nk& k)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = k.n;
    const size_t nn = (size_t)n * n;
    int bdl_iter = c.init_bundle_iter;
    k.mt = k.mp = k.mh = 0;
    int tri_add = 0, tri_sub = 0, pent_add = 0, pent_sub = 0, hept_add = 0, hept_sub = 0;
    double viol3 = 0.0, viol5 = 0.0;

    if (!nk_ipm(c, k, k.L, k.X, nullptr)) return 0.0;
    double f = k.out[0];
    const double basic_bound = f + k.fixedvalue;
    nk_fracsol(c, k);
    nk_heuristic(c, k);
    if (k.status) return 0.0;

    double bound = f + k.fixedvalue;
    double lb = nk_lb(c);
    if (bound < lb + 1.0) return bound;
    if (c.use_diff && c.rank != 0 && bound > lb + c.diff + 1.0) return bound;

    viol3 = nk_tri_update(c, k, k.gam, &tri_add, &tri_sub);
    if (k.status) return 0.0;
    // no violated triangle inequality: the basic bound is the node's bound
    // (the reference's bundle start divides by the cut count)
    if (k.mt == 0) return bound;
    // dual_gamma = the cuts' y (0 for the new ones)
    for (int i = tid; i < k.mt; i += nt) k.gam[i] = k.triy[i];
    lb = nk_lb(c);
    double t = 0.5 * (bound - lb) / (k.mt * viol3 * viol3);

    // bundle: X_bundle(0) = X, G(:,0) = 1 - B(X), F(0) = <L,X>, bundle = 1
    nk_upload_cuts(c, k);
    if (1 + bdl_iter + 2 > c.bcap) {
        k.status |= NKS_BUNDLE_CAP;
        return 0.0;
    }
    if (c.warm_p) f = nk_warm(c, k, viol3, bound - lb, f);
    for (size_t e = tid; e < nn; e += nt) k.Xb[e] = k.X[e];
    if (tid < BI_WORDS) k.istate[tid] = 0;
    __syncthreads();
    if (tid == 0) k.istate[BI_CAP] = c.bcap;
    __syncthreads();
    if (k.mt + k.mp + k.mh > 0) nk_opB(k, k.istate + BI_NEXT, 1);
    bundle_fval_body(k.L, k.Xb, n, k.istate + BI_NEXT, k.istate + BI_K, k.Fv);
    __syncthreads();
    bundle_append_body(k.slot, k.istate, c.bcap);
    __syncthreads();
    if (tid == 0) {
        k.dstate[BD_F] = f;
        k.dstate[BD_T] = t;
        k.dstate[BD_FTEST] = 0.0;
        k.dstate[BD_DEL] = 0.0;
    }
    __syncthreads();

    int count = 0;
    bool done = false, prune = false, giveup = false;
    while (!done) {
        ++count;
        const double oldf = f;
        if (k.istate[BI_K] + bdl_iter + 2 > c.bcap) {
            k.status |= NKS_BUNDLE_CAP;
            return 0.0;
        }
        nk_bundle_iterations(c, k, bdl_iter);
        if (k.status) return 0.0;
        f = k.dstate[BD_F];
        t = k.dstate[BD_T];
        __syncthreads();
        bound = f + k.fixedvalue;
        lb = nk_lb(c);
        prune = bound < lb + 1.0;
        if (!prune) {
            nk_heuristic(c, k);
            if (k.status) return 0.0;
            lb = nk_lb(c);
            prune = bound < lb + 1.0;
        }
        const double gap = bound - lb;
        if (count == c.triag_iter + c.pent_iter + c.hept_iter)
            if (gap - 1.0 > (oldf - f) * (c.max_outer_iter - count)) giveup = true;
        if (count == c.max_outer_iter)
            if (gap - 1.0 > (oldf - f) * c.extra_iter) giveup = true;
        if (count == c.max_outer_iter + c.extra_iter) giveup = true;

        if (!prune && !giveup) {
            const int triag = k.mt;
            const int penta = k.mp;
            viol3 = nk_tri_update(c, k, k.gam, &tri_add, &tri_sub);
            if (k.status) return 0.0;
            const bool do_pent = c.include_Pent && (count > c.triag_iter || viol3 < 0.2);
            if (do_pent) {
                viol5 = nk_kgon_update<5>(c, k, k.gam + triag, &pent_add, &pent_sub);
                if (k.status) return 0.0;
            }
            if (c.include_Hepta &&
                ((count > c.triag_iter + c.pent_iter) || (viol3 < 0.2 && (1 - viol5 < 0.4)))) {
                nk_kgon_update<7>(c, k, k.gam + triag + penta, &hept_add, &hept_sub);
                if (k.status) return 0.0;
            }
        } else {
            tri_add = tri_sub = pent_add = pent_sub = hept_add = hept_sub = 0;
        }
        // no cuts left: the bundle cannot move (the reference's bundle
        // calls BLAS with m = 0 there, which is undefined); stop here
        done = prune || giveup || k.mt + k.mp + k.mh == 0;
        nk_fracsol(c, k);

        if (!done) {
            const int m = k.mt + k.mp + k.mh;
            for (int i = tid; i < m; i += nt)
                k.gam[i] = i < k.mt ? k.triy[i] : (i < k.mt + k.mp ? k.penty[i - k.mt] : k.hepty[i - k.mt - k.mp]);
            __syncthreads();
            nk_upload_cuts(c, k);
            const int kb = k.istate[BI_K];
            __syncthreads();
            if (kb + 2 + bdl_iter + 2 > c.bcap) {
                k.status |= NKS_BUNDLE_CAP;
                return 0.0;
            }
            // fct_eval(PP, dual_gamma, X_test, g) into the free slot
            {
                NkTimer tm(c.prof, NKP_OPBT);
                nk_opBt(c, k, k.gam);
            }
            if (!nk_ipm(c, k, k.L0, k.Xb, k.istate + BI_NEXT)) return 0.0;
            if (m > 0) {
                nk_opB(k, k.slot, kb);
                nk_opB(k, k.istate + BI_NEXT, 1);
            }
            bundle_fval_body(k.L, k.Xb, n, k.istate + BI_NEXT, k.istate + BI_K, k.Fv);
            __syncthreads();
            bundle_append_body(k.slot, k.istate, c.bcap);
            __syncthreads();
            if (k.istate[BI_ERR] & (1 | 8)) {
                k.status |= NKS_BUNDLE_CAP;
                return 0.0;
            }
            t *= 1.05;
            if (tid == 0) k.dstate[BD_T] = t;
            __syncthreads();
        }
        bdl_iter += count % 2;
        bdl_iter = (bdl_iter < c.max_bundle_iter) ? bdl_iter : c.max_bundle_iter;
    }
    (void)basic_bound;
    return f + k.fixedvalue;
}

// Bound node `node` of the launch's arrays in this CTA's slot.
__device__ double nk_run_node(const FusedCfg& c, Nk& k, int node)
{
    const unsigned long long t_node = threadIdx.x == 0 ? nk_now() : 0ull;
    k.node = node;
    k.xf = c.xfixed + (size_t)node * k.N;
    k.sx = c.solx + (size_t)node * k.N;
    k.status = 0;
    k.best_h = -NK_BIG;
    k.hseed = nk_mix(c.seed, 2ull * node + 1ull);
    k.saseed = nk_mix(c.seed, 2ull * node + 2ull);
    k.hctr = 0;
    k.sacalls = 0;
    if (threadIdx.x == 0) c.hval[node] = -NK_BIG;
    __syncthreads();
    nk_subproblem(c, k);
    double b = 0.0;
    if (k.n > NK_NMAX)
        k.status |= NKS_SIZE;
    else
        b = nk_bound(c, k);
    __syncthreads();
    if (threadIdx.x == 0) {
        c.bound[node] = b;
        c.status[node] = k.status;
        c.node_ns[node] = nk_now() - t_node;
    }
    __syncthreads();
    return b;
}

// ---------------------------------------------------------------------------
// Device-resident node pool (src/heap.c:27-133, src/bab_functions.c:224-336
// on the device): a max-heap of open nodes keyed on the parent's bound,
// behind a lock that thread 0 of a CTA takes with a bounded wait.
// ---------------------------------------------------------------------------
constexpr unsigned long long NKQ_LOCK_NS = 1000000000ull;    // 1 s
constexpr unsigned long long NKQ_IDLE_NS = 20000000000ull;   // 20 s without work: the CTA leaves

__device__ bool nkq_lock(const FusedCfg& c)
{
    const unsigned long long t0 = nk_now();
    while (atomicCAS(&c.pstate[NKQ_LOCK], 0, 1) != 0) {
        if (nk_now() - t0 > NKQ_LOCK_NS) {
            atomicOr(&c.pstate[NKQ_ERROR], 1);
            return false;
        }
        __nanosleep(64);
    }
    __threadfence();
    return true;
}

__device__ void nkq_unlock(const FusedCfg& c)
{
    __threadfence();
    atomicExch(&c.pstate[NKQ_LOCK], 0);
}

// (lock held) push node q
__device__ void nkq_push(const FusedCfg& c, int q)
{
    volatile int* st = c.pstate;
    int i = st[NKQ_SIZE];
    const double v = c.ub[q];
    while (i > 0) {
        const int p = (i - 1) >> 1;
        if (!(((volatile double*)c.ub)[c.heap[p]] < v)) break;
        c.heap[i] = c.heap[p];
        i = p;
    }
    c.heap[i] = q;
    st[NKQ_SIZE] = st[NKQ_SIZE] + 1;
}

// (lock held) pop the open node with the largest parent bound
__device__ int nkq_pop(const FusedCfg& c)
{
    volatile int* st = c.pstate;
    const volatile double* ub = c.ub;
    const int size = st[NKQ_SIZE] - 1;
    const int top = c.heap[0];
    const int last = c.heap[size];
    st[NKQ_SIZE] = size;
    int i = 0;
    while (true) {
        int ch = 2 * i + 1;
        if (ch >= size) break;
        if (ch + 1 < size && ub[c.heap[ch + 1]] > ub[c.heap[ch]]) ++ch;
        if (!(ub[c.heap[ch]] > ub[last])) break;
        c.heap[i] = c.heap[ch];
        i = ch;
    }
    if (size > 0) c.heap[i] = last;
    return top;
}

// Thread 0: the next node to bound, -1 when the pool is finished (no open
// node and no CTA working), the deadline passed, or this CTA waited
// NKQ_IDLE_NS without work (the others go on).  Open nodes whose parent bound
// no longer exceeds the incumbent by more than 1 are dropped unbounded.
__device__ int nkq_next(const FusedCfg& c)
{
    const unsigned long long t0 = nk_now();
    volatile int* st = c.pstate;
    while (true) {
        if (st[NKQ_ERROR]) return -1;
        if (c.deadline && nk_now() > *c.deadline) {
            atomicExch(&c.pstate[NKQ_STOPPED], 1);
            return -1;
        }
        if (!nkq_lock(c)) return -1;
        const double lb = ordered_to_dbl(*(volatile unsigned long long*)c.lb);
        int node = -1;
        while (st[NKQ_SIZE] > 0) {
            const int q = nkq_pop(c);
            if (lb + 1.0 < ((volatile double*)c.ub)[q]) {
                node = q;
                break;
            }
            st[NKQ_PRUNED] = st[NKQ_PRUNED] + 1;
        }
        if (node >= 0) {
            st[NKQ_ACTIVE] = st[NKQ_ACTIVE] + 1;
            nkq_unlock(c);
            return node;
        }
        const bool finished = st[NKQ_ACTIVE] == 0;
        nkq_unlock(c);
        if (finished || nk_now() - t0 > NKQ_IDLE_NS) return -1;
        __nanosleep(2000);
    }
}

// After bounding `node` (bound b): hand a flagged node to the host, or
// branch on the variable getBranchingVariable picks (src/bab_functions.c:
// 387-423) when the bound exceeds the incumbent by more than 1 and push both
// children with b as their priority; then leave the active count.
__device__ void nkq_finish(const FusedCfg& c, Nk& k, int node, double b)
{
    __shared__ int s_ic, s_base;
    const int N = k.N;
    const bool flagged = c.status[node] != 0;
    const double lb = nk_lb(c);
    const bool branch = !flagged && lb + 1.0 < b;
    if (threadIdx.x == 0) {
        s_ic = -1;
        s_base = -1;
        if (flagged) {
            const int h = atomicAdd(&c.pstate[NKQ_HOST], 1);
            if (h < c.pool_cap) c.host_list[h] = node;
            else atomicOr(&c.pstate[NKQ_ERROR], 2);
        } else if (branch) {
            const double* fs = c.fracsol + (size_t)node * N;
            int ic = -1;
            double best = c.branching == 0 ? -NK_BIG : NK_BIG;
            for (int i = 0; i < N; ++i) {
                if (k.xf[i]) continue;
                const double d = fabs(0.5 - fs[i]);
                if (c.branching == 0 ? d > best : d < best) {
                    best = d;
                    ic = i;
                }
            }
            s_ic = ic;
            if (ic >= 0) {
                const int base = atomicAdd(&c.pstate[NKQ_CREATED], 2);
                if (base + 2 <= c.pool_cap) s_base = base;
                else atomicOr(&c.pstate[NKQ_ERROR], 2);
            }
        }
    }
    __syncthreads();
    const int ic = s_ic, base = s_base;
    if (base >= 0) {
        for (int i = threadIdx.x; i < 2 * N; i += blockDim.x) {
            const int ch = i / N, v = i % N;
            int* xf = (int*)c.xfixed + (size_t)(base + ch) * N;
            int* sx = (int*)c.solx + (size_t)(base + ch) * N;
            xf[v] = v == ic ? 1 : k.xf[v];
            sx[v] = v == ic ? ch : k.sx[v];
        }
        if (threadIdx.x < 2) {
            c.ub[base + threadIdx.x] = b;
            c.hval[base + threadIdx.x] = -NK_BIG;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&c.pstate[NKQ_EVALUATED], 1);
        __threadfence();
        if (nkq_lock(c)) {
            if (base >= 0) {
                nkq_push(c, base);
                nkq_push(c, base + 1);
            }
            c.pstate[NKQ_ACTIVE] = ((volatile int*)c.pstate)[NKQ_ACTIVE] - 1;
            nkq_unlock(c);
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(NKT, 1) nodek_kernel(FusedCfg c)
{
    Nk k;
    nk_bind(c, k, blockIdx.x);
    k.N0 = c.N0;
    k.N = c.N0 - 1;
    while (true) {
        int node = 0;
        if (threadIdx.x == 0) {
            if (c.pool) {
                node = nkq_next(c);
            } else {
                const int q = atomicAdd(c.next, 1);
                node = q < c.count ? c.order[q] : -1;
            }
        }
        node = bcast_i(node);
        if (node < 0) break;
        const double b = nk_run_node(c, k, node);
        if (c.pool) nkq_finish(c, k, node, b);
    }
}

}  // namespace

size_t nk_smem_bytes(int N0, int T, int bcap, size_t smem_optin)
{
    const size_t n = (size_t)N0, nn = n * n, nv = (n + 1) & ~(size_t)1;
    size_t need = 0;
    auto up = [&](size_t b) { need = b > need ? b : need; };
    // IPM: fixed part + F, and Zi too when both fit (as the engine places them)
    const size_t ipm1 = (ipm_reg_fixed_smem_doubles(N0) + nn) * sizeof(double);
    up(ipm1 + nn * sizeof(double) <= smem_optin ? ipm1 + nn * sizeof(double) : ipm1);
    // lambda_eta
    up(le_smem_bytes(bcap < QP_SMEM_K ? bcap : QP_SMEM_K) + 3 * (size_t)bcap * sizeof(double));
    // heuristic: Z, column buffer, d, 16 warps x (Lx, x)
    up((nn + 2 * nv + (size_t)(NKT / 32) * 2 * nv) * sizeof(double));
    // triangle separation: X^T, then the heap
    up(nn * sizeof(double));
    up((size_t)(T > 0 ? T : 1) * (sizeof(double) + sizeof(int)) + 16);
    // annealing chains: X, temperature, 256 permutations
    up((nn + 2) * sizeof(double) + n * 256 * sizeof(unsigned short));
    return (need + 255) & ~(size_t)255;
}

size_t nk_layout(FusedCfg& c)
{
    const size_t n = (size_t)c.N0, nn = n * n, N = n - 1;
    const size_t P = n * (n - 1) / 2, C3 = n * (n - 1) * (n - 2) / 6;
    const size_t M = (size_t)c.mt_cap + c.mp_cap + c.mh_cap;
    const size_t num = n;
    size_t sz[NK_COUNT];
    sz[NK_L] = nn * 8;
    sz[NK_L0] = nn * 8;
    sz[NK_X] = nn * 8;
    sz[NK_IPMWS] = 3 * nn * 8;
    sz[NK_OUT] = 8 * 8;
    sz[NK_XB] = (size_t)c.bcap * nn * 8;
    sz[NK_G] = M * c.bcap * 8;
    sz[NK_FV] = (size_t)c.bcap * 8;
    sz[NK_LAM] = (size_t)c.bcap * 8;
    sz[NK_GAM] = M * 8;
    sz[NK_GTEST] = M * 8;
    sz[NK_DGAM] = M * 8;
    sz[NK_ETA] = M * 8;
    sz[NK_DSTATE] = 8 * 8;
    sz[NK_QPWS] = (2 * (size_t)c.bcap * c.bcap + 8 * (size_t)c.bcap + 8) * 8;
    sz[NK_SLOT] = (size_t)c.bcap * 4;
    sz[NK_SLOTOLD] = (size_t)c.bcap * 4;
    sz[NK_ISTATE] = 8 * 4;
    sz[NK_TRICODE] = (size_t)c.mt_cap * 4;
    sz[NK_TRIY] = (size_t)c.mt_cap * 8;
    sz[NK_PENTKEY] = (size_t)c.mp_cap * 8;
    sz[NK_PENTY] = (size_t)c.mp_cap * 8;
    sz[NK_HEPTKEY] = (size_t)c.mh_cap * 8;
    sz[NK_HEPTY] = (size_t)c.mh_cap * 8;
    sz[NK_REC] = M * sizeof(CutRec);
    sz[NK_CSROFF] = (P + 1) * 4;
    sz[NK_CSRCUR] = P * 4;
    sz[NK_CONTRIB] = ((size_t)3 * c.mt_cap + 10 * (size_t)c.mp_cap + 21 * (size_t)c.mh_cap) * 4;
    sz[NK_HASH] = (size_t)c.hash_size * 4;
    sz[NK_TSCNT] = 4 * P * 4;
    sz[NK_TSCAND] = 4 * C3 * sizeof(TriCand);
    sz[NK_TSLIST] = (size_t)(c.TriIneq > 0 ? c.TriIneq : 1) * sizeof(TriCand);
    sz[NK_SACOST] = (size_t)(c.sa_chains > 0 ? c.sa_chains : 1) * 8;
    sz[NK_SAPERM] = (size_t)(c.sa_chains > 0 ? c.sa_chains : 1) * 7 * 4;
    sz[NK_KLIST] = (size_t)(c.sa_chains > 0 ? c.sa_chains : 1) * 8;
    sz[NK_KLISTV] = (size_t)(c.sa_chains > 0 ? c.sa_chains : 1) * 8;
    sz[NK_HZ] = nn * 8;
    sz[NK_HV] = num * n * 8;
    sz[NK_HX] = num * n * 4;
    sz[NK_HVAL] = num * 8;
    sz[NK_HSOL] = num * N * 4;
    sz[NK_HBEST] = N * 4;
    sz[NK_XH] = n * 8;
    sz[NK_FREE] = N * 4;
    sz[NK_FIXED] = N * 4;
    size_t off = 0;
    for (int a = 0; a < NK_COUNT; ++a) {
        c.off[a] = off;
        off += (sz[a] + 255) & ~(size_t)255;
    }
    c.slot_bytes = off;
    return off;
}

namespace {
__global__ void nk_deadline_kernel(unsigned long long* out, unsigned long long budget_ns)
{
    *out = nk_now() + budget_ns;
}
}  // namespace

void nk_deadline(unsigned long long* out, unsigned long long budget_ns, cudaStream_t s)
{
    nk_deadline_kernel<<<1, 1, 0, s>>>(out, budget_ns);
    BQB_COUNT_LAUNCH();
    check_launch("nk_deadline_kernel");
}

void nk_launch(const FusedCfg& cfg, int slots, cudaStream_t s)
{
    BQB_SMEM_LIMIT(nodek_kernel, cfg.smem_bytes);
    nodek_kernel<<<slots, NKT, cfg.smem_bytes, s>>>(cfg);
    BQB_COUNT_LAUNCH();
    check_launch("nodek_kernel");
}

}  // namespace bqb
