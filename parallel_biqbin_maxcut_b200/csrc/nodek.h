// Fused node bounding: one CTA bounds a whole B&B node on the device.
#pragma once
#include <stdint.h>

#include <vector>

#include "bqb_common.cuh"

namespace bqb {

// Arrays of one CTA's slot in the fused kernel's arena (byte offsets in
// FusedCfg::off).
enum NkArray : int {
    NK_L, NK_L0, NK_X, NK_IPMWS, NK_OUT, NK_XB, NK_G, NK_FV, NK_LAM, NK_GAM, NK_GTEST, NK_DGAM, NK_ETA,
    NK_DSTATE, NK_QPWS, NK_SLOT, NK_SLOTOLD, NK_ISTATE,
    NK_TRICODE, NK_TRIY, NK_PENTKEY, NK_PENTY, NK_HEPTKEY, NK_HEPTY, NK_REC,
    NK_CSROFF, NK_CSRCUR, NK_CONTRIB, NK_HASH,
    NK_TSCNT, NK_TSCAND, NK_TSLIST,
    NK_SACOST, NK_SAPERM, NK_KLIST, NK_KLISTV,
    NK_HZ, NK_HV, NK_HX, NK_HVAL, NK_HSOL, NK_HBEST, NK_XH, NK_FREE, NK_FIXED,
    NK_COUNT
};

// Per-node status bits of the fused kernel.  A node with any bit set is
// bounded again by an engine on the host (bqb_bound_nodes), which either
// handles the case (capacities) or reports the reference's error.
enum NkStatus : int {
    NKS_BUNDLE_CAP = 1,    // more bundle elements than the slot holds
    NKS_CUT_CAP = 2,       // more cuts than the slot holds
    NKS_QP = 4,            // lambda_eta / solve_lambda failure
    NKS_IPM = 8,           // IPM failure
    NKS_HEUR = 16,         // heuristic Cholesky failure or 1-opt overflow
    NKS_SIZE = 32,         // subproblem too large for the fused kernel
};

// Words of the device node pool's state (FusedCfg::pstate).
enum NkPoolWord : int {
    NKQ_LOCK,        // heap lock
    NKQ_SIZE,        // open nodes in the heap
    NKQ_CREATED,     // node records in use
    NKQ_ACTIVE,      // CTAs bounding a node
    NKQ_ERROR,       // bit 1: a lock wait ran out; bit 2: the pool is full
    NKQ_EVALUATED,   // nodes bounded on the device
    NKQ_HOST,        // nodes handed back to the host (host_list entries)
    NKQ_PRUNED,      // open nodes dropped unbounded (parent bound <= incumbent + 1)
    NKQ_STOPPED,     // the deadline passed
    NKQ_WORDS
};

// Phases timed inside the fused kernel (globaltimer, thread 0 of each CTA).
enum NkPhase : int {
    NKP_SUB, NKP_IPM, NKP_HEUR, NKP_TRISEP, NKP_TRILIST, NKP_KGON, NKP_CUTS, NKP_OPBT, NKP_OPB, NKP_LAMBDA,
    NKP_STEP, NKP_COUNT
};

struct FusedCfg {
    // problem
    const double* P0L;   // SP->L, N0 x N0
    int N0;
    int count;           // nodes in this launch
    int rank;
    double diff;
    // reference parameters (src/biqbin.h:49-84)
    int init_bundle_iter, max_bundle_iter, triag_iter, pent_iter, hept_iter, max_outer_iter, extra_iter;
    double violated_TriIneq;
    int TriIneq, PentIneq, HeptaIneq, Pent_Trials, Hepta_Trials, include_Pent, include_Hepta, use_diff;
    unsigned long long seed;
    // slot capacities
    int bcap;            // bundle slots (physical)
    int mt_cap, mp_cap, mh_cap;
    int hash_size;       // power of two >= 2 mt_cap
    int sa_chains;       // max(Pent_Trials * 3, Hepta_Trials * 4)
    size_t smem_bytes;   // dynamic shared memory of the launch
    // node I/O (device)
    const int* xfixed;   // count x (N0 - 1)
    const int* solx;     // count x (N0 - 1)
    double* bound;       // count
    double* fracsol;     // count x (N0 - 1)
    double* hval;        // count: best value the node's heuristic calls reported
    int* hsol;           // count x (N0 - 1): its 0/1 solution
    int* status;         // count
    unsigned long long* node_ns;   // count: device time of each node's bound
    const int* order;    // count: the order in which CTAs take the nodes
    int* next;           // node counter
    unsigned long long* lb;   // incumbent, order-preserving bits of a double
    double* ipm_stats;
    unsigned long long* prof;   // NKP_COUNT phase times (ns, summed over CTAs)
    unsigned long long* le_prof;   // (may be null) lambda_eta counters, as the engines' (bqb_lambda_eta_profile)
    // learned warm start (warm.h): BF16 weights (null: off) and the
    // {kept, rejected} proposal counters
    const void* warm_p;
    unsigned long long* warm_stats;
    // device-resident node pool (pool != 0): the CTAs pop the open node with
    // the largest parent bound, bound it, branch it on the device and push
    // its children, until no node is open and no CTA is working.  The node
    // I/O arrays above are then indexed by pool node (pool_cap records).
    int pool;
    int pool_cap;
    int branching;          // params.branchingStrategy (0 least, 1 most fractional)
    int* heap;              // pool_cap node indices, a max-heap on ub
    double* ub;             // pool_cap: the parent's bound of each node
    int* pstate;            // NKQ_* words
    int* host_list;         // pool_cap: nodes the kernel hands back to the host
    const unsigned long long* deadline;   // globaltimer value after which no node is popped (null: none)
    // slot arena
    unsigned char* arena;
    size_t slot_bytes;
    size_t off[NK_COUNT];
};

// Largest N0 the fused kernel handles (register-resident IPM).
constexpr int NK_NMAX = 128;

// Shared-memory bytes the fused kernel needs for problems up to N0 with
// TriIneq = T and bcap bundle slots.
size_t nk_smem_bytes(int N0, int T, int bcap, size_t smem_optin);

// Lay out the arena: fills cfg.off and cfg.slot_bytes from the capacities
// in cfg; returns the bytes of one slot.
size_t nk_layout(FusedCfg& cfg);

void nk_launch(const FusedCfg& cfg, int slots, cudaStream_t s);
// *out = the device's globaltimer + budget_ns (the pool's deadline).
void nk_deadline(unsigned long long* out, unsigned long long budget_ns, cudaStream_t s);

}  // namespace bqb
