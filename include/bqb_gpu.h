/*
 * bqb_gpu.h -- C ABI of libbqb_gpu.so, the B200 implementation of BiqBin's
 * per-node SDP bounding path.
 *
 * Part 1 (drop-in): the exact entry points the reference's host code
 * (bounding.c, bundle.c's callers, bab_functions.c, evaluate.c, the pybind
 * bridge) calls today.  Signatures, argument meaning, global-state contract
 * and fatal-error behaviour follow the reference declarations cited beside
 * each.  Linking the reference's host objects against this library instead
 * of ipm_mc_pk.c, bundle.c, operators.c, cutting_planes.c,
 * qap_simulated_annealing.c and heuristic.c makes its branch-and-bound loop
 * run its bounding on the GPU.
 *
 * Global state: like the reference, these functions read and write the
 * process globals X, Z, X_bundle, X_test, dual_gamma, dgamma, gamma_test,
 * lambda, eta, F, G, g, f, Cuts, List, Pent_Cuts, Pent_List, Hepta_Cuts,
 * Hepta_List, params, SP, PP, BabPbSize (src/global_var.h:1-48,
 * src/heap.c:7-8).  The library defines them too; when the host program
 * defines them (the reference's allocate_free.c / heap.c), the program's
 * definitions are the ones used.
 *
 * Part 2 (additions): initialisation and status, the batched and
 * device-pointer entry points used by the batched B&B driver and the
 * benchmarks, and a standalone solver.
 *
 * Errors: numeric failures on the path are fatal in the reference
 * (MPI_Abort(MPI_COMM_WORLD, 10), e.g. src/ipm_mc_pk.c:132-136).  Here they
 * call the abort hook (default: print and exit(10)); bqb_last_error() keeps
 * the message.  There is no CPU fallback: without a usable CUDA device every
 * entry point fails through the same hook.
 */
#ifndef BQB_GPU_H
#define BQB_GPU_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- types (layouts identical to the reference) --------------------- */
#define BQB_NMAX 1024                 /* src/biqbin_cpp_api.h:38 NMAX */
#define BQB_MAX_TRI_INEQ 50000        /* src/biqbin.h:37 MaxTriIneqAdded */
#define BQB_MAX_PENT_INEQ 50000       /* src/biqbin.h:38 */
#define BQB_MAX_HEPTA_INEQ 50000      /* src/biqbin.h:39 */
#define BQB_MAX_BUNDLE 400            /* src/biqbin.h:42 MaxBundle */

#ifndef BIQBIN_CPP_API_H
/* src/biqbin_cpp_api.h:27-35 */
typedef struct Problem {
    double *L;
    int n;
    int NIneq;
    int NPentIneq;
    int NHeptaIneq;
    int bundle;
} Problem;

/* src/biqbin_cpp_api.h:41-63 */
typedef struct BabSolution {
    int X[BQB_NMAX];
} BabSolution;

typedef struct BabNode {
    int xfixed[BQB_NMAX];
    BabSolution sol;
    double fracsol[BQB_NMAX];
    int level;
    double upper_bound;
} BabNode;
#endif

#ifndef BIQBIN_H
/* src/biqbin.h:81-107 */
typedef struct Triangle_Inequality {
    int i, j, k, type;
    double value;
    double y;
} Triangle_Inequality;

typedef struct Pentagonal_Inequality {
    int type;
    int permutation[5];
    double value;
    double y;
} Pentagonal_Inequality;

typedef struct Heptagonal_Inequality {
    int type;
    int permutation[7];
    double value;
    double y;
} Heptagonal_Inequality;

/* src/biqbin.h:49-84 (PARAM_FIELDS, same order and types) */
typedef struct BiqBinParameters {
    int init_bundle_iter;
    int max_bundle_iter;
    int triag_iter;
    int pent_iter;
    int hept_iter;
    int max_outer_iter;
    int extra_iter;
    double violated_TriIneq;
    int TriIneq;
    int adjust_TriIneq;
    int PentIneq;
    int HeptaIneq;
    int Pent_Trials;
    int Hepta_Trials;
    int include_Pent;
    int include_Hepta;
    int root;
    int use_diff;
    int time_limit;
    int branchingStrategy;
} BiqBinParameters;
#endif

/* ==== Part 1: drop-in entry points ==================================== */

/* Basic SDP bound, src/ipm_mc_pk.c:28 (decl. src/biqbin.h:181).
 * L: n x n column-major; X: n x n output; phi: output. print is ignored. */
void ipm_mc_pk(double *L, int n, double *X, double *phi, int print);

/* y -= B(X) over the global cut lists, src/operators.c:51 (biqbin.h:186). */
void op_B(const Problem *P, double *y, const double *X);
/* X -= B^T(tt), src/operators.c:140 (biqbin.h:187). */
void op_Bt(const Problem *P, double *X, const double *tt);
/* diag / Diag, src/operators.c:14,26 (biqbin.h:184-185). */
void diag(const double *X, double *y, int n);
void Diag(double *X, const double *y, int n);

/* Dual function value and subgradient, src/bundle.c:242 (biqbin.h:145). */
double fct_eval(const Problem *PP, double *dual_gamma, double *X, double *g);
/* Bundle QP pieces, src/bundle.c:390 and :292 (biqbin.h:146-147). */
void solve_lambda(int k, double *Q, double *c, double *lambda);
void lambda_eta(const Problem *PP, double *zeta, double *G, double *dual_gamma, double *dgamma,
                double *lambda, double *eta, double *t);
/* Proximal bundle iterations on the globals, src/bundle.c:9 (biqbin.h:148). */
void bundle_method(Problem *PP, double *t, int bdl_iter);

/* Separation, src/cutting_planes.c:20,48,132,224,316,416,509 (biqbin.h:151-157). */
double evaluateTriangleInequality(double *XX, int N, int type, int ii, int jj, int kk);
double getViolated_TriangleInequalities(double *X, int N, Triangle_Inequality *List, int *ListSize);
double updateTriangleInequalities(Problem *PP, double *y, int *NumAdded, int *NumSubtracted);
double getViolated_PentagonalInequalities(double *X, int N, Pentagonal_Inequality *Pent_List,
                                          int *ListSize);
double updatePentagonalInequalities(Problem *PP, double *y, int *NumAdded, int *NumSubtracted,
                                    int triag);
double getViolated_HeptagonalInequalities(double *X, int N, Heptagonal_Inequality *Hepta_List,
                                          int *ListSize);
double updateHeptagonalInequalities(Problem *PP, double *y, int *NumAdded, int *NumSubtracted,
                                    int hept_index);
/* src/qap_simulated_annealing.c:12 (biqbin.h:192). */
double qap_simulated_annealing(int *H, int k, double *X, int n, int *pent);

/* Heuristic, src/heuristic.c:11,19,119,195,304 (biqbin.h:170-174,
 * biqbin_cpp_api.h:65,68). */
double runHeuristic(Problem *P0, Problem *P, BabNode *node, int *x);
double runHeuristic_unpacked(double *P0_L, int P0_N, double *P_L, int P_N, int *node_xfixed,
                             int *node_sol_X, int *x);
double GW_heuristic(double *P0_L, int P0_N, double *P_L, int P_N, int *node_xfixed,
                    int *node_sol_X, int *x, int num);
double mc_1opt(int *x, double *P_L, int P_N);
int update_best(int *xbest, int *xnew, double *best, int P0_N);

/* Node bound orchestrator, src/bounding.c:24 (biqbin.h:142), with all
 * matrices resident on the device; reads/writes the same globals. */
double SDPbound(BabNode *node, Problem *SP, Problem *PP, int rank);

/* Host B&B pieces the bound calls (restated for standalone use; a host
 * program's own definitions take precedence): src/evaluate.c:11,38,123,
 * src/bab_functions.c:96,114,387,425, src/heap.c:15,185,
 * src/process_input.c:201,259. */
double Evaluate(BabNode *node, Problem *SP, Problem *PP, int rank);
void createSubproblem(BabNode *node, Problem *SP, Problem *PP);
double getFixedValue(BabNode *node, Problem *SP);
double evaluateSolution(int *sol);
int updateSolution(int *x);
int getBranchingVariable(BabNode *node);
int countFixedVariables(BabNode *node);
double Bab_LBGet(void);
int Bab_LBUpd(double new_lb, BabSolution *bs);
int Bab_numEvalNodes(void);
double *readData(const char *instance, int *adj_N);
int process_adj_matrix(double *Adj, int Adj_N);

/* ==== Part 2: additions =============================================== */

/* Parameters: header defaults (src/biqbin.h:49-78) and a params-file
 * reader ("name = value" lines, src/process_input.c:158-197). */
void bqb_default_params(BiqBinParameters *p);
int bqb_read_params(const char *path, BiqBinParameters *p);

/* Standalone solver: serial best-first B&B to optimality with every node
 * bounded on the GPU.  adj: num_vertices x num_vertices symmetric integer
 * weights; the last vertex is fixed to 0 as in the reference.  prm NULL
 * means the reference's shipped `params` file values.  rand() is seeded
 * with 2020 as the reference's Bab_Init does. */
typedef struct bqb_solve_result {
    double best_value;      /* "Maximum value" */
    double root_bound;      /* "Root node bound" */
    int nodes;              /* evaluated B&B nodes */
    int stopped;            /* time limit reached */
    double seconds;         /* wall time of the B&B */
    int num_vertices;
    int solution[BQB_NMAX]; /* 0/1 per vertex (vertex i+1 in the cut set if 1) */
} bqb_solve_result;
int bqb_solve(const double *adj, int num_vertices, const BiqBinParameters *prm, bqb_solve_result *out);

/* The same B&B with `threads` nodes bounded at the same time, each by its
 * own bounding engine (CUDA stream, device buffers, cut lists, random
 * stream) on its own host thread: the reference's MPI workers
 * (src/bab_functions.c:224-336, src/main.c:195-240) as engines of one
 * process.  The root is bounded first on the library globals with rank 0;
 * later nodes with rank 1.  Engine i draws its random numbers from the
 * stream srandom(2021 + i) starts, so node order and heuristic cuts (not the
 * optimum) can differ from the serial solver's.  threads <= 1: bqb_solve. */
int bqb_solve_parallel(const double *adj, int num_vertices, const BiqBinParameters *prm, int threads,
                       bqb_solve_result *out);

/* Host heuristic plug-in (the reference's Python `set_heuristic`,
 * src/wrapper.cpp:205-227, reached through runHeuristic,
 * src/heuristic.c:11-17): a function with runHeuristic_unpacked's contract
 * (P0_L, P0_N, P_L, P_N, node xfixed, node sol.X, x -> value; x receives
 * the 0/1 solution of the BabPbSize original variables) that SDPbound on
 * the library's default engine calls instead of the GPU heuristic; the
 * global X holds the node's X during the call, as runHeuristic_unpacked
 * expects.  NULL restores the GPU heuristic.  Engines and the fused kernel
 * always use their own GPU heuristic. */
typedef double (*bqb_heuristic_fn)(double *P0_L, int P0_N, double *P_L, int P_N, int *xfixed, int *sol_X,
                                   int *x);
void bqb_set_heuristic_hook(bqb_heuristic_fn fn);
/* Heuristic calls made by SDPbound on the default engine and on engines
 * since the last reset (reset != 0 resets after reading; the fused kernel's
 * calls are not counted). */
long long bqb_heuristic_runs(int reset);
/* Bundle iterations (one fct_eval each, src/bundle.c:9-239) run by SDPbound
 * on the default engine and on engines since the last reset (reset != 0
 * resets after reading; the fused kernel's are not counted).  No reference
 * counterpart. */
long long bqb_bundle_iterations(int reset);

/* Root effort: full != 0 makes SDPbound run its outer loop to
 * max_outer_iter + extra_iter rounds at rank 0 (the root) unless the node is
 * pruned, skipping the two early give-up tests (src/bounding.c:203-214).
 * Nodes with rank != 0 keep the reference's rule.  Off by default.  No
 * reference counterpart. */
void bqb_set_root_effort(int full);

/* Parent start: on != 0 makes every node bounded by SDPbound export its
 * final cuts (triangle, pentagonal, heptagonal) and multipliers, and makes
 * bqb_solve_parallel start each child from its parent's: the parent's cuts
 * that avoid the child's fixed vertices join the child's first cut list
 * with the parent's multipliers; that start is evaluated once (one IPM) and
 * kept when its dual value is below the plain start's.  Bounds stay valid
 * (inherited cuts are valid for the child; any multipliers >= 0 bound).  A
 * loaded warm-start model (bqb_warm_enable) takes precedence.  Off by
 * default.  No reference counterpart. */
void bqb_set_parent_start(int on);

/* Trace of SDPbound's outer loop (inspection): on != 0 clears the trace and
 * starts recording; bqb_bound_trace copies up to max_rows rows of 9 values
 * (node number, rank, round, bound, incumbent, triangle / pentagonal /
 * heptagonal cuts after the round, seconds since the node's loop started)
 * and returns the rows recorded.  No reference counterpart. */
void bqb_bound_trace_enable(int on);

/* Restart the engines' random streams: engine i draws from the stream
 * srand(base + i) gives (base 2021 by default) and seeds its annealing
 * chains from base + i.  Returns 1 (nothing changed) while an engine is
 * leased, else 0.  No reference counterpart. */
int bqb_seed_engines(unsigned base);
int bqb_bound_trace(double *out, int max_rows);

/* Tensor-core product D = A B^T (tcgen05.mma kind::tf32, FP32 accumulation
 * in tensor memory, operands staged by TMA): the kernel behind the batched
 * Goemans-Williamson projection S = Lf V of many hyperplanes at once (the
 * reference projects one hyperplane at a time, src/heuristic.c:142-151).
 * A: M x K and B: N x K row-major FP32 device arrays with row pitch Kp (a
 * multiple of 32, zeros beyond K, 16-byte aligned); D: M x N column-major
 * FP32 (leading dimension M).  Synchronous on the library stream.  Returns
 * 0; 1 on bad sizes or no tensor-map encoder; 2 on a CUDA error or a
 * bounded wait inside the kernel that ran out.  No reference counterpart. */
int bqb_tc_gemm_tf32(const float *A, const float *B, float *D, int M, int N, int Kp);
/* Hyperplanes per Goemans-Williamson round of the concurrent engines'
 * heuristic (bqb_bound_nodes, bqb_solve_parallel, and the engines behind
 * bqb_solve_fused above 128 vertices).  0, the default: the reference's
 * P0_N hyperplanes per round, drawn on the host in rand() order
 * (src/heuristic.c:83,142-143).  H > 0: H hyperplanes per round drawn on the
 * device and projected at once by bqb_tc_gemm_tf32's kernel with the sign
 * in its epilogue, then 1-opt and exact evaluation of every cut as before.
 * The drop-in entry points always follow the reference.  Clamped to
 * 0..65536.  No reference counterpart. */
void bqb_set_gw_hyperplanes(int H);

/* The same B&B with the nodes bounded in batches by the fused node kernel
 * (bqb_fused_submit / bqb_fused_collect): after the root (rank 0, library
 * globals), batches of at most `batch` open nodes with the largest parent
 * bounds, up to `depth` (<= 8) batches in flight, every node bounded with
 * rank 1 and branched as the reference's workers branch
 * (src/bab_functions.c:224-336).  Children are queued with their parent's
 * bound as priority; a node whose parent bound no longer exceeds the
 * incumbent by more than 1 is pruned unbounded.  Problems above 128
 * vertices go to bqb_solve_parallel.  Returns 0, 1 on bad input, 2 when a
 * submission fails. */
int bqb_solve_fused(const double *adj, int num_vertices, const BiqBinParameters *prm, int batch, int depth,
                    bqb_solve_result *out);

/* The same B&B with the open-node pool on the device: after the root (rank
 * 0, library globals), one persistent launch of the fused node kernel runs
 * the whole tree, each CTA popping the open node with the largest parent
 * bound (src/heap.c:27-133), bounding it with rank 1, branching it as the
 * reference's workers do (src/bab_functions.c:224-336, getBranchingVariable)
 * and pushing its two children, until no node is open; the incumbent lives
 * on the device.  Nodes the kernel flags are bounded by engines on the host
 * and their children pushed back.  pool_nodes: node records on the device
 * (<= 0: 65536).  Problems above 128 vertices go to bqb_solve_parallel.
 * Returns 0, 1 on bad input or a full pool, 2 on an engine error.  No
 * reference counterpart (the reference keeps one heap per MPI process). */
int bqb_solve_device(const double *adj, int num_vertices, const BiqBinParameters *prm, int pool_nodes,
                     bqb_solve_result *out);

/* Bound `count` independent nodes of the problem set up by
 * process_adj_matrix (SP) with `threads` concurrent engines: bounds[i] is
 * SDPbound(nodes[i], SP, <engine subproblem>, rank) (src/bounding.c:24-342)
 * and nodes[i].fracsol is filled as SDPbound fills it.  L_dev: NULL (each
 * subproblem is built on the host by createSubproblem), or count device
 * pointers to the subproblem matrices createSubproblem would build (n x n,
 * column-major, n = BabPbSize + 1 - fixed variables).  Returns 0, or 1 when
 * SP is not set up.  No reference counterpart (the reference bounds one
 * node per MPI process). */
int bqb_bound_nodes(BabNode *nodes, int count, int rank, int threads, const double *const *L_dev,
                    double *bounds);

/* The same bounds as bqb_bound_nodes, computed by one persistent kernel in
 * which every CTA (one per SM) bounds whole nodes on the device: the
 * subproblem, the basic IPM, the heuristic, the separations and cut-list
 * updates and the bundle iterations of SDPbound (src/bounding.c:24-342)
 * with no host round trip.  The incumbent enters as Bab_LBGet(); heuristic
 * improvements are passed to Bab_LBUpd after the kernel, in node order.
 * nodes[i].fracsol and bounds[i] are filled as SDPbound fills them.  The
 * heuristic and the annealing chains draw from counter-based streams of
 * their own.  Nodes beyond the kernel's capacities (N0 > 128, bundle
 * larger than 64, more cuts than the slot holds) or meeting a numerical
 * failure are bounded again by bqb_bound_nodes.  Returns 0, or 1 when SP
 * is not set up.  No reference counterpart. */
int bqb_bound_nodes_fused(BabNode *nodes, int count, int rank, double *bounds);
/* The same as a submission and a collection, so that several batches are
 * in flight at once (up to 8, each on its own stream and device arena):
 * the CTAs of a later batch take the SMs an earlier batch's last nodes
 * leave idle.  bqb_fused_submit copies the nodes' fixings and returns a
 * ticket >= 0 (-1: eight submissions are uncollected; -2: SP not set up;
 * -3: the problem is outside the fused kernel's range, use
 * bqb_bound_nodes; -4: count <= 0).  The incumbent each batch starts from
 * is Bab_LBGet() at its submission.  bqb_fused_collect waits for a ticket
 * and fills bounds[i] and nodes[i].fracsol of the array that was submitted
 * (nodes the kernel hands back are bounded again by engines here);
 * returns 0, or 1 for an unknown ticket. */
long long bqb_fused_submit(const BabNode *nodes, int count, int rank);
int bqb_fused_collect(long long ticket, BabNode *nodes, double *bounds);
/* Nodes bqb_bound_nodes_fused handed back to engines so far. */
long long bqb_fused_fallbacks(void);
/* Set the incumbent value Bab_LBGet returns (lower or higher; BabSol is
 * left unchanged), so that a benchmark or a test can bound every batch from
 * the same incumbent.  No reference counterpart. */
void bqb_reset_incumbent(double value);
/* Timing of bqb_bound_nodes_fused since the last reset: out[5] = {calls,
 * nodes, fused-kernel milliseconds (CUDA events), nodes bounded again by
 * engines, milliseconds of that}. */
void bqb_fused_stats(double *out);
/* Fused-kernel launches since the last bqb_fused_stats_reset: submissions
 * made while a launch runs wait on the host and start together, as one
 * launch with a heaviest-first order over all their nodes, at the next
 * collect (or the next submission that finds the GPU idle). */
long long bqb_fused_launches(void);
void bqb_fused_stats_reset(void);
/* Seconds spent per phase inside the fused kernel since the last reset,
 * summed over its CTAs: out[11] = {subproblem, IPM, heuristic, triangle
 * scan, triangle list update, k-gonal separation, cut upload, B^T, B,
 * lambda_eta, bundle step}. */
void bqb_fused_profile(double *out);
/* Calls per phase of the fused kernel since the last reset, the phases of
 * bqb_fused_profile (out[11]; out[2] = heuristic runs). */
void bqb_fused_phase_calls(long long *out);
/* Seconds per phase of SDPbound on the engines (bqb_bound_nodes, the
 * parallel and serial solvers, the drop-in), summed over engines and calls
 * since the last reset: out[12] = {IPM, lambda_eta, L - B^T(gamma), op_B of
 * the new bundle element + bundle step, heuristic, triangle separation,
 * pentagonal / heptagonal separation, the rest, whole calls, cut upload,
 * fracsol, bundle growth}.  Off by default; with it on every phase boundary
 * synchronises the engine's stream.  For profiling; no reference
 * counterpart. */
void bqb_engine_profile_enable(int on);
void bqb_engine_profile(double *out, int reset);
/* With the engines' profile on: out[6] = {lambda_eta calls, rounds of its
 * lambda / eta alternation, sum of the bundle sizes, SM cycles in the QP,
 * SM cycles in the calls, sum of the cut counts}.  No reference
 * counterpart. */
void bqb_lambda_eta_profile(double *out, int reset);
/* Device milliseconds each node of the last bqb_bound_nodes_fused call took
 * (node order of that call); writes at most `count`, returns how many. */
int bqb_fused_node_times(double *out, int count);

/* Pentagonal (k = 5) / heptagonal (k = 7) separation chains on the GPU:
 * `chains` independent runs of the annealing of qap_simulated_annealing
 * (src/qap_simulated_annealing.c:12-160), chain c for type (c % types) + 1
 * of src/cutting_planes.c:239-244 / 431-438, each drawing from its own
 * SplitMix64 stream started at seed + (c + 1) * 0xD1B54A32D192ED03 instead
 * of rand().  X: host, n x n column-major.  cost[c] and perm[7c .. 7c+k-1]
 * receive each chain's best value and permutation.  Returns 0, 1 if a chain
 * was stopped at the 80-round limit, 2 on bad arguments.  This is the
 * separation extra engines run (bqb_bound_nodes, bqb_solve_parallel); no
 * reference counterpart (the reference runs the chains one after another
 * on rand()).  Not re-entrant. */
int bqb_kgon_sa(const double *X, int n, int k, int types, int chains, unsigned long long seed, double *cost,
                int *perm);

/* Bind the library to a CUDA device (default 0) and create its stream.
 * Called implicitly by every entry point; returns 0 on success. */
int bqb_init(int device);
/* Last error message ("" if none). */
const char *bqb_last_error(void);
/* Replace the fatal-error action (default: print, exit(10)).  The hook
 * receives the reference's abort code 10; if it returns, the failing entry
 * point returns with its outputs unspecified. */
void bqb_set_abort_hook(void (*hook)(int code));
/* Number of CUDA kernels this library has launched so far. */
unsigned long long bqb_kernel_launches(void);
/* The library's CUDA stream (a cudaStream_t). */
void *bqb_stream(void);
/* IPM work and time counters: enable per-launch CUDA-event timing, reset,
 * read out[6] = {sum(iterations * n^3), problems, iterations, line-search
 * factorizations, kernel milliseconds, timed launches}. */
void bqb_stats_enable(int on);
void bqb_stats_reset(void);
void bqb_ipm_stats(double *out);
/* Wait for all work the library queued. */
void bqb_synchronize(void);

/* Batched basic SDP bound over device-resident problems: one CTA per
 * problem, one launch.  Ls[i], Xs[i]: device pointers, n x n column-major,
 * n = ns[i] (sizes may differ); out: device array of 4*nprob doubles:
 * phi, iterations, status (0 ok), <L,X>.
 * A plan holds the device descriptors and scratch; launching it is
 * asynchronous on `stream` (a cudaStream_t; NULL = the library stream). */
typedef struct bqb_ipm_plan bqb_ipm_plan;
bqb_ipm_plan *bqb_ipm_plan_create(const double *const *Ls, double *const *Xs, const int *ns,
                                  int nprob, double *out);
int bqb_ipm_plan_launch(bqb_ipm_plan *plan, void *stream);
void bqb_ipm_plan_destroy(bqb_ipm_plan *plan);
/* create + launch + synchronize + destroy. */
int bqb_ipm_batch_device(const double *const *Ls, double *const *Xs, const int *ns, int nprob,
                         double *out, void *stream);

/* Per-size schedule of the multi-CTA IPM (n > 128, one cooperative launch
 * per call): bqb_ipm_schedule_set uses `grid` CTAs for every n with the
 * same number of 32-column panels (grid <= 0: back to one CTA per 32 x 32
 * tile).  bqb_ipm_autotune times `reps` calls for each candidate grid on a
 * seeded problem of size n and keeps the fastest (best_grid / best_ms may
 * be NULL); returns 0, 1 for n <= 128.  No reference counterpart. */
void bqb_ipm_schedule_set(int n, int grid);
/* Timing of the multi-CTA IPM by parts (its first CTA, summed over calls;
 * off by default): out[8] = {ms waiting at grid barriers, ms in panel
 * factorisations, ms in tile updates, ms in the products, ms in whole
 * calls, grid barriers, sweep phases, ms of the panel factorisations
 * spent loading the panel block}; reset != 0 zeroes after reading.  For
 * profiling; no reference counterpart. */
void bqb_ipm_coop_profile_enable(int on);
void bqb_ipm_coop_profile(double *out, int reset);
int bqb_ipm_autotune(int n, int reps, int *best_grid, double *best_ms);

/* FP64 certificate of a basic SDP bound (csrc/certificate.cu).  L: n x n
 * column-major, y: any dual vector (host).  out[0] = an upper bound on
 * max <L, X> over diag(X) = e, X psd that holds for every y: the sum of y
 * plus n times an FP64 lower bound on -lambda_min(Diag(y) - L) when that
 * minimum is negative, every rounding error bounded (a completed Cholesky
 * factorisation of Diag(y) - L + tI and its backward error); out[1] = the
 * lower bound on lambda_min; out[2] = the shift t the factorisation needed
 * (0 when Diag(y) - L factors as it is); out[3] = 0, or 1 when no shift
 * worked.  Returns 0, or 1 on bad arguments.  No reference counterpart (the
 * reference's bound is the IPM's dual value, src/ipm_mc_pk.c:313-334). */
int bqb_sdp_certificate(const double *L, const double *y, int n, double *out);
/* ipm_mc_pk (src/ipm_mc_pk.c:28-359) that also returns the dual vector y of
 * the last iterate (host, n doubles; phi is its sum): out[4] = {phi,
 * iterations, status, <L, X>}; X may be NULL.  Returns 0, or 1 on bad
 * arguments.  No reference counterpart. */
int bqb_ipm_dual(const double *L, int n, double *X, double *y, double *out);
/* Certificates of the engines' node bounds on (1) / off (0, default): each
 * node's final bound is certified by one more IPM at its final multipliers
 * and bqb_sdp_certificate.  bqb_certify_stats: out[6] = {nodes, largest and
 * mean excess of the certified bound over the node's bound, relative to
 * max(1, |bound|), nodes whose certificate failed, largest shift, largest
 * relative difference between the rerun IPM's value and the bundle's};
 * reset != 0 zeroes them.  No reference counterpart. */
void bqb_certify_enable(int on);
void bqb_certify_stats(double *out, int reset);

/* Basic SDP bound of one problem without any device allocation.  No
 * counterpart in the reference: it exists for callers that may not call
 * cudaMalloc while they run (e.g. inside a host application whose memory
 * manager owns the GPU, or in a loop that must not synchronise on an
 * allocation).  L, X: device pointers, n x n column-major; out: device, 4
 * doubles (phi, iterations, status, <L,X>).  Scratch is a fixed array in the
 * library's static device memory (3 * 128^2 doubles per GPU, held until
 * exit), so n <= BQB_IPM_NOALLOC_NMAX.  The first call on a device resolves
 * the array's address and should precede any stream capture.  Calls share
 * the array: calls that overlap on the GPU race.  Asynchronous on `stream`
 * (a cudaStream_t; NULL = the legacy default stream).  Returns 0 on success;
 * 1, with a message in bqb_last_error(), when n < 1 or n > 128, when L, X or
 * out is NULL, or when the IPM's placement for this n on this device needs
 * more scratch than the array holds (the placement keeps the Cholesky
 * workspace in shared memory; a device with less opt-in shared memory than
 * a B200 would need it in the array); 2 on a CUDA error. */
#define BQB_IPM_NOALLOC_NMAX 128
int bqb_ipm_noalloc(const double *L, double *X, int n, double *out, void *stream);

/* Same, host memory in and out (copies included), synchronous. */
int bqb_ipm_batch(const double *const *Ls, double *const *Xs, const int *ns, int nprob,
                  double *phi, int *iters, int *status);

/* ==== Learned warm start of the bundle multipliers ====================
 * No reference counterpart.  After a node's first triangle separation the
 * reference starts its bundle at gamma = 0 (src/bounding.c:121-131).  With
 * a model loaded and the warm start switched on, SDPbound on every engine
 * evaluates a network's proposal gamma >= 0 for those cuts once (one IPM on
 * L - B^T(gamma)) and starts the bundle there when its dual value is below
 * the plain start's; any gamma >= 0 gives a valid bound, and the bundle then
 * runs to the reference's stopping rules.  Off by default.  Network: 12 cut
 * features -> 32 -> 32 (ReLU) -> softplus, in units of the node's objective
 * scale (mean |L_ij|); FP32 training (Adam) with this library's kernels,
 * BF16-weight inference.  Parameters: BQB_WARM_NPARAM floats, layout
 * W1[12][32], b1[32], W2[32][32], b2[32], w3[32], b3. */
#define BQB_WARM_NPARAM 1569
/* out[3] = {features per cut, hidden units, parameters}. */
void bqb_warm_dims(int *out);
/* Train from params (in/out) on N rows: feats[N x 12], targets[N]; Adam,
 * `steps` minibatches of `batch` rows (seeded shuffle); losses[steps] may be
 * NULL.  Returns 0, or -1 on bad arguments. */
int bqb_warm_train(const float *feats, const float *targets, int N, int steps, int batch, float lr,
                   unsigned seed, float *params, float *losses);
/* Full-batch loss and gradient at params (the training kernels). */
int bqb_warm_grad(const float *params, const float *feats, const float *targets, int N, float *grad,
                  float *loss);
/* Inference path (BF16 weights) on N feature rows: out[N]. */
int bqb_warm_predict(const float *params, const float *feats, int N, double *out);
/* Load the model SDPbound uses (NULL unloads); call before bounding. */
int bqb_warm_set_model(const float *params);
/* Warm start on (a model must be loaded) / off. */
void bqb_warm_enable(int on);
/* Record training pairs while bounding (features of each node's first-
 * separation cuts, the multipliers they end with; off by default). */
void bqb_warm_record(int on);
/* Copy min(count, cap) recorded pairs out; returns the count. */
long long bqb_warm_dataset(float *feats, float *targets, long long cap);
void bqb_warm_dataset_clear(void);
/* out[2] = {proposals kept, proposals rejected}; reset != 0 zeroes them. */
void bqb_warm_stats(long long *out, int reset);
/* The features of m triangle cuts (cuts: m x {type, i, j, k}, values: their
 * violations) at X and the objective L (host, n x n column-major) into
 * out[m x 14]; parent_gamma (may be NULL): the multiplier each cut ended
 * with in the parent node's final cut list, -1 for a cut the parent did not
 * hold.  For checking against the oracle.  Returns 0, or -1 on bad
 * arguments (an index outside 0..n-1, a type outside 1..4). */
int bqb_warm_features(const double *X, const double *L, int n, const int *cuts, const double *values, int m,
                      double viol3, double gap, const double *parent_gamma, float *out);

#ifdef __cplusplus
}
#endif

#endif /* BQB_GPU_H */
