// Host branch-and-bound runtime around the GPU bounding path, and a
// standalone serial solver.
//
// Restated from the reference's host files so that the library can be used
// on its own (the reference's own host objects, when linked against this
// library, take precedence over every symbol defined here):
//   heap.c         priority queue on upper_bound, incumbent (LB, BabSol)
//   bab_functions.c evaluateSolution, updateSolution, getBranchingVariable,
//                  countFixedVariables, the worker step
//   evaluate.c     Evaluate, createSubproblem, getFixedValue
//   process_input.c process_adj_matrix (SP->L from an adjacency matrix),
//                  the Rudy reader and the parameter-file reader
// The driver is serial and best-first: the root is bounded with rank 0
// (recording diff), its two children are queued, then nodes are popped and
// bounded with rank 1 (so the use_diff give-up test applies), as one worker
// of the reference's MPI code does when it never finds a free peer.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <atomic>
#include <condition_variable>
#include <mutex>
#include <unordered_map>
#include <thread>
#include <vector>

#include "engine.h"
#include "globals.h"

extern "C" {
double SDPbound(BabNode* node, Problem* SP_, Problem* PP_, int rank);
__attribute__((visibility("default"))) double diff = 0.0;
__attribute__((visibility("default"))) double root_bound = 0.0;
__attribute__((visibility("default"))) double TIME = 0.0;
__attribute__((visibility("default"))) int stopped = 0;
__attribute__((visibility("default"))) BabSolution* BabSol = nullptr;
}

namespace {

constexpr double BIG_NUMBER = 1e9;
// The incumbent value is read by every concurrent bound; updates are
// serialised so the value and BabSol change together.
std::atomic<double> g_LB{0.0};
std::mutex g_lb_mu;
int g_num_nodes = 0;

double wtime()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

// Binary max-heap on upper_bound with the reference's comparison and
// sift rules (src/heap.c:27-133).
struct NodeHeap {
    std::vector<BabNode*> data;
    int used = 0;
    static int cmp(const BabNode* a, const BabNode* b) { return a->upper_bound > b->upper_bound ? 1 : -1; }
    void swap_e(int i, int j)
    {
        BabNode* t = data[i];
        data[i] = data[j];
        data[j] = t;
    }
    void down(int cur)
    {
        int child = 2 * cur + 1;
        if (child + 1 < used && cmp(data[child + 1], data[child]) > 0) child++;
        while (child < used && cmp(data[cur], data[child]) < 0) {
            swap_e(cur, child);
            cur = child;
            child = 2 * cur + 1;
            if (child + 1 < used && cmp(data[child + 1], data[child]) > 0) child++;
        }
    }
    void up(int cur)
    {
        int parent = (cur - 1) / 2;
        while (cur > 0 && cmp(data[parent], data[cur]) < 0) {
            swap_e(cur, parent);
            cur = parent;
            parent = (cur - 1) / 2;
        }
    }
    void push(BabNode* n)
    {
        if ((int)data.size() <= used) data.resize(used + 64, nullptr);
        data[used++] = n;
        up(used - 1);
    }
    BabNode* pop()
    {
        BabNode* n = data[0];
        data[0] = nullptr;
        used--;
        swap_e(0, used);
        down(0);
        return n;
    }
    bool empty() const { return used == 0; }
};

BabNode* new_node(const BabNode* parent)
{
    BabNode* node = (BabNode*)malloc(sizeof(BabNode));
    if (!node) {
        fprintf(stderr, "Error: Not enough memory for creating new node.\n");
        exit(10);
    }
    for (int i = 0; i < BabPbSize; ++i) {
        node->xfixed[i] = parent ? parent->xfixed[i] : 0;
        node->sol.X[i] = (parent && node->xfixed[i]) ? parent->sol.X[i] : 0;
    }
    node->level = parent ? parent->level + 1 : 0;
    node->upper_bound = 0.0;
    return node;
}

}  // namespace

// ---- incumbent (src/heap.c:15, 172-193) -----------------------------------
BQB_API double Bab_LBGet(void) { return g_LB.load(); }

BQB_API int Bab_LBUpd(double new_lb, BabSolution* bs)
{
    std::lock_guard<std::mutex> lock(g_lb_mu);
    if (new_lb > g_LB.load()) {
        g_LB.store(new_lb);
        if (BabSol) *BabSol = *bs;
        return 1;
    }
    return 0;
}

BQB_API int Bab_numEvalNodes(void) { return g_num_nodes; }

// Set the incumbent value (the solution is left as it is), lower or higher:
// lets a benchmark or a test start every batch from the same incumbent.
BQB_API void bqb_reset_incumbent(double value)
{
    std::lock_guard<std::mutex> lock(g_lb_mu);
    g_LB.store(value);
}

// ---- src/bab_functions.c:96-134 --------------------------------------------
BQB_API double evaluateSolution(int* sol)
{
    double val = 0.0;
    for (int i = 0; i < BabPbSize; ++i)
        for (int j = 0; j < BabPbSize; ++j) val += SP->L[j + (size_t)i * SP->n] * sol[i] * sol[j];
    return val;
}

BQB_API int updateSolution(int* x)
{
    BabSolution solx;
    for (int i = 0; i < BabPbSize; ++i) solx.X[i] = x[i];
    const double v = evaluateSolution(x);
    return Bab_LBUpd(v, &solx);
}

// ---- src/bab_functions.c:387-436 -------------------------------------------
BQB_API int countFixedVariables(BabNode* node)
{
    int c = 0;
    for (int i = 0; i < BabPbSize; ++i) c += node->xfixed[i] ? 1 : 0;
    return c;
}

BQB_API int getBranchingVariable(BabNode* node)
{
    int ic = -1;
    if (params.branchingStrategy == 0) {   // LEAST_FRACTIONAL
        double maxv = -BIG_NUMBER;
        for (int i = 0; i < BabPbSize; ++i)
            if (!node->xfixed[i] && fabs(0.5 - node->fracsol[i]) > maxv) {
                ic = i;
                maxv = fabs(0.5 - node->fracsol[ic]);
            }
    } else if (params.branchingStrategy == 1) {   // MOST_FRACTIONAL
        double minv = BIG_NUMBER;
        for (int i = 0; i < BabPbSize; ++i)
            if (!node->xfixed[i] && fabs(0.5 - node->fracsol[i]) < minv) {
                ic = i;
                minv = fabs(0.5 - node->fracsol[ic]);
            }
    } else {
        fprintf(stderr, "Error: Wrong value for params.branchingStrategy\n");
        exit(10);
    }
    return ic;
}

// ---- src/evaluate.c:38-138 --------------------------------------------------
BQB_API void createSubproblem(BabNode* node, Problem* SP_, Problem* PP_)
{
    PP_->n = BabPbSize + 1 - countFixedVariables(node);
    const int N = SP_->n;
    const int n = PP_->n;
    std::vector<double> fixedRow(n > 1 ? n - 1 : 1, 0.0);
    int index = 0;
    for (int i = 0; i < BabPbSize; ++i) {
        double row_sum = 0.0;
        int fixed = 0;
        for (int j = 0; j < BabPbSize; ++j) {
            if (!node->xfixed[i] && !node->xfixed[j]) {
                PP_->L[index] = SP_->L[j + (size_t)i * N];
                row_sum += PP_->L[index];
                ++index;
            } else if ((node->xfixed[i] && node->sol.X[i] == 1) && !node->xfixed[j]) {
                fixedRow[fixed] += SP_->L[j + (size_t)i * N];
                ++fixed;
            }
        }
        if (!node->xfixed[i]) PP_->L[index++] = row_sum;
    }
    for (int i = 0; i < n - 1; ++i) PP_->L[i + (size_t)(n - 1) * n] = PP_->L[n - 1 + (size_t)i * n];
    double sum = 0.0;
    for (int i = 0; i < n - 1; ++i) {
        PP_->L[i + (size_t)i * n] += 2 * fixedRow[i];
        PP_->L[n - 1 + (size_t)i * n] += 2 * fixedRow[i];
        PP_->L[i + (size_t)(n - 1) * n] += 2 * fixedRow[i];
        sum += PP_->L[i + (size_t)(n - 1) * n];
    }
    PP_->L[n - 1 + (size_t)(n - 1) * n] = sum;
    const size_t nn = (size_t)n * n;
    for (size_t e = 0; e < nn; ++e) PP_->L[e] *= 0.25;
}

BQB_API double getFixedValue(BabNode* node, Problem* SP_)
{
    const int N = SP_->n;
    double v = 0.0;
    for (int i = 0; i < BabPbSize; ++i)
        for (int j = 0; j < BabPbSize; ++j)
            if (node->xfixed[i] && node->xfixed[j]) v += SP_->L[j + (size_t)i * N] * node->sol.X[i] * node->sol.X[j];
    return v;
}

BQB_API double Evaluate(BabNode* node, Problem* SP_, Problem* PP_, int rank)
{
    createSubproblem(node, SP_, PP_);
    return SDPbound(node, SP_, PP_, rank);
}

// ---- src/process_input.c:259-344 --------------------------------------------
BQB_API int process_adj_matrix(double* Adj, int num_vertices)
{
    // fused submissions waiting on the host were made for the current problem
    bqb::fused_launch_pending();
    BabPbSize = num_vertices - 1;
    ++bqb::g_sp_generation;
    if (!SP) SP = (Problem*)calloc(1, sizeof(Problem));
    if (!PP) PP = (Problem*)calloc(1, sizeof(Problem));
    SP->n = num_vertices;
    free(SP->L);
    free(PP->L);
    SP->L = (double*)calloc((size_t)num_vertices * num_vertices, sizeof(double));
    PP->L = (double*)calloc((size_t)num_vertices * num_vertices, sizeof(double));
    PP->n = SP->n;
    const int nv = num_vertices;
    std::vector<double> Adje(nv, 0.0);
    for (int ii = 0; ii < nv; ++ii)
        for (int jj = 0; jj < nv; ++jj) Adje[ii] += Adj[jj + (size_t)ii * nv];
    double sum = 0.0;
    for (int ii = 0; ii < nv; ++ii) {
        double sum_row = 0.0;
        for (int jj = 0; jj < nv; ++jj) {
            const size_t e = jj + (size_t)ii * nv;
            if (ii < nv - 1 && jj < nv - 1) {
                SP->L[e] = (ii == jj ? Adje[ii] : 0.0) - Adj[e];
                sum_row += SP->L[e];
            } else if (jj == nv - 1 && ii != nv - 1) {
                SP->L[e] = sum_row;
                sum += sum_row;
            } else if (ii == nv - 1 && jj != nv - 1) {
                SP->L[e] = SP->L[ii + (size_t)jj * nv];
            } else {
                SP->L[e] = sum;
            }
        }
    }
    memcpy(PP->L, SP->L, (size_t)nv * nv * sizeof(double));
    return 0;
}

// Rudy edge list: "n m" then m lines "i j w" (1-based, integer weights),
// src/process_input.c:201-253.  Returns a calloc'd n x n matrix or NULL.
BQB_API double* readData(const char* instance, int* adj_N)
{
    FILE* fh = fopen(instance, "r");
    if (!fh) {
        fprintf(stderr, "Error: problem opening input file %s\n", instance);
        return nullptr;
    }
    int nv = 0, ne = 0;
    if (fscanf(fh, "%d %d \n", &nv, &ne) != 2 || nv <= 0) {
        fprintf(stderr, "\nError: Problem reading number of vertices and edges\n");
        fclose(fh);
        return nullptr;
    }
    double* A = (double*)calloc((size_t)nv * nv, sizeof(double));
    for (int e = 0; e < ne; ++e) {
        int i, j;
        double w;
        if (fscanf(fh, "%d %d %lf \n", &i, &j, &w) != 3 || i < 1 || i > nv || j < 1 || j > nv ||
            (double)(int)w != w) {
            fprintf(stderr, "\nError: Problem reading edges of the graph\n");
            fclose(fh);
            free(A);
            return nullptr;
        }
        A[(size_t)nv * (j - 1) + (i - 1)] = w;
        A[(size_t)nv * (i - 1) + (j - 1)] = w;
    }
    fclose(fh);
    *adj_N = nv;
    return A;
}

// Parameter defaults of src/biqbin.h:49-78.
BQB_API void bqb_default_params(BiqBinParameters* p)
{
    p->init_bundle_iter = 3;
    p->max_bundle_iter = 15;
    p->triag_iter = 5;
    p->pent_iter = 5;
    p->hept_iter = 5;
    p->max_outer_iter = 20;
    p->extra_iter = 10;
    p->violated_TriIneq = 1e-3;
    p->TriIneq = 5000;
    p->adjust_TriIneq = 1;
    p->PentIneq = 5000;
    p->HeptaIneq = 5000;
    p->Pent_Trials = 60;
    p->Hepta_Trials = 50;
    p->include_Pent = 1;
    p->include_Hepta = 1;
    p->root = 0;
    p->use_diff = 1;
    p->time_limit = 0;
    p->branchingStrategy = 1;
}

// "name = value" lines (src/process_input.c:158-197); unknown names ignored.
BQB_API int bqb_read_params(const char* path, BiqBinParameters* p)
{
    bqb_default_params(p);
    FILE* fh = fopen(path, "r");
    if (!fh) return 1;
    char line[256], name[64];
    while (fgets(line, sizeof line, fh)) {
        if (sscanf(line, "%63[^=^ ]", name) != 1) continue;
        const char* eq = strchr(line, '=');
        if (!eq) continue;
        const double v = atof(eq + 1);
#define BQB_PI(field) \
    if (strcmp(name, #field) == 0) p->field = (int)v;
#define BQB_PD(field) \
    if (strcmp(name, #field) == 0) p->field = v;
        BQB_PI(init_bundle_iter) BQB_PI(max_bundle_iter) BQB_PI(triag_iter) BQB_PI(pent_iter)
        BQB_PI(hept_iter) BQB_PI(max_outer_iter) BQB_PI(extra_iter) BQB_PD(violated_TriIneq)
        BQB_PI(TriIneq) BQB_PI(adjust_TriIneq) BQB_PI(PentIneq) BQB_PI(HeptaIneq)
        BQB_PI(Pent_Trials) BQB_PI(Hepta_Trials) BQB_PI(include_Pent) BQB_PI(include_Hepta)
        BQB_PI(root) BQB_PI(use_diff) BQB_PI(time_limit) BQB_PI(branchingStrategy)
#undef BQB_PI
#undef BQB_PD
    }
    fclose(fh);
    return 0;
}

// Allocate the reference globals the bounding path reads on the host
// (src/allocate_free.c:8-42).  X_bundle and G stay on the device in this
// driver, so their host copies are not allocated.
// The solvers keep their incumbent cut in a record of their own: BabSol may
// point at memory a host program or binding has since released.  Zeroed.
static BabSolution* solver_solution()
{
    static BabSolution sol;
    memset(&sol, 0, sizeof sol);
    return &sol;
}

static void alloc_globals(int N)
{
    // Only arrays this function allocated earlier are freed: a host program
    // (or a binding) may have pointed the globals at memory of its own.
    static std::vector<void*> owned;
    auto give = [](void** slot, size_t count, size_t size) {
        for (size_t q = 0; q < owned.size(); ++q)
            if (owned[q] == *slot) {
                free(*slot);
                owned.erase(owned.begin() + q);
                break;
            }
        *slot = calloc(count > 0 ? count : 1, size);
        owned.push_back(*slot);
    };
    const size_t mmax = (size_t)BQB_MAX_TRI_INEQ + BQB_MAX_PENT_INEQ + BQB_MAX_HEPTA_INEQ;
    const size_t nn = (size_t)N * N;
    give((void**)&Cuts, BQB_MAX_TRI_INEQ, sizeof(Triangle_Inequality));
    give((void**)&List, params.TriIneq, sizeof(Triangle_Inequality));
    give((void**)&Pent_Cuts, BQB_MAX_PENT_INEQ, sizeof(Pentagonal_Inequality));
    give((void**)&Pent_List, params.PentIneq, sizeof(Pentagonal_Inequality));
    give((void**)&Hepta_Cuts, BQB_MAX_HEPTA_INEQ, sizeof(Heptagonal_Inequality));
    give((void**)&Hepta_List, params.HeptaIneq, sizeof(Heptagonal_Inequality));
    give((void**)&X, nn, sizeof(double));
    give((void**)&Z, nn, sizeof(double));
    give((void**)&X_test, nn, sizeof(double));
    give((void**)&dual_gamma, mmax, sizeof(double));
    give((void**)&dgamma, mmax, sizeof(double));
    give((void**)&gamma_test, mmax, sizeof(double));
    give((void**)&eta, mmax, sizeof(double));
    give((void**)&g, mmax, sizeof(double));
    give((void**)&lambda, BQB_MAX_BUNDLE, sizeof(double));
    give((void**)&F, BQB_MAX_BUNDLE, sizeof(double));
}

// Serial best-first B&B to optimality on the GPU bounding path.  adj:
// num_vertices^2 symmetric integer weights (column-major = row-major);
// prm: parameters (NULL: the reference's shipped `params` file values).
// Seeds rand() with 2020 as Bab_Init does (src/bab_functions.c:82).
BQB_API int bqb_solve(const double* adj, int num_vertices, const BiqBinParameters* prm, bqb_solve_result* out)
{
    if (num_vertices < 3 || num_vertices > BQB_NMAX) return 1;
    if (prm) {
        params = *prm;
    } else {
        bqb_default_params(&params);
        params.init_bundle_iter = 5;
        params.violated_TriIneq = 0.05;
    }
    std::vector<double> A(adj, adj + (size_t)num_vertices * num_vertices);
    process_adj_matrix(A.data(), num_vertices);
    if (params.adjust_TriIneq) params.TriIneq = SP->n * 10;
    srand(2020);
    BabSol = solver_solution();
    g_LB.store(0.0);
    g_num_nodes = 0;
    stopped = 0;
    diff = 0.0;
    alloc_globals(SP->n);

    TIME = wtime();
    NodeHeap heap;
    BabNode* root = new_node(nullptr);
    ++g_num_nodes;
    root_bound = Evaluate(root, SP, PP, 0);
    root->upper_bound = root_bound;
    if (Bab_LBGet() + 1.0 < root->upper_bound)
        heap.push(root);
    else
        free(root);

    auto branch = [&](BabNode* node) {
        const int ic = getBranchingVariable(node);
        for (int xic = 0; xic <= 1; ++xic) {
            BabNode* child = new_node(node);
            child->xfixed[ic] = 1;
            child->sol.X[ic] = xic;
            ++g_num_nodes;
            heap.push(child);
        }
    };
    if (!heap.empty() && !params.root) {
        BabNode* node = heap.pop();
        branch(node);
        free(node);
        while (!heap.empty()) {
            if (params.time_limit > 0 && (wtime() - TIME) > params.time_limit) {
                stopped = 1;
                break;
            }
            BabNode* nd = heap.pop();
            nd->upper_bound = Evaluate(nd, SP, PP, 1);
            if (Bab_LBGet() + 1.0 < nd->upper_bound) branch(nd);
            free(nd);
        }
    }
    while (!heap.empty()) free(heap.pop());

    if (out) {
        out->best_value = Bab_LBGet();
        out->root_bound = root_bound;
        out->nodes = g_num_nodes;
        out->stopped = stopped;
        out->seconds = wtime() - TIME;
        out->num_vertices = num_vertices;
        for (int i = 0; i < BQB_NMAX; ++i) out->solution[i] = (i < BabPbSize) ? BabSol->X[i] : 0;
    }
    return 0;
}

// ---- concurrent bounding ----------------------------------------------------
// Many nodes are bounded at the same time, each by its own engine (stream,
// device buffers, host cut lists, random stream) on its own host thread; the
// GPU runs their kernels side by side on different SMs.  This is the
// reference's own parallelism (independent B&B nodes on MPI workers) with
// engines in place of processes.

namespace {

std::mutex g_pool_mu;
std::vector<bqb::Engine*> g_pool;
std::vector<char> g_pool_busy;
unsigned g_pool_seed = 2021u;

// k private engines leased to the caller alone (concurrent callers get
// different engines; an engine and its buffers are never shared by two
// bounding threads), sized for problems up to N x N.  The first free
// engines are taken in creation order, so a single caller always gets
// engines 0..k-1; engine i draws random numbers from the stream srand(base + i)
// would give (base 2021 unless bqb_seed_engines changed it).  The lease ends
// when the returned object goes away.
struct EngineLease {
    std::vector<bqb::Engine*> e;
    EngineLease(int k, int N)
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        for (size_t i = 0; i < g_pool.size() && (int)e.size() < k; ++i)
            if (!g_pool_busy[i]) {
                g_pool_busy[i] = 1;
                e.push_back(g_pool[i]);
            }
        while ((int)e.size() < k) {
            g_pool.push_back(bqb::engine_create(g_pool_seed + (unsigned)g_pool.size()));
            g_pool_busy.push_back(1);
            e.push_back(g_pool.back());
        }
        for (bqb::Engine* x : e) x->ensure_private(N);
    }
    ~EngineLease()
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        for (bqb::Engine* x : e)
            for (size_t i = 0; i < g_pool.size(); ++i)
                if (g_pool[i] == x) g_pool_busy[i] = 0;
    }
    bqb::Engine* operator[](int t) const { return e[t]; }
};

}  // namespace

// Restart the engines' random streams: engine i (existing or created later)
// draws from the stream srand(base + i) gives, and its annealing chains from
// seeds derived from base + i.  Returns 1 while an engine is leased (nothing
// changes), else 0.
BQB_API int bqb_seed_engines(unsigned base)
{
    std::lock_guard<std::mutex> lock(g_pool_mu);
    for (char b : g_pool_busy)
        if (b) return 1;
    g_pool_seed = base;
    for (size_t i = 0; i < g_pool.size(); ++i) {
        g_pool[i]->rng.seed(base + (unsigned)i);
        g_pool[i]->sa_seed = (uint64_t)(base + (unsigned)i) << 32;
        g_pool[i]->sa_calls = 0;
    }
    return 0;
}

// Bound `count` independent nodes of the problem in SP (set up by
// process_adj_matrix) with `threads` concurrent engines; bounds[i] receives
// the bound of nodes[i] (fracsol is filled as SDPbound does).  L_dev
// (optional): device pointers to each node's subproblem matrix (PP->L as
// createSubproblem builds it), used instead of building it on the host.
BQB_API int bqb_bound_nodes(BabNode* nodes, int count, int rank, int threads, const double* const* L_dev,
                            double* bounds)
{
    if (count <= 0) return 0;
    if (!SP || !SP->L) return 1;
    bqb::rt();
    if (threads < 1) threads = 1;
    if (threads > count) threads = count;
    const EngineLease pool(threads, SP->n);
    std::atomic<int> next{0};
    const int dev = bqb::rt().device;
    auto work = [&](int t) {
        bqb::t_pool_worker = t > 0;
        BQB_CUDA(cudaSetDevice(dev));
        bqb::Engine& E = *pool[t];
        Problem& P = E.PP;
        int i;
        while ((i = next.fetch_add(1)) < count) {
            if (L_dev) {
                P.n = BabPbSize + 1 - countFixedVariables(&nodes[i]);
                P.L = const_cast<double*>(L_dev[i]);
            } else {
                P.L = E.PPL.data();
                createSubproblem(&nodes[i], SP, &P);
            }
            bounds[i] = bqb::sdp_bound(E, &nodes[i], SP, &P, rank);
            P.L = E.PPL.data();
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < threads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    return 0;
}

// Best-first B&B to optimality with `threads` nodes bounded concurrently.
// The root is bounded first with rank 0 (sets diff); then workers pop the
// node with the largest upper bound, bound it with rank 1 and branch, as the
// reference's MPI workers do.  With threads <= 1 this is bqb_solve.
BQB_API int bqb_solve_parallel(const double* adj, int num_vertices, const BiqBinParameters* prm, int threads,
                               bqb_solve_result* out)
{
    if (threads <= 1) return bqb_solve(adj, num_vertices, prm, out);
    if (num_vertices < 3 || num_vertices > BQB_NMAX) return 1;
    if (prm) {
        params = *prm;
    } else {
        bqb_default_params(&params);
        params.init_bundle_iter = 5;
        params.violated_TriIneq = 0.05;
    }
    std::vector<double> A(adj, adj + (size_t)num_vertices * num_vertices);
    process_adj_matrix(A.data(), num_vertices);
    if (params.adjust_TriIneq) params.TriIneq = SP->n * 10;
    srand(2020);
    BabSol = solver_solution();
    g_LB.store(0.0);
    g_num_nodes = 0;
    stopped = 0;
    diff = 0.0;
    alloc_globals(SP->n);

    TIME = wtime();
    NodeHeap heap;
    const EngineLease pool(threads, SP->n);
    BabNode* root = new_node(nullptr);
    ++g_num_nodes;
    {
        // the root on engine 0 (rank 0 sets diff): its heuristic and k-gonal
        // separation run on the device as every other node's do
        bqb::Engine& E0 = *pool[0];
        E0.PP.L = E0.PPL.data();
        createSubproblem(root, SP, &E0.PP);
        root_bound = bqb::sdp_bound(E0, root, SP, &E0.PP, 0);
    }
    root->upper_bound = root_bound;
    std::mutex mu;
    std::condition_variable cv;
    int active = 0;
    bool stop = false;
    // with the learned warm start, the recorder or the parent start on, each
    // child bounds with its parent's final cuts (bqb::Engine::parent)
    std::unordered_map<BabNode*, std::shared_ptr<bqb::ParentCuts>> parent_of;
    auto branch = [&](BabNode* node, const std::shared_ptr<bqb::ParentCuts>& cuts = nullptr) {
        const int ic = getBranchingVariable(node);
        for (int xic = 0; xic <= 1; ++xic) {
            BabNode* child = new_node(node);
            child->xfixed[ic] = 1;
            child->sol.X[ic] = xic;
            ++g_num_nodes;
            heap.push(child);
            if (cuts) parent_of[child] = cuts;
        }
    };
    if (Bab_LBGet() + 1.0 < root->upper_bound && !params.root)
        branch(root, std::move(pool[0]->final_cuts));
    free(root);

    const int dev = bqb::rt().device;
    auto work = [&](int t) {
        bqb::t_pool_worker = t > 0;
        BQB_CUDA(cudaSetDevice(dev));
        bqb::Engine& E = *pool[t];
        Problem& P = E.PP;
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            cv.wait(lk, [&] { return !heap.empty() || active == 0 || stop; });
            if (stop || heap.empty()) {
                cv.notify_all();
                return;
            }
            if (params.time_limit > 0 && (wtime() - TIME) > params.time_limit) {
                stopped = 1;
                stop = true;
                cv.notify_all();
                return;
            }
            BabNode* node = heap.pop();
            ++active;
            std::shared_ptr<bqb::ParentCuts> pc;
            auto it = parent_of.find(node);
            if (it != parent_of.end()) {
                pc = std::move(it->second);
                parent_of.erase(it);
            }
            lk.unlock();
            P.L = E.PPL.data();
            createSubproblem(node, SP, &P);
            E.parent = pc.get();
            node->upper_bound = bqb::sdp_bound(E, node, SP, &P, 1);
            E.parent = nullptr;
            std::shared_ptr<bqb::ParentCuts> mine = std::move(E.final_cuts);
            lk.lock();
            if (Bab_LBGet() + 1.0 < node->upper_bound) branch(node, mine);
            free(node);
            --active;
            cv.notify_all();
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < threads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    while (!heap.empty()) free(heap.pop());
    parent_of.clear();

    if (out) {
        out->best_value = Bab_LBGet();
        out->root_bound = root_bound;
        out->nodes = g_num_nodes;
        out->stopped = stopped;
        out->seconds = wtime() - TIME;
        out->num_vertices = num_vertices;
        for (int i = 0; i < BQB_NMAX; ++i) out->solution[i] = (i < BabPbSize) ? BabSol->X[i] : 0;
    }
    return 0;
}

// ---- B&B with fused batches ------------------------------------------------
extern "C" {
long long bqb_fused_submit(const BabNode* nodes, int count, int rank);
int bqb_fused_collect(long long ticket, BabNode* nodes, double* bounds);
}

// Best-first B&B whose nodes are bounded in batches by the fused node kernel
// (bqb_fused_submit / bqb_fused_collect), up to `depth` batches in flight.
// The root is bounded first with rank 0 on the library globals (sets diff);
// then batches of at most `batch` open nodes with the largest parent bounds
// are bounded with rank 1, and every node whose bound exceeds the incumbent
// by more than 1 is branched (src/bab_functions.c:224-336).  A child is
// queued with its parent's bound as priority, and a node whose parent bound
// no longer exceeds the incumbent by more than 1 is pruned without being
// bounded (the parent bound is a valid bound of the child).  Problems the
// fused kernel does not take (N0 > 128) go to bqb_solve_parallel.
BQB_API int bqb_solve_fused(const double* adj, int num_vertices, const BiqBinParameters* prm, int batch, int depth,
                            bqb_solve_result* out)
{
    if (num_vertices < 3 || num_vertices > BQB_NMAX) return 1;
    if (num_vertices > 128) return bqb_solve_parallel(adj, num_vertices, prm, 16, out);
    if (batch < 1) batch = 1;
    if (depth < 1) depth = 1;
    if (depth > 8) depth = 8;
    if (prm) {
        params = *prm;
    } else {
        bqb_default_params(&params);
        params.init_bundle_iter = 5;
        params.violated_TriIneq = 0.05;
    }
    std::vector<double> A(adj, adj + (size_t)num_vertices * num_vertices);
    process_adj_matrix(A.data(), num_vertices);
    if (params.adjust_TriIneq) params.TriIneq = SP->n * 10;
    srand(2020);
    BabSol = solver_solution();
    g_LB.store(0.0);
    g_num_nodes = 0;
    stopped = 0;
    diff = 0.0;
    alloc_globals(SP->n);

    TIME = wtime();
    NodeHeap heap;
    BabNode* root = new_node(nullptr);
    ++g_num_nodes;
    root_bound = Evaluate(root, SP, PP, 0);
    root->upper_bound = root_bound;
    auto branch = [&](const BabNode* node, double bound) {
        const int ic = getBranchingVariable(const_cast<BabNode*>(node));
        for (int xic = 0; xic <= 1; ++xic) {
            BabNode* child = new_node(node);
            child->xfixed[ic] = 1;
            child->sol.X[ic] = xic;
            child->upper_bound = bound;
            ++g_num_nodes;
            heap.push(child);
        }
    };
    if (Bab_LBGet() + 1.0 < root->upper_bound && !params.root) branch(root, root->upper_bound);
    free(root);

    struct Flight {
        long long ticket;
        std::vector<BabNode> nodes;
        std::vector<double> bounds;
    };
    std::vector<Flight> flight;
    int rc = 0;
    while (!heap.empty() || !flight.empty()) {
        if (params.time_limit > 0 && (wtime() - TIME) > params.time_limit) stopped = 1;
        while (!stopped && (int)flight.size() < depth && !heap.empty()) {
            Flight f;
            while ((int)f.nodes.size() < batch && !heap.empty()) {
                BabNode* nd = heap.pop();
                if (Bab_LBGet() + 1.0 < nd->upper_bound) f.nodes.push_back(*nd);
                free(nd);
            }
            if (f.nodes.empty()) continue;
            f.bounds.assign(f.nodes.size(), 0.0);
            f.ticket = bqb_fused_submit(f.nodes.data(), (int)f.nodes.size(), 1);
            if (f.ticket < 0) {
                rc = 2;
                break;
            }
            flight.push_back(std::move(f));
        }
        if (rc || flight.empty()) break;
        Flight f = std::move(flight.front());
        flight.erase(flight.begin());
        rc = bqb_fused_collect(f.ticket, f.nodes.data(), f.bounds.data());
        if (rc) break;
        for (size_t i = 0; i < f.nodes.size(); ++i) {
            f.nodes[i].upper_bound = f.bounds[i];
            if (!stopped && Bab_LBGet() + 1.0 < f.bounds[i]) branch(&f.nodes[i], f.bounds[i]);
        }
    }
    while (!heap.empty()) free(heap.pop());
    for (Flight& f : flight) bqb_fused_collect(f.ticket, f.nodes.data(), f.bounds.data());

    if (out) {
        out->best_value = Bab_LBGet();
        out->root_bound = root_bound;
        out->nodes = g_num_nodes;
        out->stopped = stopped;
        out->seconds = wtime() - TIME;
        out->num_vertices = num_vertices;
        for (int i = 0; i < BQB_NMAX; ++i) out->solution[i] = (i < BabPbSize) ? BabSol->X[i] : 0;
    }
    return rc;
}

// ---- B&B with the node pool on the device -------------------------------
// The root is bounded with rank 0 on the library globals (sets diff) as the
// reference's master does; its two children seed the device-resident pool
// (fused_pool_bab: nodek_kernel pops the open node with the largest parent
// bound, bounds it with rank 1, branches it (src/bab_functions.c:224-336)
// and pushes its children, all on the device).  Problems the fused kernel
// does not take (N0 > 128) go to bqb_solve_parallel.  `pool_nodes`: node
// records on the device (<= 0: 65536).
BQB_API int bqb_solve_device(const double* adj, int num_vertices, const BiqBinParameters* prm, int pool_nodes,
                             bqb_solve_result* out)
{
    if (num_vertices < 3 || num_vertices > BQB_NMAX) return 1;
    if (num_vertices > 128) return bqb_solve_parallel(adj, num_vertices, prm, 16, out);
    if (prm) {
        params = *prm;
    } else {
        bqb_default_params(&params);
        params.init_bundle_iter = 5;
        params.violated_TriIneq = 0.05;
    }
    std::vector<double> A(adj, adj + (size_t)num_vertices * num_vertices);
    process_adj_matrix(A.data(), num_vertices);
    if (params.adjust_TriIneq) params.TriIneq = SP->n * 10;
    srand(2020);
    BabSol = solver_solution();
    g_LB.store(0.0);
    g_num_nodes = 0;
    stopped = 0;
    diff = 0.0;
    alloc_globals(SP->n);

    TIME = wtime();
    BabNode* root = new_node(nullptr);
    g_num_nodes = 1;
    root_bound = Evaluate(root, SP, PP, 0);
    root->upper_bound = root_bound;
    std::vector<BabNode> open;
    if (Bab_LBGet() + 1.0 < root->upper_bound && !params.root) {
        const int ic = getBranchingVariable(root);
        for (int xic = 0; xic <= 1; ++xic) {
            BabNode child = *root;
            child.xfixed[ic] = 1;
            child.sol.X[ic] = xic;
            child.upper_bound = root->upper_bound;
            child.level = root->level + 1;
            open.push_back(child);
        }
    }
    free(root);
    int rc = 0;
    if (!open.empty()) {
        long long created = 0, evaluated = 0;
        int st = 0;
        const double budget = params.time_limit > 0 ? params.time_limit - (wtime() - TIME) : 0.0;
        rc = bqb::fused_pool_bab(open, pool_nodes > 0 ? pool_nodes : 65536, budget > 0 ? budget : 0.0, &created,
                            &evaluated, &st);
        g_num_nodes = 1 + (int)created;
        stopped = st;
    }
    if (out) {
        out->best_value = Bab_LBGet();
        out->root_bound = root_bound;
        out->nodes = g_num_nodes;
        out->stopped = stopped;
        out->seconds = wtime() - TIME;
        out->num_vertices = num_vertices;
        for (int i = 0; i < BQB_NMAX; ++i) out->solution[i] = (i < BabPbSize) ? BabSol->X[i] : 0;
    }
    return rc;
}
