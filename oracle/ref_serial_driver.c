/*
 * Serial best-first branch-and-bound driver for the reference BiqBin C
 * sources (test infrastructure: the CPU oracle / CPU baseline, never the
 * GPU product).
 *
 * It replaces the reference's MPI process driver src/main.c:25-278 with one
 * process that plays both roles:
 *   - "master" part: Init_PQ evaluates the root with rank 0
 *     (src/bab_functions.c:39-69), then the root is branched into its two
 *     children exactly as src/main.c:129-162 does (Bab_incEvalNodes per
 *     child);
 *   - "worker" part: the reference's own worker_Bab_Main
 *     (src/bab_functions.c:224-332) is called with rank 1 until the local
 *     queue is empty; with the single-process MPI stub every "free worker"
 *     query answers 0, so all children stay in this queue.  Each branching
 *     adds two evaluated nodes, as the master counts them in
 *     src/bab_functions.c:199-200.
 *
 * Usage: bqb_ref_bab <instance.rudy> <params>
 * Environment: BQB_REF_SEED=<s> re-seeds rand() with s after Bab_Init's
 * srand(2020) (src/bab_functions.c:82), before the root is evaluated, to
 * sample the spread of the random parts (heuristic, k-gonal annealing).
 * Output: the reference's printFinalOutput block (src/bab_functions.c:351-371).
 */
#include <stdio.h>
#include <stdlib.h>

#include "biqbin.h"

extern Heap *heap;
extern BiqBinParameters params;
extern double TIME;
extern int stopped;
extern FILE *output;

/* defined by src/main.c in the MPI build */
int num_workers_used = 0;
int rank = 0;
int heuristic_counter = 0;

void abort_alloc_fail(int abort_code)
{
    MPI_Abort(MPI_COMM_WORLD, abort_code);
}

int main(int argc, char **argv)
{
    heap = Init_Heap(1000000);
    if (Bab_Init(argc, argv, 0))
        return 1;

    const char *seed = getenv("BQB_REF_SEED");
    if (seed) srand((unsigned)strtoul(seed, NULL, 10));

    TIME = MPI_Wtime();

    int over = Init_PQ();
    if (over != -1 && !params.root) {
        BabNode *node = Bab_PQPop();
        int ic = getBranchingVariable(node);
        for (int xic = 0; xic <= 1; ++xic) {
            BabNode *child = newNode(node);
            child->xfixed[ic] = 1;
            child->sol.X[ic] = xic;
            Bab_incEvalNodes();
            Bab_PQInsert(child);
        }
        free(node);

        while (!isPQEmpty()) {
            if (params.time_limit > 0 && (MPI_Wtime() - TIME) > params.time_limit) {
                stopped = 1;
                break;
            }
            int before = heap->used;
            worker_Bab_Main(0, 0, 1);
            if (heap->used == before + 1) { /* popped one, pushed two */
                Bab_incEvalNodes();
                Bab_incEvalNodes();
            }
        }
    }

    printFinalOutput(stdout, Bab_numEvalNodes());
    if (output) {
        printFinalOutput(output, Bab_numEvalNodes());
        fclose(output);
    }
    return 0;
}
