/*
 * Component-oracle shim for the reference BiqBin C sources (test
 * infrastructure only).  Linked together with the reference objects into
 * oracle/_ref/libbqb_ref.so so that tests can call the reference's own
 * ipm_mc_pk, op_B, op_Bt, fct_eval, getViolated_TriangleInequalities,
 * runHeuristic_unpacked, mc_1opt, solve_lambda, lambda_eta, bundle_method,
 * SDPbound ... on inputs chosen by the test, through ctypes.
 *
 * The reference keeps its state in globals (src/global_var.h:1-48) that
 * allocMemory (src/allocate_free.c:8-42) sizes from SP->n; this shim builds
 * SP/PP from an adjacency matrix with the reference's own process_adj_matrix
 * (src/process_input.c:259-344), applies the parameter defaults of the
 * PARAM_FIELDS table (src/biqbin.h:49-78) and the adjust_TriIneq rule
 * (src/process_input.c:135-136), and allocates the globals.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "biqbin.h"

extern BiqBinParameters params;
extern Problem *SP;
extern Problem *PP;
extern int BabPbSize;
extern double diff;

int num_workers_used = 0;
int rank = 0;
int heuristic_counter = 0;

void abort_alloc_fail(int abort_code)
{
    MPI_Abort(MPI_COMM_WORLD, abort_code);
}

/* Reset every parameter to its PARAM_FIELDS default. */
void bqbref_params_default(void)
{
#define P(type, name, format, def_value) params.name = def_value;
    PARAM_FIELDS
#undef P
}

/* Set one parameter by name (ints and doubles share this entry).
 * Returns 0 on success, 1 if the name is unknown. */
int bqbref_param_set(const char *name, double value)
{
#define P(type, pname, format, def_value)                 \
    if (strcmp(#pname, name) == 0) {                      \
        params.pname = (type)value;                       \
        return 0;                                         \
    }
    PARAM_FIELDS
#undef P
    return 1;
}

double bqbref_param_get(const char *name)
{
#define P(type, pname, format, def_value)                 \
    if (strcmp(#pname, name) == 0)                        \
        return (double)params.pname;
    PARAM_FIELDS
#undef P
    return -1.0;
}

/* Build SP/PP from a dense adjacency matrix (num_vertices^2, symmetric,
 * integer weights) and allocate the reference globals.  Parameters are the
 * values currently in `params`; adjust_TriIneq is applied here as in
 * processCommandLineArguments. */
int bqbref_setup(double *adj, int num_vertices)
{
    int err = process_adj_matrix(adj, num_vertices);
    if (err)
        return err;
    if (params.adjust_TriIneq)
        params.TriIneq = SP->n * 10;
    initializeBabSolution();
    allocMemory();
    diff = 0.0;
    return 0;
}

void bqbref_teardown(void)
{
    freeMemory();
}

int bqbref_babpbsize(void) { return BabPbSize; }

/* Force the global lower bound (B&B incumbent value) for SDPbound tests. */
void bqbref_set_lb(double lb)
{
    BabSolution bs;
    memset(&bs, 0, sizeof(bs));
    Bab_LBUpd(lb, &bs);
}

void bqbref_set_diff(double d) { diff = d; }
double bqbref_get_diff(void) { return diff; }

size_t bqbref_sizeof_babnode(void) { return sizeof(BabNode); }
