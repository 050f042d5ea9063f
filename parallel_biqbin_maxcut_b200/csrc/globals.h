// Declarations of the reference's process globals (src/global_var.h:1-48,
// src/heap.c:7-8) as seen by this library, plus the export macro.
#pragma once
#include "../../include/bqb_gpu.h"

#define BQB_API extern "C" __attribute__((visibility("default")))

extern "C" {
extern BiqBinParameters params;
extern Problem* SP;
extern Problem* PP;
extern double* X;
extern double* Z;
extern double* X_bundle;
extern double* X_test;
extern double* dual_gamma;
extern double* dgamma;
extern double* gamma_test;
extern double* lambda;
extern double* eta;
extern double* F;
extern double* G;
extern double* g;
extern double f;
extern Triangle_Inequality* Cuts;
extern Triangle_Inequality* List;
extern Pentagonal_Inequality* Pent_Cuts;
extern Pentagonal_Inequality* Pent_List;
extern Heptagonal_Inequality* Hepta_Cuts;
extern Heptagonal_Inequality* Hepta_List;
extern int BabPbSize;
}
