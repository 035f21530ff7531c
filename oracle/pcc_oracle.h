/*
 * Plain-C restatement of the reference simulator's per-timestep collision
 * path at one rank -- the CPU oracle the device library is checked against.
 *
 * Test infrastructure: only tests/, the smoke check and the CPU-baseline leg
 * of bench.py load the library built from this file.  The operation order of
 * every floating-point expression follows the reference source cited at each
 * function (file:line inside code/cpp/src of the reference project), with
 * PETSc's sequential kernels for the matrix/vector products, so that a strict
 * IEEE build of this file and a strict build of the reference itself agree
 * bit for bit.
 */
#ifndef PCC_ORACLE_H
#define PCC_ORACLE_H

#include <stddef.h>

#include "pcc_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pcco_colony pcco_colony;

pcco_colony* pcco_create(const pcc_params* p);
void pcco_destroy(pcco_colony* c);
const char* pcco_last_error(pcco_colony* c);
int pcco_set_cells(pcco_colony* c, const pcc_cells* cells, size_t n);
int pcco_get_cells(pcco_colony* c, pcc_cells* out, size_t cap, size_t* n);
int pcco_solve(pcco_colony* c, double dt, int iter, pcc_step_stats* st);
int pcco_step(pcco_colony* c, pcc_step_stats* st);
int pcco_run(pcco_colony* c, double end_radius, long long max_steps, long long* steps_done, double* cell_steps,
             pcc_step_stats* last);
int pcco_detect(pcco_colony* c, double tol, int phase, pcc_contacts* out, size_t cap, size_t* n);
int pcco_get_constraints(pcco_colony* c, pcc_contacts* out, size_t cap, size_t* n);
double pcco_get_dt(pcco_colony* c);
void pcco_set_dt(pcco_colony* c, double dt);
double pcco_colony_radius(pcco_colony* c);
unsigned long long pcco_division_count(pcco_colony* c);
unsigned int pcco_division_seed(unsigned long long seed, unsigned long long k);
double pcco_division_length(unsigned long long seed, unsigned long long k, double len);

#ifdef __cplusplus
}
#endif

#endif
