/*
 * seren_oracle.h - TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the SEREN grad-h SPH force hot path, used by
 * tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the checker.
 * It is never linked into or called by the product library.
 *
 * Parity status: UNPINNED.  The reference ships no golden vectors, known-answer
 * tests or fixtures for this path (its src/tests and testsuite/ directories are
 * absent), and it is Fortran 90 with no Fortran compiler on either machine, so
 * it cannot be run to generate any.  This restatement follows the cited Fortran
 * line by line (same expression association, no FMA contraction, libm pow) and
 * is cross-checked by physical invariants in the tests.
 *
 * The entry points mirror include/seren_gpu.h one for one (same arguments,
 * same id base, same error codes) so a test can run both on the same inputs.
 */
#ifndef SEREN_ORACLE_H
#define SEREN_ORACLE_H

#include <stdint.h>
#include "../include/seren_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct seren_oracle seren_oracle;

/* Interaction counters of the last call of each stage (instrumentation used by
 * the roofline flop model; ids as in the field names). */
typedef struct {
  int64_t grav_cells;        /* cell (monopole+quadrupole) terms          */
  int64_t grav_pairs;        /* gravity_gradh / gravity_meanh pair terms  */
  int64_t grav_nodes;        /* cells visited by the gravity walks        */
  int64_t gradh_tests;       /* candidate distance tests, iteration passes*/
  int64_t gradh_pairs;       /* accepted pairs, iteration passes          */
  int64_t gradh_passes;      /* density passes (iterations) in total      */
  int64_t gradh_walks;       /* hgather walks                             */
  int64_t gradh_final_tests; /* candidate tests, final pass               */
  int64_t gradh_final_pairs; /* accepted pairs, final pass                */
  int64_t neib_tests;        /* get_neib candidate tests                  */
  int64_t neib_pairs;        /* neighbours found (sum of pptot)           */
  int64_t hydro_pairs;       /* hydro pairs inside either kernel          */
  int64_t hydro_visc;        /* of which with dv.dr < 0 (viscosity)       */
  int64_t gradh_bisections;  /* particles whose iteration reached the
                                bisection (all_sph_gradh.F90:256-260)     */
} seren_oracle_counts;

int seren_oracle_create(seren_oracle** o, int64_t pmax, const seren_gpu_params* prm);
void seren_oracle_destroy(seren_oracle* o);
int seren_oracle_last_error(seren_oracle* o, char* buf, int32_t len);
int seren_oracle_set_threads(int32_t nthreads);

int seren_oracle_tree_update(seren_oracle* o, int32_t ptot, double* parray,
                             int32_t do_build, int32_t do_reorder, int32_t* perm_out);
int seren_oracle_sph_update(seren_oracle* o, int32_t ptot, const int32_t* acclist,
                            int32_t nacc, double* parray, const double* v, double* rho,
                            double* omega, double* div_v, double* drhodt, int32_t* pptot,
                            int32_t* pplist, int32_t first_call);
int seren_oracle_get_neib(seren_oracle* o, int32_t ptot, const int32_t* acclist,
                          int32_t nacc, const double* h, int32_t* pptot, int32_t* pplist);
int seren_oracle_h_gather(seren_oracle* o, int32_t ptot, const int32_t* acclist, int32_t nacc,
                          double* parray);
int seren_oracle_hydro_forces(seren_oracle* o, const int32_t* acclist, int32_t nacc,
                              const double* press, const double* sound, double* a);
int seren_oracle_grav_forces(seren_oracle* o, const int32_t* acclist, int32_t nacc,
                             double* a, double* gpot, int32_t nsink, const double* sink_rmh);
int seren_oracle_sink_forces(seren_oracle* o, int32_t nsink, const double* sink_rmh,
                             double* sink_a, double* sink_gpot);
/* direct_sph_gravity (sph/direct_sph_gravity.F90:64-79) for the particles in
 * ids[n]: a[n][3], gpot[n], O(n*ptot). */
int seren_oracle_direct_gravity(seren_oracle* o, const int32_t* ids, int32_t n,
                                double* a, double* gpot);
int seren_oracle_tree_export(seren_oracle* o, int32_t* ctot, int32_t* ltot, int32_t* leaf,
                             int32_t* nextcell, int32_t* ifopen, int32_t* plist,
                             int32_t* first_cell, int32_t* last_cell, double* grav_r,
                             double* grav_m, double* grav_q, double* dminsqd,
                             double* hydro_r, double* rmax, double* hrangemax);
int seren_oracle_get_counts(seren_oracle* o, seren_oracle_counts* out);
/* Kernel tables (setup/kernel.F90): tab[9][KERNTOT+1] = w0,w1,w2,w3,w4,w5,w6,wh,wg */
int seren_oracle_kernel_tables(int32_t kernel, double* tab);
/* Per-stage wall seconds of the last call sequence, in the reference's timing
 * marker order: BH_TREE, ALL_SPH_GRADH, BHHYDRO_UPDATE, GET_NEIB, HYDRO_FORCES,
 * GRAVITY_FORCES. */
int seren_oracle_stage_seconds(seren_oracle* o, double* sec /*[6]*/);

#ifdef __cplusplus
}
#endif

#endif
