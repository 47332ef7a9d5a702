/*
 * amrlbm_oracle.h - C interface of the CPU oracle (test infrastructure only).
 *
 * The oracle is a line-by-line C++/OpenMP restatement of the hot path of
 * AMR-LBM-OpenMP-2D (GPL-3.0, A. Fakhari). Only tests/, the smoke check of
 * __graft_entry__.py and the CPU-baseline leg of bench.py may load it; the
 * product library never does.
 *
 * PARITY UNPINNED: the reference ships no tests, fixtures or golden vectors,
 * and it is Fortran 90 with no Fortran compiler on this machine or on the GPU
 * machines, so the restatement cannot be checked against the reference's own
 * outputs. It is checked against known answers derived from the reference's
 * formulas (tests/test_oracle_kat.py) and invariants.
 */
#ifndef AMRLBM_ORACLE_H
#define AMRLBM_ORACLE_H

#include <stdint.h>
#include "amrlbm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

orc_sim* orc_create(const amrlbm_params* p, int nthreads);
void orc_destroy(orc_sim* s);
void orc_set_threads(orc_sim* s, int nthreads);
int orc_last_error(const orc_sim* s);       /* sticky AMRLBM_ERR_* code      */
int orc_level_jump_count(const orc_sim* s); /* "Error in SUB_Fill_*" prints  */
void orc_physics(const orc_sim* s, amrlbm_physics* out);
void orc_set_physics(orc_sim* s, const amrlbm_physics* ph);

/* driver */
int orc_init_rising_bubble(orc_sim* s);
int orc_init_fields(orc_sim* s);
int orc_step(orc_sim* s, int nsteps);
/* seconds spent per phase so far, in the order of Main_Loop's timer printout
 * (AMR_Rising_2D_OMP.f90:366-375): Macroscopic_h, Macroscopic_g, collision,
 * advection, Ghost_C, Ghost_C2, Ghost_hg, refine */
void orc_phase_times(const orc_sim* s, double out[8]);

/* Main_Loop phases */
void orc_min_max_levels(orc_sim* s);
void orc_set_level_range(orc_sim* s, int lmin, int lmax);
void orc_fill_c2(orc_sim* s);
void orc_collide(orc_sim* s);
void orc_fill_hg(orc_sim* s);
void orc_stream(orc_sim* s);
void orc_macro_h(orc_sim* s);
void orc_fill_c(orc_sim* s);
void orc_macro_g(orc_sim* s);
int orc_regrid(orc_sim* s, double refin_tol, double deref_tol);

/* state */
void orc_counts(const orc_sim* s, int32_t out[5]);
int orc_get_topology(const orc_sim* s, int32_t* level, int32_t* dx, int32_t* bi,
                     int32_t* bj, int32_t* parent, int32_t* child, int32_t* nbr_owner,
                     int32_t* nbr_slot, uint8_t* flags, int32_t* n_free,
                     int32_t* free_list);
int orc_set_topology(orc_sim* s, int32_t nblks, const int32_t* level, const int32_t* dx,
                     const int32_t* bi, const int32_t* bj, const int32_t* parent,
                     const int32_t* child, const int32_t* nbr_owner,
                     const int32_t* nbr_slot, const uint8_t* flags, int32_t n_free,
                     const int32_t* free_list, int32_t kk);
int orc_get_neighbours(const orc_sim* s, int32_t* nbr);
int orc_get_leaves(const orc_sim* s, int32_t* leaves);
int orc_get_block(const orc_sim* s, int id, double* h, double* g, double* C, double* P,
                  double* Ux, double* Uy);
int orc_set_block(orc_sim* s, int id, const double* h, const double* g, const double* C,
                  const double* P, const double* Ux, const double* Uy);
int orc_block_error(const orc_sim* s, int id, double* err);
int orc_diag(const orc_sim* s, double out[8]);

/* single routines on caller arrays (reference layouts), for unit tests */
void orc_collision_block(const orc_sim* s, int dx, const double* C, const double* P,
                         const double* Ux, const double* Uy, double* h, double* g);
void orc_macro_g_block(const orc_sim* s, int dx, const double* g, const double* C,
                       double* P, double* Ux, double* Uy);
void orc_stream_block(const orc_sim* s, int dx, double* f);
void orc_biquadratic_from_fine(int i2, int j2, int X2, int Y2, const double* cin,
                               double* cout);
void orc_biquadratic_from_coarse(int I2, int J2, int x2, int y2, const double* cin,
                                 double* cout);
void orc_bilinear_from_fine(int i2, int j2, int X2, int Y2, const double* cin,
                            double* cout);
void orc_mrt(double s9, const double* geq, double* g);
void orc_equilibrium(const orc_sim* s, double C, double U, double V, double ni,
                     double nj, double* gamma, double* heq);

#ifdef __cplusplus
}
#endif

#endif
