/*
 * ep2d_oracle.h -- CPU oracle for the EffPlast2D pseudo-transient solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's FP64
 * algorithm (beacon1143/EffPlast2D, EffPlast2D.cu) that tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg check results against.  The product
 * (effplast2d_b200, libep2d.so) never links or calls it.
 *
 * The API mirrors include/ep2d.h one to one (orc_* <-> ep2d_*) so that a test can
 * drive both with the same inputs and compare fields and records.
 */
#ifndef EP2D_ORACLE_H
#define EP2D_ORACLE_H

#include "../include/ep2d.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_state orc_state;

int orc_create(const ep2d_params* params, orc_state** out);
int orc_destroy(orc_state* s);
int orc_set_threads(int n);
int orc_iterate(orc_state* s, int64_t n_iter);
int orc_get_field(orc_state* s, int32_t field, double* out);
int orc_set_field(orc_state* s, int32_t field, const double* in);
int orc_solve_step(orc_state* s, int32_t step, double load_step_value, const double load_type[3],
                   int32_t n_time_steps, ep2d_step_record* out);
int orc_get_record(orc_state* s, int32_t step, int32_t time_step, ep2d_step_record* out);
int orc_get_check_errors(orc_state* s, int32_t step, int32_t time_step, double* errors_out,
                         int32_t max_n, int32_t* n_out);
int orc_compute_eff_damping(orc_state* s, double init_load_value, const double load_type[3],
                            int32_t n_time_steps, double load_value, int64_t* total_iterations);
int orc_compute_eff_moduli(orc_state* s, double init_load_value, const double load_type[3],
                           int32_t n_time_steps, ep2d_result* out);
/* SaveAnStatic2D (EffPlast2D.cu:1060-1292).  Numerical fields always; the analytic
 * fields and error maps are written only when nPores == 1 (pointers may be NULL
 * otherwise).  stats[6] = Uabs max, avg, J1 max, avg, J2 max, avg (NaN if N != 1). */
int orc_static_fields(orc_state* s, double delta_p, double tau_infty,
                      double* unu_abs, double* j1nu, double* j2nu,
                      double* uan_abs, double* error_uabs, double* j1an, double* j2an,
                      double* error_j1, double* error_j2, double stats[6]);
/* kernel-level pore masks as evaluated by ComputeStress (EffPlast2D.cu:77-97):
 * node mask nx*ny and corner mask (nx-1)*(ny-1), 1 = inside a pore */
int orc_get_masks(orc_state* s, uint8_t* node_mask, uint8_t* corner_mask);
/* get_sigma_2D.m's plastic zone: on = 1 clears Plast/PlastXY and marks, from then on,
 * every node / corner whose trial J2 exceeds coh at any iteration (:126-138); 0 stops. */
int orc_track_plastic_zone(orc_state* s, int32_t on);
/* get_sigma_2D.m:170-194 with that zone: polar stresses (numerical snrr/snff, analytic
 * sarr/saff) and the Plast count per node. */
int orc_polar_fields(orc_state* s, double load_value, double* snrr, double* snff, double* sarr, double* saff,
                     uint8_t* count_out);

#ifdef __cplusplus
}
#endif
#endif
