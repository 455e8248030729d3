/* Test infrastructure (the oracle): CPU restatement of the reference's explicit-dynamics step.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it; the product library
 * (melody2d_b200/csrc) never links or calls it. */
#ifndef MEL_ORACLE_H
#define MEL_ORACLE_H
#include "melgpu.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_model orc_model;

/* Builds the model and runs the set-up of Code/main.cpp:104-127. n_regions[b] is the
 * NUMBER_REGIONS of each deformable body (Code/IO.h:1743-1755); NULL means 1 region. */
int  orc_create(const mel_model_desc* d, const int* n_regions, orc_model** out);
void orc_destroy(orc_model* m);
/* nsteps iterations of the solver + proximity cadence of Code/main.cpp:141-196. */
int  orc_step(orc_model* m, int nsteps, int run_proximity);
int  orc_update_proximity(orc_model* m);
double orc_time(orc_model* m);
double orc_dt(orc_model* m);
int  orc_n_contacts(orc_model* m);
int  orc_get_contacts(orc_model* m, mel_contact* out, int cap);
int  orc_set_contacts(orc_model* m, const mel_contact* c, int n);
/* 12 doubles per node, as mel_model_desc::node_state */
void orc_get_node_state(orc_model* m, double* st);
void orc_set_node_state(orc_model* m, const double* st);
void orc_get_positions(orc_model* m, double* xy);
/* force components [2*n_nodes]: internal, contact, neumann, dirichlet, total (any may be NULL) */
void orc_get_forces(orc_model* m, double* fint, double* fcon, double* fneu, double* fdir, double* ftot);
void orc_get_rigid(orc_model* m, double* rigid, double* rigid_forces);
void orc_set_rigid(orc_model* m, const double* rigid);
void orc_get_works(orc_model* m, double* works);
void orc_monitor(orc_model* m, mel_monitor* out);
/* neighbour list of every body: [body, body2, border2, shift] rows; returns the row count */
int  orc_get_neighbours(orc_model* m, int* rows, int cap);
/* counts Closest_2_segment calls that left the shape weights unset (stale values reused,
 * Code/Body.h:1347 declares them outside the contact loop) */
long orc_stale_shape_events(orc_model* m);
/* Time, Deltat and Next_contact_update (restart) */
void orc_set_time(orc_model* m, double time, double dt, double next_contact_update);
/* border contact pressures x, y per border entry (Update_contact_pressures, Code/Proximity.h:1014-1069) */
void orc_get_contact_pressures(orc_model* m, double* px, double* py);
/* Solver_step outputs of the last iteration: neval, max_error, mean_error, total_mass, max_mass */
void orc_solver_stats(orc_model* m, double* out5);
/* 0: x^(-1/2), cos and sin through glibc pow, cos and sin, as the reference (default);
 * 1: correctly rounded x^(-1/2), cos and sin, the values the GPU kernels compute (mel_rsqrt.h,
 *    mel_sincos.h). */
void orc_set_rsqrt_mode(int correctly_rounded);
/* body statuses (MEL_STATUS_*), which Update_status changes after proximity updates */
void orc_get_body_status(const orc_model* m, int* status);
/* Body::damage of every body, as Update_damage left it (0 until a Damage entry is evaluated) */
void orc_get_damage(orc_model* m, double* out);
/* the MATRICES stiffness and damping entries after the set-up (n_matrix each); 0 when there are none */
int orc_get_matrices(orc_model* m, double* k, double* c);
/* Body::Update_damage of body b (the Damage entry of Monitoring), returning the new damage */
double orc_update_damage(orc_model* m, int b);
/* Monitoring's Damage entries for the listed bodies: after every later step, before its proximity
 * update, Update_damage of each is logged (at most cap steps); orc_damage_log copies the log and
 * returns its steps */
void orc_monitor_damage(orc_model* m, const int* bodies, int n, int cap);
int orc_damage_log(orc_model* m, double* out);

#ifdef __cplusplus
}
#endif
#endif
