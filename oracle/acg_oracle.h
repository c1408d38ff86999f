/*
 * acg_oracle — CPU restatement of the reference's MD timestep.
 * TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg, to check results against; never linked into
 * the product.
 *
 * One FP64 system at a time, single process, following the reference's
 * operation order so that, for boxes with at least 3 cells per dimension, the
 * results are bit-identical to the reference compiled from its own sources
 * (tests pin this).  For boxes with fewer cells the reference's neighbour-cell
 * map repeats cells and counts pairs twice (MDcode/cell_list+forces.c:37-49);
 * the restatement visits each distinct neighbour cell once instead.
 */
#ifndef ACG_ORACLE_H
#define ACG_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_sys ora_sys;

/* list_mode 0: keep pairs with r < 2.85 for every type pair (the reference's
 * Cell_cut, MDcode/global.h:30); 1: keep pairs with r < 2.5*sigma_ab + skin.
 * rebuild_factor: rebuild when factor * maxD^2 > skin^2 (the reference uses 3,
 * MDcode/time_evolve.c:508). */
ora_sys *ora_create(int n, int nact, double L, double T, double f0, int tau_p_steps,
                    double rebuild_factor, int list_mode);
void ora_destroy(ora_sys *s);
void ora_set_state(ora_sys *s, const double *x, const double *xu, const double *p,
                   const int *type, const int *act_tag);
void ora_get_state(const ora_sys *s, double *x, double *xu, double *p, double *F);
void ora_set_k(ora_sys *s, const int *k);
void ora_get_k(const ora_sys *s, int *k);
void ora_set_nhc(ora_sys *s, const double *eta, const double *p_eta);
void ora_get_nhc(const ora_sys *s, double *out9);
void ora_set_thermostat(ora_sys *s, double T);
void ora_seed_rng(ora_sys *s, unsigned long seed);
void ora_shuffle(ora_sys *s);
void ora_rebuild(ora_sys *s);
void ora_forces(ora_sys *s, double *F, double *out3);
int ora_run(ora_sys *s, long start, int nsteps, int do_shuffle, int do_drift);
void ora_fix_drift(ora_sys *s);
double ora_adjust_temp(ora_sys *s, double T);
long ora_ramp(ora_sys *s, double T_start, double T_end, double rate);
int ora_run_nve(ora_sys *s, int nsteps);
void ora_get_scalars(const ora_sys *s, double *out6);
int ora_get_cells(const ora_sys *s, int *dims, int *counts, int *members);
long ora_get_neighbors(const ora_sys *s, int *counts, int *pairs);

void ora_cell_geometry(double L, int *nc3, double *inv3);
int ora_log_schedule(unsigned long long run_length, int num_origins, double factor,
                     unsigned long long *out, int cap);

#ifdef __cplusplus
}
#endif
#endif
