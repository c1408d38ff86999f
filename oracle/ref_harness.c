/*
 * Reference harness — TEST INFRASTRUCTURE ONLY (results are checked against it; never the product).
 *
 * This file is compiled together with the reference MD engine's own sources
 * (MDcode/*.c, built in place by oracle/Makefile with a single-rank MPI shim
 * and a GSL shim) into oracle/_ref/libref_md_n<N>.so.  It drives the
 * reference's globals directly — the reference has no function arguments
 * anywhere (MDcode/global.h:81-162) — so the tests can hand the reference an
 * exact state and read back what its own routines computed:
 *
 *   ref_setup          state -> sphere[], SetUpParallel/SetUpCellList
 *                      (MDcode/Parallel.c:6-106), CommunicateCoordinates(0),
 *                      update_cell_list (MDcode/cell_list+forces.c:58-148),
 *                      calculate_forces
 *   ref_forces         calculate_forces (MDcode/cell_list+forces.c:153-227)
 *   ref_run            run() loop body (MDcode/main.c:244-248): ShuffleActDirec
 *                      every TAU_per steps + AdvanceTimeNVTNoseHoover
 *                      (MDcode/time_evolve.c:495-526)
 *   ref_run_nve        advance_time_NVEFrog (MDcode/time_evolve.c:104-171)
 *   ref_get_cells      InCellCount / InCell after the last rebuild
 *   ref_log_schedule   prepareSavingArray (MDcode/main.c:62-119)
 *   ref_write_restart  write_restart_state (MDcode/main.c:272-288)
 *
 * Seeds: time() is wrapped (-Wl,--wrap=time) to a settable constant so the
 * reference's time-derived seeds are reproducible here.
 */
#include "global.h"
#include "subroutine.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

extern unsigned long long int *nextStepIndex; /* MDcode/main.c:4 */
void prepareSavingArray(unsigned long long int runLength, int numOfOrigins, double factor);
void write_restart_state(char *outFileName, int iter, int last_saved_index);

static time_t fake_time = 1700000000;
time_t __wrap_time(time_t *t) {
  if (t) *t = fake_time;
  return fake_time;
}
void ref_set_time(long t) { fake_time = (time_t)t; }

static int arrays_ready = 0;

/* In the reference program built with the drop-in files (the timestep on the
 * GPU), the harness's direct reads and writes of the reference's globals go
 * through the drop-in's host mirror: refresh before reading sphere[], report
 * edits.  Absent (null) in the reference's own build. */
void acg_legacy_sync_host(void) __attribute__((weak));
void acg_legacy_host_touched(void) __attribute__((weak));
static void mirror_read(void) {
  if (acg_legacy_sync_host) acg_legacy_sync_host();
}
static void mirror_written(void) {
  if (acg_legacy_host_touched) acg_legacy_host_touched();
}

int ref_n(void) { return N; }
int ref_nact(void) { return Nact; }
int ref_tau_per(void) { return TAU_per; }
int ref_max_cells(void) { return MaxCells; }

void ref_seed_rng(unsigned long seed) {
  if (!rng_ptr) rng_ptr = gsl_rng_alloc(gsl_rng_mt19937);
  gsl_rng_set(rng_ptr, seed);
}

/* x, xu, p: [N][3] (reduced wrapped, reduced unfolded, momenta);
 * act_tag[N] (-1 or index into k); k: [3][Nact] = kx, ky, kz. */
void ref_setup(double Lbox, double Tset, double f0set, const double *x, const double *xu,
               const double *p, const int *type, const int *act_tag, const int *k) {
  node = 0;
  Nprocs = 1;
  L = Lbox;
  inv_L = 1.0 / L;
  T = Tset;
  f0 = f0set;
  DENSITY = (double)N / (L * L * L);
  if (!xold) {
    xold = calloc(N, sizeof(double));
    yold = calloc(N, sizeof(double));
    zold = calloc(N, sizeof(double));
  }
  for (int i = 0; i < N; i++) {
    sphere[i].x = x[3 * i];
    sphere[i].y = x[3 * i + 1];
    sphere[i].z = x[3 * i + 2];
    sphere[i].x_u = xu ? xu[3 * i] : x[3 * i];
    sphere[i].y_u = xu ? xu[3 * i + 1] : x[3 * i + 1];
    sphere[i].z_u = xu ? xu[3 * i + 2] : x[3 * i + 2];
    sphere[i].px = p[3 * i];
    sphere[i].py = p[3 * i + 1];
    sphere[i].pz = p[3 * i + 2];
    sphere[i].Fx = sphere[i].Fy = sphere[i].Fz = 0.0;
    sphere[i].type = type[i];
    sphere[i].actTag = act_tag[i];
    if (act_tag[i] >= 0 && act_tag[i] < Nact) activeParticleIndex[act_tag[i]] = i;
  }
  for (int a = 0; a < Nact; a++) {
    kx[a] = k[a];
    ky[a] = k[Nact + a];
    kz[a] = k[2 * Nact + a];
  }
  mirror_written();
  if (!arrays_ready) {
    GetDataTypeSLAB();
    GetDataTypeSLABF();
    AllocateArrays();
    arrays_ready = 1;
  }
  SetUpParallel();
  SetUpCellList();
  CommunicateCoordinates(0);
  update_cell_list();
  calculate_forces(); /* as initialise_restart_state (MDcode/main.c:331-332) */
}

void ref_set_k(const int *k) {
  for (int a = 0; a < Nact; a++) {
    kx[a] = k[a];
    ky[a] = k[Nact + a];
    kz[a] = k[2 * Nact + a];
  }
  mirror_written();
}
void ref_get_k(int *k) {
  for (int a = 0; a < Nact; a++) {
    k[a] = kx[a];
    k[Nact + a] = ky[a];
    k[2 * Nact + a] = kz[a];
  }
}

/* the rebuild branch of AdvanceTimeNVTNoseHoover (MDcode/time_evolve.c:508-512) */
void ref_rebuild(void) {
  ExchangeParticlesInBlocks();
  CommunicateCoordinates(0);
  update_cell_list();
}

/* out: pe (peblk), virial (virialblk, already /3), vir_act (vir_actblk) */
void ref_forces(double *F, double *out) {
  calculate_forces();
  for (int i = 0; i < N; i++) {
    F[3 * i] = sphere[i].Fx;
    F[3 * i + 1] = sphere[i].Fy;
    F[3 * i + 2] = sphere[i].Fz;
  }
  out[0] = peblk;
  out[1] = virialblk;
  out[2] = vir_actblk;
}

void ref_init_nhc(void) { InitialiseNoseHoover(); }
void ref_set_nhc(const double *eta_in, const double *p_eta_in) {
  tau = 0.20;
  for (int i = 0; i < M; i++) q[i] = T * tau * tau;
  q[0] = DOF * T * tau * tau;
  for (int i = 0; i < M; i++) {
    eta[i] = eta_in[i];
    p_eta[i] = p_eta_in[i];
  }
}
void ref_get_nhc(double *out) {
  mirror_read();
  for (int i = 0; i < M; i++) {
    out[i] = eta[i];
    out[M + i] = p_eta[i];
    out[2 * M + i] = q[i];
  }
}

/* run() body (MDcode/main.c:244-265) for steps [start, start+nsteps):
 * ShuffleActDirec every TAU_per steps, the step, and (do_drift) fixDrift after
 * every 100000th step.  Returns the number of steps that rebuilt the
 * cell/neighbour lists, i.e. took the 3*maxmaxD > skin^2 branch
 * (MDcode/time_evolve.c:508). */
/* the drop-in build's count of list rebuilds (its step leaves maxmaxD and the
 * other scalars to the next sync point); weak, absent from the reference build */
long long acg_legacy_rebuilds(void) __attribute__((weak));

int ref_run(long start, int nsteps, int do_shuffle, int do_drift) {
  int rebuilds = 0;
  const long long r0 = acg_legacy_rebuilds ? acg_legacy_rebuilds() : 0;
  for (long i = start; i < start + nsteps; i++) {
    if (do_shuffle && !(i % TAU_per)) ShuffleActDirec();
    AdvanceTimeNVTNoseHoover();
    if (!acg_legacy_rebuilds && 3.0 * maxmaxD > skin * skin) rebuilds++;
    if (do_drift && i % 100000 == 0) fixDrift();
  }
  if (acg_legacy_rebuilds) rebuilds = (int)(acg_legacy_rebuilds() - r0);
  return rebuilds;
}

/* fixDrift (MDcode/initialise.c:104-138) */
void ref_fix_drift(void) { fixDrift(); }

/* advance_time_NVT_Berendsen (MDcode/time_evolve.c:173-256), nsteps times; a
 * weak reference: the drop-in build does not provide it (returns -1 there) */
void advance_time_NVT_Berendsen(void) __attribute__((weak));
int ref_run_berendsen(int nsteps) {
  if (!advance_time_NVT_Berendsen) return -1;
  for (int i = 0; i < nsteps; i++) advance_time_NVT_Berendsen();
  return 0;
}

/* AdvanceTimeNVTGaussOSM (MDcode/time_evolve.c:351-470), nsteps times; weak
 * like the Berendsen step */
void AdvanceTimeNVTGaussOSM(void) __attribute__((weak));
int ref_run_gauss(int nsteps) {
  if (!AdvanceTimeNVTGaussOSM) return -1;
  for (int i = 0; i < nsteps; i++) AdvanceTimeNVTGaussOSM();
  return 0;
}

/* advance_time_NPT (MDcode/time_evolve.c:258-348), nsteps times at target
 * pressure Pset; weak like the Berendsen step */
void advance_time_NPT(void) __attribute__((weak));
int ref_run_npt(int nsteps, double Pset) {
  if (!advance_time_NPT) return -1;
  P = Pset;
  for (int i = 0; i < nsteps; i++) advance_time_NPT();
  return 0;
}

/* Nose-Hoover NPT state as InitialiseNoseHooverNPT (MDcode/time_evolve.c:614-652)
 * leaves it, with the chain momenta given instead of drawn: tau = 0.2,
 * tau_baro = 2, L0 = L, eps = 0, the masses from T */
void ref_set_npt(const double *eta_in, const double *p_eta_in, const double *eta_baro_in,
                 const double *p_eta_baro_in, double p_eps_in) {
  tau = .20;
  tau_baro = 2.0;
  L0 = L;
  w_eps = DOF * T * tau_baro * tau_baro;
  eps = 0.0;
  for (int i = 0; i < M; i++) {
    q[i] = T * tau * tau;
    eta[i] = eta_in[i];
    p_eta[i] = p_eta_in[i];
    q_baro[i] = T * tau_baro * tau_baro;
    eta_baro[i] = eta_baro_in[i];
    p_eta_baro[i] = p_eta_baro_in[i];
  }
  q[0] = DOF * T * tau * tau;
  p_eps = p_eps_in;
}

/* AdvanceTimeNPTNoseHoover (MDcode/time_evolve.c:654-696), nsteps times at
 * target pressure Pset */
void AdvanceTimeNPTNoseHoover(void) __attribute__((weak));
int ref_run_nhc_npt(int nsteps, double Pset) {
  if (!AdvanceTimeNPTNoseHoover) return -1;
  P = Pset;
  for (int i = 0; i < nsteps; i++) AdvanceTimeNPTNoseHoover();
  return 0;
}

/* out: eps, p_eps, eta_baro[3], p_eta_baro[3], eta[3], p_eta[3] */
void ref_get_npt(double *out) {
  out[0] = eps;
  out[1] = p_eps;
  for (int i = 0; i < 3; i++) {
    out[2 + i] = eta_baro[i];
    out[5 + i] = p_eta_baro[i];
    out[8 + i] = eta[i];
    out[11 + i] = p_eta[i];
  }
}

/* advance_time_ActiveBrown_PC (MDcode/time_evolve.c:855-974) with the
 * random forces given instead of drawn: the library is linked with
 * --wrap=normal, so normal() as called from time_evolve.c returns the step's
 * value for particle InBlock[node][k/3], component k%3 (k = the call count
 * within the step) from noise[step][particle][3]; without a buffer it draws
 * as the program does.  The constants are initializeOverDampedBD's
 * (MDcode/initialise.c:287-291). */
double __real_normal(double mean, double sigma);
static const double *noise_buf;
static long noise_k, noise_step;
double __wrap_normal(double mean, double sigma) {
  if (!noise_buf) return __real_normal(mean, sigma);
  const long k = noise_k++;
  const int part = InBlock[node][k / 3];
  return mean + sigma * noise_buf[((size_t)noise_step * N + part) * 3 + k % 3];
}
void advance_time_ActiveBrown_PC(void) __attribute__((weak));
int ref_run_brown(int nsteps, const double *noise) {
  if (!advance_time_ActiveBrown_PC) return -1;
  SqrtVariance = sqrt(2.0 * T * T / (time_step * D0));
  InvD0 = 1.0 / D0;
  D0ByT = D0 / T;
  TByD0 = T / D0;
  expFactor = exp(-time_step * TByD0);
  noise_buf = noise;
  for (int s = 0; s < nsteps; s++) {
    noise_k = 0;
    noise_step = s;
    advance_time_ActiveBrown_PC();
  }
  noise_buf = NULL;
  return 0;
}

/* out: L, inv_L, DENSITY */
void ref_get_box(double *out) {
  out[0] = L;
  out[1] = inv_L;
  out[2] = DENSITY;
}

/* one NVT step composed from the propagators, as AdvanceTimeNVTNoseHoover's
 * body does (MDcode/time_evolve.c:495-526) */
void ref_step_propagators(void) {
  U4Propagator(time_step * 0.25, M - 1, 0);
  U3Propagator(time_step * 0.50);
  U4Propagator(time_step * 0.25, 0, M - 1);
  U2Propagator();
  U1Propagator();
  if (3.0 * maxmaxD > skin * skin) {
    ExchangeParticlesInBlocks();
    CommunicateCoordinates(0);
    update_cell_list();
  } else {
    CommunicateCoordinates(1);
  }
  calculate_forces();
  U2Propagator();
  U4Propagator(time_step * 0.25, M - 1, 0);
  U3Propagator(time_step * 0.50);
  U4Propagator(time_step * 0.25, 0, M - 1);
  ke = ke * 0.5;
  inst_T = 2.0 * ke / DOF;
}

/* adjustInitialTemp (MDcode/initialise.c:141-151); returns inst_T after */
double ref_adjust_temp(double Tset) {
  adjustInitialTemp(Tset);
  return inst_T;
}

/* coldstart / breakxal (MDcode/initialise.c:166-201) with the reference's
 * global T left at final_temp afterwards, as they leave it */
void ref_coldstart(double rate, double final_temp) { coldstart(rate, final_temp); }
void ref_breakxal(double rate, double final_temp) { breakxal(rate, final_temp); }

/* initializeSystem (MDcode/initialise.c:203-227) as main() runs it for a fresh
 * start (MDcode/main.c:462-472): box from N and the density, srand(srand_seed),
 * then the random lattice, the active particles, coldstart and breakxal at T.
 * dir receives the files the routine writes (ini.dat, ActiveFileIndex.dat). */
int ref_initialize_system(double density, double Tset, double f0set, int job, unsigned int srand_seed,
                          const char *dir) {
  /* initializeSystem allocates the reference's arrays, once per process */
  if (arrays_ready) return -1;
  node = 0;
  Nprocs = 1;
  jobno = job;
  DENSITY = density;
  T = Tset;
  f0 = f0set;
  snprintf(sub_dir, sizeof(sub_dir), "%s", dir);
  L = pow((double)N / DENSITY, 0.33333333);
  inv_L = 1.0 / L;
  if (!xold) {
    xold = calloc(N, sizeof(double));
    yold = calloc(N, sizeof(double));
    zold = calloc(N, sizeof(double));
  }
  srand(srand_seed);
  initializeSystem();
  arrays_ready = 1;
  return 0;
}

int ref_run_nve(int nsteps) {
  int rebuilds = 0;
  for (int i = 0; i < nsteps; i++) {
    advance_time_NVEFrog();
    if (3.0 * maxmaxD > skin * skin) rebuilds++;
  }
  return rebuilds;
}

void ref_get_state(double *x, double *xu, double *p, double *F) {
  mirror_read();
  for (int i = 0; i < N; i++) {
    if (x) {
      x[3 * i] = sphere[i].x;
      x[3 * i + 1] = sphere[i].y;
      x[3 * i + 2] = sphere[i].z;
    }
    if (xu) {
      xu[3 * i] = sphere[i].x_u;
      xu[3 * i + 1] = sphere[i].y_u;
      xu[3 * i + 2] = sphere[i].z_u;
    }
    if (p) {
      p[3 * i] = sphere[i].px;
      p[3 * i + 1] = sphere[i].py;
      p[3 * i + 2] = sphere[i].pz;
    }
    if (F) {
      F[3 * i] = sphere[i].Fx;
      F[3 * i + 1] = sphere[i].Fy;
      F[3 * i + 2] = sphere[i].Fz;
    }
  }
}

/* out: peblk, ke, virialblk, vir_actblk, inst_T, maxmaxD */
void ref_get_scalars(double *out) {
  mirror_read();
  out[0] = peblk;
  out[1] = ke;
  out[2] = virialblk;
  out[3] = vir_actblk;
  out[4] = inst_T;
  out[5] = maxmaxD;
}

/* dims[3] = Ncellx, Ncelly, Ncellz; counts[NCell]; members: the InCell
 * lists concatenated in cell order.  Returns NCell. */
int ref_get_cells(int *dims, int *counts, int *members) {
  dims[0] = Ncellx;
  dims[1] = Ncelly;
  dims[2] = Ncellz;
  int m = 0;
  for (int c = 0; c < NCell; c++) {
    if (counts) counts[c] = InCellCount[c];
    if (members)
      for (int j = 0; j < InCellCount[c]; j++) members[m++] = InCell[c][j];
  }
  return NCell;
}

/* half Verlet list: counts[N], and pairs (i, j) flattened into pairs[2*total].
 * Returns the total number of pairs. */
long ref_get_neighbors(int *counts, int *pairs) {
  long m = 0;
  for (int i = 0; i < N; i++) {
    if (counts) counts[i] = NeibListCount[i];
    for (int k = 0; k < NeibListCount[i]; k++) {
      if (pairs) {
        pairs[2 * m] = i;
        pairs[2 * m + 1] = NeibList[i][k];
      }
      m++;
    }
  }
  return m;
}

/* prepareSavingArray (MDcode/main.c:62-119): writes the schedule into out
 * (capacity cap) and returns its length.  The routine also writes
 * <dir>/time_index_file.dat, so dir must exist. */
int ref_log_schedule(unsigned long long runLength, int numOfOrigins, double factor,
                     const char *dir, unsigned long long *out, int cap) {
  long size = numOfOrigins * (10 + (int)(log((double)(runLength / DIVIDE_TO)) / log(factor)));
  free(nextStepIndex);
  /* zero-filled like the fresh heap pages the reference's malloc gets at
   * start-up: prepareSavingArray's 1-based shell sort reads one element past
   * the schedule (MDcode/main.c:17-41, 96) */
  nextStepIndex = (unsigned long long int *)calloc((size_t)size + 1, sizeof(unsigned long long int));
  snprintf(sub_dir, sizeof(sub_dir), "%s", dir);
  prepareSavingArray(runLength, numOfOrigins, factor);
  char path[300];
  snprintf(path, sizeof(path), "%s/time_index_file.dat", dir);
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  int n = 0;
  if (fscanf(f, "total timesteps equals %d", &n) != 1) {
    fclose(f);
    return -1;
  }
  for (int i = 0; i < n && i < cap; i++) out[i] = nextStepIndex[i];
  fclose(f);
  return n;
}

/* write_restart_state (MDcode/main.c:272-288) into path. */
void ref_write_restart(const char *path, int iter, int last_saved_index) {
  char buf[300];
  snprintf(buf, sizeof(buf), "%s", path);
  write_restart_state(buf, iter, last_saved_index);
}
