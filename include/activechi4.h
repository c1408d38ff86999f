/*
 * activechi4.h — C ABI of the B200 (sm_100a) MD timestep for the active
 * Kob-Andersen glass.
 *
 * The reference engine (AnoopMut/activeChi4, MDcode/) keeps all state in
 * process globals and exposes argument-less C routines (MDcode/subroutine.h).
 * This library keeps the state resident on one GPU behind an opaque handle
 * that may hold many independent systems ("a batch"); one system is simply a
 * batch of one.  The reference routines are re-implemented on top of this ABI
 * in activechi4_b200/legacy/*.c, which a C host program links in place of
 * MDcode/cell_list+forces.c, MDcode/active.c and the NVT part of
 * MDcode/time_evolve.c.
 *
 * Units and layouts follow the reference: positions are reduced coordinates
 * (box = unit cube; x in [0,1) wrapped, xu unfolded), momenta and forces are
 * absolute (unit mass).  Per-particle arrays are interleaved [n][3] doubles in
 * the caller's particle order; the library reorders internally and always
 * returns the caller's order.
 *
 * Every entry point returns ACG_OK (0) or a negative ACG_ERR_* code; the
 * message of the last failure on the calling thread is acg_last_error().
 * Calls on one handle must come from one host thread at a time.
 */
#ifndef ACTIVECHI4_H
#define ACTIVECHI4_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ACG_OK 0
#define ACG_ERR_INVALID (-1)    /* bad argument or parameter */
#define ACG_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define ACG_ERR_NOMEM (-3)      /* device allocation failed / footprint too large */
#define ACG_ERR_NONFINITE (-4)  /* a system's kinetic energy became NaN/inf */
#define ACG_ERR_STATE (-5)      /* call not valid in the handle's current state */
#define ACG_ERR_BOX (-6)        /* a constant-pressure system's box left the cell grid it was
                                   created with ((int)((int)L / Cell_cut) changed) */

#define ACG_PREC_FP64 0 /* pair forces in FP64 (the reference's arithmetic) */
#define ACG_PREC_FP32 1 /* pair forces in FP32; positions, velocities, thermostat,
                           energies and virials stay FP64 */

/* Parameters of one system.  Defaults (acg_params_default) are the
 * reference's constants: MDcode/global.h:24-58, para_file (MDcode/main.c:410-426). */
typedef struct acg_params {
  int n;                  /* particles (N, MDcode/global.h:15) */
  int nact;               /* active particles; -1 = (int)(0.1*n) (Nact, MDcode/global.h:55) */
  double L;               /* box length; <= 0 means pow(n/density, 0.33333333) (MDcode/main.c:465) */
  double density;         /* DENSITY (para_file line 4) */
  double T;               /* thermostat temperature (para_file line 4) */
  double f0;              /* active force magnitude (para_file line 6) */
  int tau_p_steps;        /* direction persistence in steps (TAU_per, MDcode/global.h:58) */
  double dt;              /* time_step (MDcode/global.h:32) */
  double skin;            /* Verlet skin (MDcode/global.h:28) */
  double rebuild_factor;  /* rebuild when factor*maxD^2 > skin^2 (MDcode/time_evolve.c:508 uses 3) */
  int list_mode;          /* 0: list cut 2.5+skin for all pairs (Cell_cut, global.h:29);
                             1: list cut 2.5*sigma_ab+skin per type pair */
  int thermostat;         /* 1: Nose-Hoover chain NVT (AdvanceTimeNVTNoseHoover);
                             0: NVE velocity Verlet (advance_time_NVEFrog);
                             2: Berendsen NVT, the momenta scaled by
                                sqrt(1 + (T/inst_T - 1) dt/tau_T) after each step
                                (advance_time_NVT_Berendsen, MDcode/time_evolve.c:173-256);
                             3: Gaussian isokinetic, each half kick p = f1 (p + f2 F)
                                with f1, f2 from sum p.F, sum F^2, sum p^2
                                (AdvanceTimeNVTGaussOSM, MDcode/time_evolve.c:351-470);
                                T is not used and acg_start_ramp is refused;
                             4: Berendsen NPT: before each step the box is scaled by
                                chi_P = (1 + dt (pressure - P)/tau_P)^(1/3), pressure =
                                DENSITY inst_T + virial/L^3, and the forces recomputed;
                                then the Berendsen NVT step (advance_time_NPT,
                                MDcode/time_evolve.c:258-348, with UpdateBoxForNPT :823-850).
                                The box keeps the cell count it was created with
                                (ACG_ERR_BOX when the reference's count would change);
                             5: Nose-Hoover NPT: particle and barostat chains, p_eps and
                                L = L0 exp(eps) (AdvanceTimeNPTNoseHoover with
                                U1..U4PropagatorNPT, MDcode/time_evolve.c:654-822); the
                                barostat state comes from acg_set_barostat; same cell-grid
                                rule as 4;
                             6: active Brownian dynamics, predictor-corrector with random
                                forces sqrt(2 T^2/dt) N(0,1) minus their mean
                                (advance_time_ActiveBrown_PC, MDcode/time_evolve.c:855-974,
                                D0 = 1); the normals come from a counter-based stream
                                (Philox4x32-10 keyed by `seed`, counter = particle and step)
                                in place of the reference's GSL draws.
                             Ramps (acg_start_ramp) are refused for 3, 5 and 6 */
  int shuffle;            /* re-randomise the active directions every tau_p_steps steps
                             (ShuffleActDirec cadence, MDcode/main.c:245-247):
                             1: on the device in the reference's order (per component,
                                swap k[i] with k[(int)(Nact*u)], MDcode/active.c:58-75)
                                on an MT19937 stream seeded like gsl_rng_set(seed), so
                                the directions equal the reference's for the same seed;
                             2: a uniformly random permutation per component (parallel,
                                not the reference's distribution);
                             0: the caller sets them (acg_set_directions) */
  int precision;          /* ACG_PREC_FP64 or ACG_PREC_FP32 */
  int nb_capacity;        /* neighbour-list row capacity; 0 = automatic.  Particles
                             with more neighbours are served from the cell list
                             (the reference's MaxNeibs, MDcode/global.h:19, is
                             unchecked) */
  uint64_t seed;          /* direction-shuffle stream (gsl_rng_set seed; 0 is taken as 4357) */
  int drift_every;        /* remove the mean momentum (fixDrift, MDcode/initialise.c:104-138)
                             after every step whose index is a multiple of this, as run()
                             does every 100000 steps (MDcode/main.c:261); 0 = never */
  double P;               /* target pressure of the Berendsen barostat (thermostat 4;
                             para_file line 4, MDcode/main.c:422) */
} acg_params;

/* Scalars of one system at the last step boundary. */
typedef struct acg_thermo {
  double pe;       /* potential energy (peblk, MDcode/cell_list+forces.c:194) */
  double ke;       /* kinetic energy 0.5*sum p^2 (ke, MDcode/time_evolve.c:520) */
  double virial;   /* pair virial / 3 (virialblk, MDcode/cell_list+forces.c:220) */
  double vir_act;  /* active virial (vir_actblk, MDcode/cell_list+forces.c:214) */
  double inst_T;   /* 2 ke / DOF (MDcode/time_evolve.c:524) */
  double maxD;     /* max squared displacement since the last rebuild (maxmaxD) */
  double heff;     /* conserved NHC energy (Heff, MDcode/print.c:85-87) */
  double eta[3], p_eta[3], q[3]; /* thermostat chain (MDcode/time_evolve.c:476-493) */
  int64_t step;    /* steps taken (the run() loop index) */
  int64_t rebuilds;/* cell/neighbour list rebuilds so far */
  int overflow;    /* particles that overflowed the neighbour-list capacity at the
                      last rebuild (served from the cell list instead) */
  int status;      /* 0, ACG_ERR_NONFINITE or ACG_ERR_BOX */
  double L;        /* current box length (changes under thermostats 4 and 5) */
  double pressure; /* DENSITY inst_T + virial/L^3 at the last box update (thermostat 4) */
  double eps, p_eps;                 /* barostat (thermostat 5): L = L0 exp(eps) */
  double eta_baro[3], p_eta_baro[3]; /* barostat chain (thermostat 5) */
} acg_thermo;

typedef struct acg_engine acg_engine;

/* Fill *p with the reference defaults for n particles. */
int acg_params_default(acg_params *p, int n);

/* Create an engine holding nsys systems (params[0..nsys-1]) on CUDA device
 * `device`.  Allocates all device memory up front; no allocation happens on
 * the stepping path.  Replaces the set-up half of main()
 * (AllocateArrays, SetUpParallel, SetUpCellList: MDcode/Parallel.c:6-106,
 * 778-809) — there is no domain decomposition, each system lives whole on
 * the device. */
int acg_create(const acg_params *params, int nsys, int device, acg_engine **out);
int acg_destroy(acg_engine *e);
/* Destroy the CUDA graphs of engines destroyed so far.  acg_destroy frees an
 * engine's memory in stream order but only retires its graphs: destroying a
 * graph that holds conditional nodes waits for the whole device, which would
 * stall other engines' work.  Call this when the device may idle (the run
 * server does when no run is active); it also happens by itself once 256
 * graphs are retired.  No counterpart in the reference. */
int acg_release_retired(void);

/* Bytes of device memory acg_create would allocate for these systems
 * (admission control for serving). */
int acg_footprint(const acg_params *params, int nsys, size_t *bytes);

/* Load one system's particles (caller order).  x: [n][3] wrapped reduced
 * coordinates; xu: unfolded (NULL = x); p: momenta; type[n]: 0 = A, 1 = B;
 * act_tag[n]: -1 or the particle's index into the direction arrays.
 * Replaces BcastInitState / read_restart_state + initialise_restart_state
 * (MDcode/Parallel.c:618-656, MDcode/main.c:290-334).  Forces, cells and
 * neighbour lists are rebuilt before the next step. */
int acg_set_state(acg_engine *e, int sys, const double *x, const double *xu, const double *p,
                  const int *type, const int *act_tag);

/* Read one system back in the caller's order; any pointer may be NULL.
 * F are the forces of the last evaluation. */
int acg_get_state(acg_engine *e, int sys, double *x, double *xu, double *p, double *F);

/* Active directions k[3][nact] = kx, ky, kz in {-1,+1}
 * (kx/ky/kz, MDcode/active.c:30-41; readActiveDirection :101-122). */
int acg_set_directions(acg_engine *e, int sys, const int *k);
int acg_get_directions(acg_engine *e, int sys, int *k);

/* Re-randomise one system's directions now on the device: ShuffleActDirec,
 * MDcode/active.c:45-85, in the reference's order on the system's MT19937
 * stream (shuffle modes 0 and 1), or a uniformly random permutation per
 * component (mode 2). */
int acg_shuffle_directions(acg_engine *e, int sys);
/* Reseed one system's MT19937 direction stream: gsl_rng_set(rng_ptr, seed)
 * of initializeGsl (MDcode/initialise.c:5-11). */
int acg_seed_shuffle(acg_engine *e, int sys, uint64_t seed);

/* fixDrift (MDcode/initialise.c:104-138) now: subtract the mean momentum of
 * one system (acg_step also does it by itself every drift_every steps). */
int acg_fix_drift(acg_engine *e, int sys);

/* adjustInitialTemp (MDcode/initialise.c:141-151): scale one system's momenta
 * by sqrt(T / inst_T); *inst_T (may be NULL) receives the temperature after
 * the scaling (calculate_temp, :153-164). */
int acg_adjust_temperature(acg_engine *e, int sys, double T, double *inst_T);

/* The heating and cooling ramps of initialisation, coldstart and breakxal
 * (MDcode/initialise.c:166-201): rescale one system's momenta to T_start now,
 * then, for each of the next *steps steps of that system, rescale to the ramp
 * temperature (starting at the temperature reached, changing by
 * dt * rate per step towards T_end until it passes T_end) and take one NVE
 * leap-frog step (advance_time_NVEFrog, MDcode/time_evolve.c:104-171).  The
 * ramp steps run inside the following acg_step calls; during them the
 * system's step counter, direction shuffles, drift removal and observables
 * wait.  coldstart(rate, T) = acg_start_ramp(e, s, 0.5 T, T, rate, ..);
 * breakxal(rate, T) = acg_start_ramp(e, s, 1.5 T, T, rate, ..). */
int acg_start_ramp(acg_engine *e, int sys, double T_start, double T_end, double rate, int64_t *steps);
/* Lengthen one system's armed ramp to total_steps steps: the steps after the
 * ramp itself rescale to T_end, so systems whose ramps differ in length can
 * run them inside one engine and finish together.  No counterpart in the
 * reference (one system per program). */
int acg_extend_ramp(acg_engine *e, int sys, int64_t total_steps);

/* GetFccGrid placement (MDcode/initialise.c:34-101) on the device: particle k
 * at grid site site[k] of the troot^3 grid (troot = smallest integer with
 * troot^3 >= n), positions with the reference's arithmetic, xu = x; type,
 * momenta p [n][3] and act_tag as acg_set_state.  The random choices (sites,
 * types, momenta) are the caller's, e.g. the reference's rand() draws. */
int acg_set_lattice(acg_engine *e, int sys, const int *site, const int *type, const double *p,
                    const int *act_tag);

/* Thermostat chain state (InitialiseNoseHoover, MDcode/time_evolve.c:476-493:
 * eta = 0, p_eta drawn by the caller).  q follows from T and n. */
int acg_set_nhc(acg_engine *e, int sys, const double *eta3, const double *p_eta3);
/* Barostat state of a Nose-Hoover NPT system (thermostat 5) at the step
 * boundary: chain eta_baro[3], p_eta_baro[3] and p_eps (InitialiseNoseHooverNPT,
 * MDcode/time_evolve.c:614-652, draws them; eps starts at 0 with L0 = the
 * creation length).  The next step's first half is recomputed. */
int acg_set_barostat(acg_engine *e, int sys, const double *eta_baro3, const double *p_eta_baro3, double p_eps);

/* Change a system's thermostat temperature (and with it q). */
int acg_set_temperature(acg_engine *e, int sys, double T);

/* update_cell_list (MDcode/cell_list+forces.c:58-148) for every system:
 * counting-sort cell build + neighbour lists. */
int acg_rebuild(acg_engine *e);

/* calculate_forces (MDcode/cell_list+forces.c:153-227) for every system at
 * the current positions (rebuilding cells/lists first when needed). */
int acg_compute_forces(acg_engine *e);

/* Advance every system nsteps steps: for each step the direction shuffle
 * when due (MDcode/main.c:245-247) then AdvanceTimeNVTNoseHoover
 * (MDcode/time_evolve.c:495-526) or advance_time_NVEFrog
 * (MDcode/time_evolve.c:104-171).  Runs as CUDA-graph launches on the
 * engine's stream; returns after queuing (acg_sync waits). */
int acg_step(acg_engine *e, int nsteps);
/* The same steps launched kernel by kernel without a CUDA graph (every
 * rebuild kernel is launched and skips the systems that need no rebuild). */
int acg_step_eager(acg_engine *e, int nsteps);
/* Prime the engine and build the CUDA graphs acg_step launches, without
 * stepping.  Instantiating a graph can wait for the work already queued on
 * the device, so a host that drives several engines may call this from a
 * second thread while it keeps feeding the others.  No counterpart in the
 * reference. */
int acg_prepare(acg_engine *e);
int acg_sync(acg_engine *e);
/* Non-blocking: *done = 1 when all work queued on the engine has finished. */
int acg_poll(acg_engine *e, int *done);

int acg_get_thermo(acg_engine *e, int sys, acg_thermo *out);

/* Cell list of the last rebuild: dims[3] cells per side, counts[ncell],
 * members[n] = particle indices (caller order) per cell, ascending within a
 * cell (InCellCount / InCell, MDcode/cell_list+forces.c:71-80).  counts and
 * members may be NULL; returns the number of cells via *ncell. */
int acg_get_cells(acg_engine *e, int sys, int *dims, int *ncell, int *counts, int *members);

/* ---- in-place observables on the log-time schedule -----------------------
 * The reference writes unfolded coordinates at the steps of prepareSavingArray
 * (MDcode/main.c:62-119, 252-257) and computes the overlap Q(t), chi4(t), the
 * MSD and its moments and Fs(q,t) offline (Analysis/overlap.c, msd_pos.c,
 * Fsqt.c).  Here the same sums are accumulated on the device while stepping:
 * origin snapshots stay in device memory and every (origin, later step) pair of
 * the schedule adds to its time bin.  The schedule starts at the system's
 * current step. */
typedef struct acg_obs_config {
  int64_t run_length;     /* steps of the run (runLength) */
  int num_origins;        /* origins, every run_length/num_origins steps (200) */
  double factor;          /* offset growth factor (1.4) */
  int64_t max_interval;   /* offsets analysed are < max_interval; <= 0: run_length/2 */
  double a;               /* overlap cut (0.3, Analysis/main.c:6) */
  int nq;                 /* wave vectors for Fs (0..256) */
  const int *qvec;        /* [nq][3] integers n, q = 2 pi n / L */
  int max_live_origins;   /* origin snapshots kept (device memory n*24 bytes each) */
} acg_obs_config;
int acg_obs_configure(acg_engine *e, int sys, const acg_obs_config *c);
/* Raw per-bin sums over the pairs accumulated so far: *nbins bins with
 * offset[m] steps and sums[m][7] = {sum Q, sum Q^2, sum msd, sum msd_d4,
 * sum msd_r4, sum Fs, count}; Q(t) = sum Q / count, chi4 = sum Q^2/count -
 * Q(t)^2 (not x N, as Analysis/overlap.c:118), msd = <|dr|^2>, msd_d4 =
 * <dx^4+dy^4+dz^4>, msd_r4 = <|dr|^4> (Analysis/msd_pos.c:88-91). */
int acg_obs_sums(acg_engine *e, int sys, int *nbins, int64_t *offset, double *sums);

/* Number of systems, particles of one system, and the engine's CUDA stream
 * (a cudaStream_t) for callers that time or order work around it. */
int acg_num_systems(acg_engine *e);
int acg_system_size(acg_engine *e, int sys, int *n, int *nact);
void *acg_stream(acg_engine *e);
/* Scheduling priority of the engine's stream among the work of other engines
 * on the same device: 0 = default, higher levels are scheduled first (clamped
 * to the device's range).  No counterpart in the reference (one program per
 * rank); the run server uses it to keep large runs from being crowded out by
 * many small ones. */
int acg_set_priority(acg_engine *e, int level);

/* Kernel timing for profiling: average device time in ms of `reps`
 * back-to-back launches of one stage over all systems, timed with CUDA events
 * on the engine stream.  stage: 0 = kick+drift, 1 = pair forces + kick,
 * 2 = full cell/neighbour rebuild. */
int acg_time_stage(acg_engine *e, int stage, int reps, double *ms);

/* Benchmark timing: advance every system exactly nsteps steps as CUDA-graph
 * launches (one graph of nsteps steps up to 256, else graphs of 32 steps and
 * one of the remainder), recording CUDA events on the engine stream around
 * each launch, and write flush_bytes (> L2) with cudaMemsetAsync before each
 * launch (untimed) so that every timed launch starts from a cold L2.  *ms =
 * summed device time of the launches; *launches = kernels launched inside
 * them (counted from the rebuilds, shuffles, drift removals and observable
 * events they took).  No counterpart in the reference. */
int acg_bench_steps(acg_engine *e, int64_t nsteps, size_t flush_bytes, double *ms, int64_t *launches);

/* Measured FP64 FMA throughput of `device` in TFLOP/s (2 flops per FMA):
 * independent DFMA chains on every SM, timed with CUDA events. */
int acg_measure_fp64_peak(int device, double *tflops);

/* Launch-configuration knobs (the autotuner sets these). tpp: threads per
 * particle in the force kernel (1,2,4,8,16,32); block: threads per block. */
int acg_set_launch(acg_engine *e, int tpp, int block);
int acg_get_launch(acg_engine *e, int *tpp, int *block);
/* Threads per particle (1, 2 or 4) of the cell-group force kernel (boxes with
 * >= 5 cells per side, or larger than the whole-box limit) and of the
 * whole-box force kernel (2 to 4 cells per side, N <= 8192). */
int acg_set_group_tpp(acg_engine *e, int gtpp);
/* Cells per block of the whole-box kernels (systems with 3 or 4 cells per
 * side; two-cell boxes keep one cell per block), 1 to 8: the partition of
 * the force and list grids over the batch.  Results do not depend on it (the
 * per-system sums are taken per particle, in slot order).  No counterpart in
 * the reference. */
int acg_set_box_cells(acg_engine *e, int cells);
int acg_get_box_cells(acg_engine *e, int *cells);

const char *acg_last_error(void);
const char *acg_version(void);

/* ---- allocation-free force evaluation -----------------------------------
 * No counterpart in the reference: this entry point exists for callers that
 * cannot allocate device memory — code running inside a framework that owns
 * all device memory through its own pool, hosts that forbid allocation once a
 * latency-bounded loop has started, and plug-ins that are only handed device
 * pointers by their host.  It computes calculate_forces' result (pair forces,
 * active forces, pe, virial, vir_act) for one system from arrays the caller
 * already has on the device, and allocates nothing: its intermediates live in
 * one file-scope device array of ACG_NOALLOC_SCRATCH_BYTES that every GPU
 * which loads the library holds until the process exits.
 *
 * All pointers are device pointers on the current device: x [n][3] wrapped
 * reduced coordinates, xu [n][3] unfolded (NULL = x, used for vir_act only),
 * type[n], act_tag[n] (-1 or index into k), k [3][nact]; outputs F [n][3]
 * and scalars[3] = {pe, virial, vir_act}.  stream is a cudaStream_t (NULL =
 * the default stream); the call only queues work on it.
 * Limits: 2 <= n <= ACG_NOALLOC_MAX_N and at most ACG_NOALLOC_MAX_CELLS cells
 * of side >= 2.85 (cells per side = (int)((int)L / 2.85) >= 2); larger sizes
 * return ACG_ERR_INVALID with a message.
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  Calls share the array and it keeps the last
 * call's contents (each call clears what must start at zero); calls that
 * overlap on the GPU (two streams, or two host threads) race on it and must
 * be serialised by the caller.
 * The looked-up address is kept per device index for the process: it belongs
 * to the device's primary context (the one the CUDA runtime uses); after
 * cudaDeviceReset, or from a different context made current through the
 * driver API, it is no longer valid, so such callers must not use this entry
 * point.  Particles are placed in their cells by atomic counters, so the
 * order in which each particle's pair terms are summed can change from call
 * to call: results repeat to FP64 rounding (max|dF|/rms|F| ~ 1e-15), not bit
 * for bit. */
#define ACG_NOALLOC_MAX_N 262144
#define ACG_NOALLOC_MAX_CELLS 32768
#define ACG_NOALLOC_SCRATCH_BYTES (3u << 20)
int acg_forces_noalloc(const double *x, const double *xu, const int *type, const int *act_tag,
                       const int *k, int n, int nact, double L, double f0, double *F,
                       double *scalars, void *stream);

#ifdef __cplusplus
}
#endif
#endif
