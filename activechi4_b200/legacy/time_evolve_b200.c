/*
 * time_evolve.c on the GPU: AdvanceTimeNVTNoseHoover, advance_time_NVEFrog,
 * InitialiseNoseHoover, applypbc1/applypbc, the propagators U1..U4 on the
 * host mirror, and the host<->device mirror of the reference's globals used
 * by the drop-in files (acg_legacy.h).
 *
 * Compiled inside a program built from the reference's MDcode sources: it
 * includes that program's global.h (sphere[], N, Nact, L, T, f0, eta, ...).
 *
 * Mirror: the device holds the state.  AdvanceTimeNVTNoseHoover, the hot
 * step, reads back only the step's scalars; sphere[] is refreshed from the
 * device at the sync points, the routines of the reference that read or
 * write sphere[] (sync_points_b200.c), and host edits are detected at the
 * next device call.  With ACG_LEGACY_EAGER defined (a program linked
 * without the sync-point wrappers), every step mirrors the whole state.
 */
#include <math.h>
#include <string.h>

#include "acg_legacy.h"

/* set before the reference's global.h is included: it defines `skin` as a
 * macro, which would rewrite the acg_params field of that name */
static void params_set_skin(acg_params *p, double s) { p->skin = s; }

#include "global.h"
#include "subroutine.h"

static acg_engine *eng[4];  /* [0] Nose-Hoover NVT, [1] NVE, [2] Berendsen NVT, [3] Gaussian isokinetic */
static acg_engine *owner;   /* the engine whose device state is current */
static int host_stale;      /* the device has stepped since sphere[] was last refreshed */
static int host_touched = 1;/* host code may have edited sphere[] since the last push */
static int dirs_touched = 1;/* host code may have changed kx, ky, kz */
/* what the device holds, to detect edits of the globals by host code */
static double *sh_x, *sh_xu, *sh_p;
static int *sh_type, *sh_act, *sh_k;
static double sh_eta[3], sh_peta[3];
static double *b_x, *b_xu, *b_p, *b_F;
static int *b_type, *b_act, *b_k;

void acg_legacy_die(const char *where, int rc) {
  fprintf(stderr, "activechi4: %s failed (%d): %s\n", where, rc, acg_last_error());
  exit(1);
}

static void *xalloc(size_t n) {
  void *p = calloc(n, 1);
  if (!p) {
    fprintf(stderr, "activechi4: host allocation failed\n");
    exit(1);
  }
  return p;
}

acg_engine *acg_legacy_engine(int kind) {
  if (Nprocs > 1) {
    fprintf(stderr, "activechi4: run one MPI rank per system (the whole system lives on one GPU)\n");
    exit(1);
  }
  if (!b_x) {
    sh_x = xalloc(sizeof(double) * 3 * N);
    sh_xu = xalloc(sizeof(double) * 3 * N);
    sh_p = xalloc(sizeof(double) * 3 * N);
    b_x = xalloc(sizeof(double) * 3 * N);
    b_xu = xalloc(sizeof(double) * 3 * N);
    b_p = xalloc(sizeof(double) * 3 * N);
    b_F = xalloc(sizeof(double) * 3 * N);
    sh_type = xalloc(sizeof(int) * N);
    sh_act = xalloc(sizeof(int) * N);
    b_type = xalloc(sizeof(int) * N);
    b_act = xalloc(sizeof(int) * N);
    sh_k = xalloc(sizeof(int) * 3 * (Nact + 1));
    b_k = xalloc(sizeof(int) * 3 * (Nact + 1));
  }
  if (!eng[kind]) {
    static const int thermostat_of[4] = {1, 0, 2, 3};
    acg_params p;
    acg_params_default(&p, N);
    p.nact = Nact;
    p.L = L;
    p.density = DENSITY;
    p.T = T > 0 ? T : 1.0;
    p.f0 = f0;
    p.tau_p_steps = TAU_per;
    p.dt = time_step;
    params_set_skin(&p, skin);
    p.rebuild_factor = 3.0; /* MDcode/time_evolve.c:508 */
    p.list_mode = 0;
    p.thermostat = thermostat_of[kind];
    p.shuffle = 0; /* ShuffleActDirec stays the program's own (host RNG) */
    p.drift_every = 0; /* fixDrift stays the program's own call (MDcode/main.c:261) */
    const char *prec = getenv("ACG_PRECISION");
    if (prec && strcmp(prec, "fp32") == 0) p.precision = ACG_PREC_FP32;
    const char *dev = getenv("ACG_DEVICE");
    int rc = acg_create(&p, 1, dev ? atoi(dev) : 0, &eng[kind]);
    if (rc) acg_legacy_die("acg_create", rc);
  }
  return eng[kind];
}

acg_engine *acg_legacy_current(void) { return owner ? owner : acg_legacy_engine(0); }

static void gather_host(void) {
  for (int i = 0; i < N; i++) {
    double x = sphere[i].x, y = sphere[i].y, z = sphere[i].z;
    /* x + 1 can round to exactly 1 in applypbc1 (MDcode/time_evolve.c:19); keep [0,1) */
    b_x[3 * i] = x >= 1.0 ? x - 1.0 : x;
    b_x[3 * i + 1] = y >= 1.0 ? y - 1.0 : y;
    b_x[3 * i + 2] = z >= 1.0 ? z - 1.0 : z;
    b_xu[3 * i] = sphere[i].x_u;
    b_xu[3 * i + 1] = sphere[i].y_u;
    b_xu[3 * i + 2] = sphere[i].z_u;
    b_p[3 * i] = sphere[i].px;
    b_p[3 * i + 1] = sphere[i].py;
    b_p[3 * i + 2] = sphere[i].pz;
    b_type[i] = sphere[i].type;
    b_act[i] = sphere[i].actTag;
  }
  for (int a = 0; a < Nact; a++) {
    b_k[a] = kx[a];
    b_k[Nact + a] = ky[a];
    b_k[2 * Nact + a] = kz[a];
  }
}

void acg_legacy_host_touched(void) {
  host_touched = 1;
  dirs_touched = 1;
}

void acg_legacy_dirs_touched(void) { dirs_touched = 1; }

void acg_legacy_sync_host(void) {
  if (host_stale && owner) acg_legacy_pull(owner);
}

static void gather_dirs(void) {
  for (int a = 0; a < Nact; a++) {
    b_k[a] = kx[a];
    b_k[Nact + a] = ky[a];
    b_k[2 * Nact + a] = kz[a];
  }
}

void acg_legacy_push(acg_engine *e) {
  int rc;
  if (e == owner && !host_touched) {
    /* nothing on the host has been refreshed or edited since the last push:
     * only the directions (when a shuffle ran) and the chain can differ */
    if (Nact > 0 && dirs_touched) {
      gather_dirs();
      if (memcmp(b_k, sh_k, sizeof(int) * 3 * Nact)) {
        rc = acg_set_directions(e, 0, b_k);
        if (rc) acg_legacy_die("acg_set_directions", rc);
        memcpy(sh_k, b_k, sizeof(int) * 3 * Nact);
      }
    }
    dirs_touched = 0;
    if (memcmp(eta, sh_eta, sizeof(sh_eta)) || memcmp(p_eta, sh_peta, sizeof(sh_peta))) {
      rc = acg_set_nhc(e, 0, eta, p_eta);
      if (rc) acg_legacy_die("acg_set_nhc", rc);
      memcpy(sh_eta, eta, sizeof(sh_eta));
      memcpy(sh_peta, p_eta, sizeof(sh_peta));
    }
    return;
  }
  /* a different engine, or host code that may have edited sphere[]: the device
   * holds nothing newer than the host here */
  acg_legacy_sync_host();
  gather_host();
  const size_t d3 = sizeof(double) * 3 * N;
  const int changed = e != owner || memcmp(b_x, sh_x, d3) || memcmp(b_xu, sh_xu, d3) || memcmp(b_p, sh_p, d3) ||
                      memcmp(b_type, sh_type, sizeof(int) * N) || memcmp(b_act, sh_act, sizeof(int) * N);
  if (changed) {
    rc = acg_set_state(e, 0, b_x, b_xu, b_p, b_type, b_act);
    if (rc) acg_legacy_die("acg_set_state", rc);
    /* forces of the reloaded state with the directions of the last force
     * evaluation: the reference kicks with those forces even after a shuffle
     * earlier in this step */
    if (Nact > 0) {
      rc = acg_set_directions(e, 0, owner ? sh_k : b_k);
      if (rc) acg_legacy_die("acg_set_directions", rc);
      if (!owner) memcpy(sh_k, b_k, sizeof(int) * 3 * Nact);
    }
    rc = acg_set_nhc(e, 0, eta, p_eta);
    if (rc) acg_legacy_die("acg_set_nhc", rc);
    acg_thermo th;
    rc = acg_get_thermo(e, 0, &th);
    if (rc) acg_legacy_die("acg_get_thermo", rc);
    memcpy(sh_x, b_x, d3);
    memcpy(sh_xu, b_xu, d3);
    memcpy(sh_p, b_p, d3);
    memcpy(sh_type, b_type, sizeof(int) * N);
    memcpy(sh_act, b_act, sizeof(int) * N);
    memcpy(sh_eta, eta, sizeof(sh_eta));
    memcpy(sh_peta, p_eta, sizeof(sh_peta));
    owner = e;
  }
  if (Nact > 0 && memcmp(b_k, sh_k, sizeof(int) * 3 * Nact)) {
    rc = acg_set_directions(e, 0, b_k);
    if (rc) acg_legacy_die("acg_set_directions", rc);
    memcpy(sh_k, b_k, sizeof(int) * 3 * Nact);
  }
  if (memcmp(eta, sh_eta, sizeof(sh_eta)) || memcmp(p_eta, sh_peta, sizeof(sh_peta))) {
    rc = acg_set_nhc(e, 0, eta, p_eta);
    if (rc) acg_legacy_die("acg_set_nhc", rc);
    memcpy(sh_eta, eta, sizeof(sh_eta));
    memcpy(sh_peta, p_eta, sizeof(sh_peta));
  }
  host_touched = 0;
  dirs_touched = 0;
}

/* the scalar globals a step sets (MDcode/time_evolve.c:495-526) */
static void pull_scalars(acg_engine *e) {
  acg_thermo th;
  int rc = acg_get_thermo(e, 0, &th);
  if (rc) acg_legacy_die("acg_get_thermo", rc);
  peblk = th.pe;
  virialblk = th.virial;
  vir_actblk = th.vir_act;
  maxD = th.maxD;
  maxmaxD = th.maxD;
  ke = th.ke;
  /* the Gaussian isokinetic step leaves inst_T = 2 sum p^2 / DOF
   * (MDcode/time_evolve.c:464-465) */
  inst_T = e == eng[3] ? 4.0 * th.ke / DOF : th.inst_T;
  if (e == eng[0]) {
    for (int k = 0; k < M; k++) {
      eta[k] = th.eta[k];
      p_eta[k] = th.p_eta[k];
      q[k] = th.q[k];
    }
    memcpy(sh_eta, eta, sizeof(sh_eta));
    memcpy(sh_peta, p_eta, sizeof(sh_peta));
  }
}

void acg_legacy_pull(acg_engine *e) {
  int rc = acg_get_state(e, 0, b_x, b_xu, b_p, b_F);
  if (rc) acg_legacy_die("acg_get_state", rc);
  for (int i = 0; i < N; i++) {
    sphere[i].x = b_x[3 * i];
    sphere[i].y = b_x[3 * i + 1];
    sphere[i].z = b_x[3 * i + 2];
    sphere[i].x_u = b_xu[3 * i];
    sphere[i].y_u = b_xu[3 * i + 1];
    sphere[i].z_u = b_xu[3 * i + 2];
    sphere[i].px = b_p[3 * i];
    sphere[i].py = b_p[3 * i + 1];
    sphere[i].pz = b_p[3 * i + 2];
    sphere[i].Fx = b_F[3 * i];
    sphere[i].Fy = b_F[3 * i + 1];
    sphere[i].Fz = b_F[3 * i + 2];
  }
  const size_t d3 = sizeof(double) * 3 * N;
  memcpy(sh_x, b_x, d3);
  memcpy(sh_xu, b_xu, d3);
  memcpy(sh_p, b_p, d3);
  pull_scalars(e);
  host_stale = 0;
  host_touched = 1; /* the caller may edit what it now sees */
}

/* applypbc1 / applypbc (MDcode/time_evolve.c:15-37): host wrap of sphere[],
 * used by the reference's Parallel.c, initialise.c and main.c */
void applypbc1() {
  for (int i = 0; i < NumInBlock[node]; i++) {
    int part = InBlock[node][i];
    while (sphere[part].x >= LENGTH) sphere[part].x -= LENGTH;
    while (sphere[part].x < 0.0) sphere[part].x += LENGTH;
    while (sphere[part].y >= LENGTH) sphere[part].y -= LENGTH;
    while (sphere[part].y < 0.0) sphere[part].y += LENGTH;
    while (sphere[part].z >= LENGTH) sphere[part].z -= LENGTH;
    while (sphere[part].z < 0.0) sphere[part].z += LENGTH;
  }
}
void applypbc() {
  for (int part = 0; part < N; part++) {
    while (sphere[part].x >= LENGTH) sphere[part].x -= LENGTH;
    while (sphere[part].x < 0.0) sphere[part].x += LENGTH;
    while (sphere[part].y >= LENGTH) sphere[part].y -= LENGTH;
    while (sphere[part].y < 0.0) sphere[part].y += LENGTH;
    while (sphere[part].z >= LENGTH) sphere[part].z -= LENGTH;
    while (sphere[part].z < 0.0) sphere[part].z += LENGTH;
  }
}

/* InitialiseNoseHoover (MDcode/time_evolve.c:476-493): chain masses from T,
 * eta = 0, p_eta drawn with the program's own random_normal; the device gets
 * the chain at the next step */
void InitialiseNoseHoover() {
  tau = .20;
  for (int i = 0; i < M; i++) {
    q[i] = T * tau * tau;
    eta[i] = 0.0e0;
  }
  q[0] = DOF * T * tau * tau;
  if (node == 0) {
    int for_ran1 = -(int)(time(0) + node);
    srand(node + 100 - for_ran1);
    for (int i = 0; i < M; i++) {
      double abc = random_normal();
      p_eta[i] = sqrt(T * q[i]) * abc;
    }
  }
  MPI_Bcast(&p_eta, M, MPI_DOUBLE, 0, MPI_COMM_WORLD);
  if (eng[0]) {
    int rc = acg_set_temperature(eng[0], 0, T);
    if (rc) acg_legacy_die("acg_set_temperature", rc);
  }
}

/* one step of the whole system on the device with engine `kind`; sphere[]
 * and the step's scalars (pe, ke, virial, maxmaxD, the chain) follow at the
 * next sync point, so a run of steps queues on the device without a wait */
static void legacy_step(int kind) {
  acg_engine *e = acg_legacy_engine(kind);
  acg_legacy_push(e);
  int rc = acg_step(e, 1);
  if (rc) acg_legacy_die("acg_step", rc);
  owner = e;
#ifdef ACG_LEGACY_EAGER
  acg_legacy_pull(e);
#else
  host_stale = 1;
#endif
}

/* list rebuilds of the engine that holds the state (for test harnesses, which
 * would otherwise read maxmaxD after every step) */
long long acg_legacy_rebuilds(void) {
  acg_thermo th;
  int rc = acg_get_thermo(acg_legacy_current(), 0, &th);
  if (rc) acg_legacy_die("acg_get_thermo", rc);
  return (long long)th.rebuilds;
}

/* AdvanceTimeNVTNoseHoover (MDcode/time_evolve.c:495-526): one NHC step of
 * the whole system on the device */
void AdvanceTimeNVTNoseHoover() {
  legacy_step(0);
  Heff = 0;
}

/* advance_time_NVT_Berendsen (MDcode/time_evolve.c:173-256): one NVE step,
 * then the momenta scaled by sqrt(1 + (T/inst_T - 1) dt/tau_T), on the device */
void advance_time_NVT_Berendsen() { legacy_step(2); }

/* AdvanceTimeNVTGaussOSM (MDcode/time_evolve.c:351-470): one Gaussian
 * isokinetic step on the device */
void AdvanceTimeNVTGaussOSM() { legacy_step(3); }

/* advance_time_NVEFrog (MDcode/time_evolve.c:104-171): one velocity-Verlet
 * step without thermostat (used by the set-up ramps of initialise.c) */
void advance_time_NVEFrog() {
  acg_engine *e = acg_legacy_engine(1);
  acg_legacy_push(e);
  int rc = acg_step(e, 1);
  if (rc) acg_legacy_die("acg_step", rc);
  /* the ramps of initialise.c read sphere[] between these steps from inside
   * their own file (no sync point): always mirror the whole state */
  acg_legacy_pull(e);
  keblk = 2.0 * ke;
}

/* ---- the propagators of the NVT step (MDcode/time_evolve.c:527-609) ------
 * AdvanceTimeNVTNoseHoover runs them fused on the device; these separate
 * entry points keep the reference's names and act on the host mirror, for
 * host code that composes its own step from them. */
void U1Propagator() {
  acg_legacy_sync_host();
  for (int i = 0; i < N; i++) {
    const double dx = sphere[i].px * time_step, dy = sphere[i].py * time_step, dz = sphere[i].pz * time_step;
    sphere[i].x += dx * inv_L;
    sphere[i].x_u += dx * inv_L;
    sphere[i].y += dy * inv_L;
    sphere[i].y_u += dy * inv_L;
    sphere[i].z += dz * inv_L;
    sphere[i].z_u += dz * inv_L;
  }
  applypbc1();
  double m = 0.0;
  for (int i = 0; i < N; i++) {
    const double dx = sphere[i].x_u - xold[i], dy = sphere[i].y_u - yold[i], dz = sphere[i].z_u - zold[i];
    const double t = dx * dx + dy * dy + dz * dz;
    if (m < t) m = t;
  }
  maxD = m * L * L;
  maxmaxD = maxD;
  acg_legacy_host_touched();
}

void U2Propagator() {
  acg_legacy_sync_host();
  for (int i = 0; i < N; i++) {
    sphere[i].px += sphere[i].Fx * half_time_step;
    sphere[i].py += sphere[i].Fy * half_time_step;
    sphere[i].pz += sphere[i].Fz * half_time_step;
  }
  acg_legacy_host_touched();
}

void U3Propagator(double t) {
  acg_legacy_sync_host();
  for (int i = 0; i < N; i++) {
    sphere[i].px = sphere[i].px * exp(-t * p_eta[0] / q[0]);
    sphere[i].py = sphere[i].py * exp(-t * p_eta[0] / q[0]);
    sphere[i].pz = sphere[i].pz * exp(-t * p_eta[0] / q[0]);
  }
  for (int i = 0; i < M; i++) eta[i] = eta[i] + t * p_eta[i] / q[i];
  acg_legacy_host_touched();
}

void U4Propagator(double t, int jStart, int jEnd) {
  acg_legacy_sync_host();
  const int dj = jStart > jEnd ? -1 : 1;
  int j = jStart;
  do {
    double gj;
    if (j == 0) {
      double kb = 0.0;
      for (int i = 0; i < N; i++)
        kb += sphere[i].px * sphere[i].px + sphere[i].py * sphere[i].py + sphere[i].pz * sphere[i].pz;
      ke = kb;
      gj = kb - DOF * T;
    } else {
      gj = (p_eta[j - 1] * p_eta[j - 1]) / q[j - 1] - T;
    }
    if (j == M - 1) {
      p_eta[j] = p_eta[j] + t * gj;
    } else {
      const double x = t * p_eta[j + 1] / q[j + 1];
      p_eta[j] = p_eta[j] * exp(-x) + t * gj * (1.0 - exp(-x)) / x;
    }
    j += dj;
  } while (j - dj != jEnd);
}
