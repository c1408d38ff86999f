/*
 * time_evolve.c on the GPU: AdvanceTimeNVTNoseHoover, advance_time_NVEFrog,
 * InitialiseNoseHoover, applypbc1/applypbc, and the host<->device mirror of
 * the reference's globals used by the drop-in files (acg_legacy.h).
 *
 * Compiled inside a program built from the reference's MDcode sources: it
 * includes that program's global.h (sphere[], N, Nact, L, T, f0, eta, ...).
 */
#include <string.h>

#include "acg_legacy.h"

/* set before the reference's global.h is included: it defines `skin` as a
 * macro, which would rewrite the acg_params field of that name */
static void params_set_skin(acg_params *p, double s) { p->skin = s; }

#include "global.h"
#include "subroutine.h"

static acg_engine *eng[2];  /* [0] Nose-Hoover NVT, [1] NVE */
static acg_engine *owner;   /* the engine whose device state is current */
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

acg_engine *acg_legacy_engine(int nve) {
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
  if (!eng[nve]) {
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
    p.thermostat = nve ? 0 : 1;
    p.shuffle = 0; /* ShuffleActDirec stays the program's own (host RNG) */
    p.drift_every = 0; /* fixDrift stays the program's own call (MDcode/main.c:261) */
    const char *prec = getenv("ACG_PRECISION");
    if (prec && strcmp(prec, "fp32") == 0) p.precision = ACG_PREC_FP32;
    const char *dev = getenv("ACG_DEVICE");
    int rc = acg_create(&p, 1, dev ? atoi(dev) : 0, &eng[nve]);
    if (rc) acg_legacy_die("acg_create", rc);
  }
  return eng[nve];
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

void acg_legacy_push(acg_engine *e) {
  int rc;
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
  acg_thermo th;
  rc = acg_get_thermo(e, 0, &th);
  if (rc) acg_legacy_die("acg_get_thermo", rc);
  peblk = th.pe;
  virialblk = th.virial;
  vir_actblk = th.vir_act;
  maxD = th.maxD;
  maxmaxD = th.maxD;
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

/* AdvanceTimeNVTNoseHoover (MDcode/time_evolve.c:495-526): one NHC step of
 * the whole system on the device */
void AdvanceTimeNVTNoseHoover() {
  acg_engine *e = acg_legacy_engine(0);
  acg_legacy_push(e);
  int rc = acg_step(e, 1);
  if (rc) acg_legacy_die("acg_step", rc);
  acg_legacy_pull(e);
  Heff = 0;
  acg_thermo th;
  rc = acg_get_thermo(e, 0, &th);
  if (rc) acg_legacy_die("acg_get_thermo", rc);
  ke = th.ke;
  inst_T = th.inst_T;
}

/* advance_time_NVEFrog (MDcode/time_evolve.c:104-171): one velocity-Verlet
 * step without thermostat (used by the set-up ramps of initialise.c) */
void advance_time_NVEFrog() {
  acg_engine *e = acg_legacy_engine(1);
  acg_legacy_push(e);
  int rc = acg_step(e, 1);
  if (rc) acg_legacy_die("acg_step", rc);
  acg_legacy_pull(e);
  acg_thermo th;
  rc = acg_get_thermo(e, 0, &th);
  if (rc) acg_legacy_die("acg_get_thermo", rc);
  keblk = 2.0 * th.ke;
}
