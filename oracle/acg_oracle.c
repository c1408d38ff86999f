/*
 * acg_oracle — CPU restatement of the reference's MD timestep.
 * TEST INFRASTRUCTURE ONLY (see acg_oracle.h): the CUDA path is checked
 * against it; never part of it.
 *
 * Each routine cites the reference lines it restates.  Loop orders, the
 * order of floating-point operations and the neighbour-list construction
 * follow the reference so that results agree bit for bit with the reference
 * compiled from its own sources whenever the box has >= 3 cells per side.
 */
#include "acg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* MDcode/global.h:24-45 and cell_list+forces.c:19-20 */
#define HALF_LENGTH 0.5
#define LENGTH 1.0
#define LCUT_SQR 6.25
#define SKIN 0.35
#define CELL_CUT (2.5 + SKIN)
#define TIME_STEP 0.005
#define HALF_TIME_STEP (TIME_STEP * 0.5)
#define C0 0.0162665594880
#define C2 (-0.001949973872640)
#define NHC_M 3
#define TAU_T 0.20
static const double SIGMA[2][2] = {{1.00, 0.80}, {0.80, 0.88}};
static const double EPSILON[2][2] = {{1.0, 1.5}, {1.5, 0.50}};

/* ------------------------------------------------------------------------ */
/* MT19937 (Matsumoto & Nishimura 1998) for the direction shuffle           */
typedef struct {
  unsigned int mt[624];
  int idx;
} mt_state;
static void mt_seed(mt_state *r, unsigned long seed) {
  if (seed == 0) seed = 4357; /* gsl_rng_set for mt19937 */
  r->mt[0] = (unsigned int)(seed & 0xffffffffUL);
  for (int i = 1; i < 624; i++) {
    unsigned int p = r->mt[i - 1];
    r->mt[i] = 1812433253U * (p ^ (p >> 30)) + (unsigned int)i;
  }
  r->idx = 624;
}
static unsigned int mt_next(mt_state *r) {
  if (r->idx >= 624) {
    for (int i = 0; i < 624; i++) {
      unsigned int y = (r->mt[i] & 0x80000000U) | (r->mt[(i + 1) % 624] & 0x7fffffffU);
      unsigned int v = r->mt[(i + 397) % 624] ^ (y >> 1);
      if (y & 1U) v ^= 0x9908b0dfU;
      r->mt[i] = v;
    }
    r->idx = 0;
  }
  unsigned int y = r->mt[r->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680U;
  y ^= (y << 15) & 0xefc60000U;
  y ^= y >> 18;
  return y;
}
/* uniform(0,1) = gsl_ran_flat(rng, 0, 1) (MDcode/initialise.c:19-21) */
static double mt_flat01(mt_state *r) {
  double u = (double)mt_next(r) / 4294967296.0;
  return 0.0 * (1.0 - u) + 1.0 * u;
}

/* ------------------------------------------------------------------------ */
typedef struct {
  int *v;
  int n, cap;
} ivec;
static void iv_push(ivec *a, int x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? 2 * a->cap : 64;
    a->v = (int *)realloc(a->v, sizeof(int) * (size_t)a->cap);
  }
  a->v[a->n++] = x;
}

struct ora_sys {
  int n, nact, tau_p, list_mode;
  double L, invL, T, f0, rebuild_factor, dof;
  double *x, *y, *z, *xu, *yu, *zu, *px, *py, *pz, *Fx, *Fy, *Fz, *xold, *yold, *zold;
  int *type, *act, *kx, *ky, *kz;
  double eta[NHC_M], p_eta[NHC_M], q[NHC_M];
  double pe, ke, vir, viract, inst_T, maxD;
  int ncx, ncy, ncz, ncell;
  double invx, invy, invz;
  int *cell_count;
  ivec *cells;
  ivec *nb;
  mt_state rng;
};

/* Parallel.c:71-80 at one rank (Lpp = L): the (int) cast binds to L, so the
 * count is trunc(trunc(L) / Cell_cut); InvCellSize = L / (L / Nc). */
void ora_cell_geometry(double L, int *nc3, double *inv3) {
  int nc = (int)((double)(int)L / CELL_CUT);
  double cs = L / (double)nc;
  for (int d = 0; d < 3; d++) {
    nc3[d] = nc;
    inv3[d] = L / cs;
  }
}

ora_sys *ora_create(int n, int nact, double L, double T, double f0, int tau_p_steps,
                    double rebuild_factor, int list_mode) {
  ora_sys *s = (ora_sys *)calloc(1, sizeof(ora_sys));
  s->n = n;
  s->nact = nact;
  s->L = L;
  s->invL = 1.0 / L;
  s->T = T;
  s->f0 = f0;
  s->tau_p = tau_p_steps;
  s->rebuild_factor = rebuild_factor;
  s->list_mode = list_mode;
  s->dof = 3.0 * (double)n - 3.0; /* MDcode/global.h:35 */
  double **arrs[] = {&s->x,  &s->y,  &s->z,  &s->xu, &s->yu,   &s->zu,   &s->px,  &s->py,
                     &s->pz, &s->Fx, &s->Fy, &s->Fz, &s->xold, &s->yold, &s->zold};
  for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); a++)
    *arrs[a] = (double *)calloc((size_t)n, sizeof(double));
  s->type = (int *)calloc((size_t)n, sizeof(int));
  s->act = (int *)calloc((size_t)n, sizeof(int));
  s->kx = (int *)calloc((size_t)(nact > 0 ? nact : 1), sizeof(int));
  s->ky = (int *)calloc((size_t)(nact > 0 ? nact : 1), sizeof(int));
  s->kz = (int *)calloc((size_t)(nact > 0 ? nact : 1), sizeof(int));
  int nc3[3];
  double inv3[3];
  ora_cell_geometry(L, nc3, inv3);
  s->ncx = nc3[0];
  s->ncy = nc3[1];
  s->ncz = nc3[2];
  s->ncell = s->ncx * s->ncy * s->ncz;
  s->invx = inv3[0];
  s->invy = inv3[1];
  s->invz = inv3[2];
  s->cell_count = (int *)calloc((size_t)s->ncell, sizeof(int));
  s->cells = (ivec *)calloc((size_t)s->ncell, sizeof(ivec));
  s->nb = (ivec *)calloc((size_t)n, sizeof(ivec));
  /* q per InitialiseNoseHoover (MDcode/time_evolve.c:476-482) */
  for (int i = 0; i < NHC_M; i++) s->q[i] = T * TAU_T * TAU_T;
  s->q[0] = s->dof * T * TAU_T * TAU_T;
  mt_seed(&s->rng, 5489UL);
  return s;
}

void ora_destroy(ora_sys *s) {
  if (!s) return;
  double *arrs[] = {s->x,  s->y,  s->z,  s->xu, s->yu,   s->zu,   s->px,  s->py,
                    s->pz, s->Fx, s->Fy, s->Fz, s->xold, s->yold, s->zold};
  for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); a++) free(arrs[a]);
  free(s->type);
  free(s->act);
  free(s->kx);
  free(s->ky);
  free(s->kz);
  for (int c = 0; c < s->ncell; c++) free(s->cells[c].v);
  free(s->cells);
  free(s->cell_count);
  for (int i = 0; i < s->n; i++) free(s->nb[i].v);
  free(s->nb);
  free(s);
}

void ora_set_state(ora_sys *s, const double *x, const double *xu, const double *p,
                   const int *type, const int *act_tag) {
  for (int i = 0; i < s->n; i++) {
    s->x[i] = x[3 * i];
    s->y[i] = x[3 * i + 1];
    s->z[i] = x[3 * i + 2];
    s->xu[i] = xu ? xu[3 * i] : x[3 * i];
    s->yu[i] = xu ? xu[3 * i + 1] : x[3 * i + 1];
    s->zu[i] = xu ? xu[3 * i + 2] : x[3 * i + 2];
    s->px[i] = p[3 * i];
    s->py[i] = p[3 * i + 1];
    s->pz[i] = p[3 * i + 2];
    s->Fx[i] = s->Fy[i] = s->Fz[i] = 0.0;
    s->type[i] = type[i];
    s->act[i] = act_tag[i];
  }
}

void ora_get_state(const ora_sys *s, double *x, double *xu, double *p, double *F) {
  for (int i = 0; i < s->n; i++) {
    if (x) {
      x[3 * i] = s->x[i];
      x[3 * i + 1] = s->y[i];
      x[3 * i + 2] = s->z[i];
    }
    if (xu) {
      xu[3 * i] = s->xu[i];
      xu[3 * i + 1] = s->yu[i];
      xu[3 * i + 2] = s->zu[i];
    }
    if (p) {
      p[3 * i] = s->px[i];
      p[3 * i + 1] = s->py[i];
      p[3 * i + 2] = s->pz[i];
    }
    if (F) {
      F[3 * i] = s->Fx[i];
      F[3 * i + 1] = s->Fy[i];
      F[3 * i + 2] = s->Fz[i];
    }
  }
}

void ora_set_k(ora_sys *s, const int *k) {
  for (int a = 0; a < s->nact; a++) {
    s->kx[a] = k[a];
    s->ky[a] = k[s->nact + a];
    s->kz[a] = k[2 * s->nact + a];
  }
}
void ora_get_k(const ora_sys *s, int *k) {
  for (int a = 0; a < s->nact; a++) {
    k[a] = s->kx[a];
    k[s->nact + a] = s->ky[a];
    k[2 * s->nact + a] = s->kz[a];
  }
}

void ora_set_nhc(ora_sys *s, const double *eta, const double *p_eta) {
  for (int i = 0; i < NHC_M; i++) {
    s->eta[i] = eta[i];
    s->p_eta[i] = p_eta[i];
  }
}
void ora_get_nhc(const ora_sys *s, double *out9) {
  for (int i = 0; i < NHC_M; i++) {
    out9[i] = s->eta[i];
    out9[NHC_M + i] = s->p_eta[i];
    out9[2 * NHC_M + i] = s->q[i];
  }
}
void ora_set_thermostat(ora_sys *s, double T) {
  s->T = T;
  for (int i = 0; i < NHC_M; i++) s->q[i] = T * TAU_T * TAU_T;
  s->q[0] = s->dof * T * TAU_T * TAU_T;
}

void ora_seed_rng(ora_sys *s, unsigned long seed) { mt_seed(&s->rng, seed); }

/* ShuffleActDirec (MDcode/active.c:45-85): per component, for each i swap
 * k[i] with k[j], j = (int)(Nact * uniform(0,1)). */
void ora_shuffle(ora_sys *s) {
  int *comp[3] = {s->kx, s->ky, s->kz};
  for (int c = 0; c < 3; c++) {
    int *k = comp[c];
    for (int i = 0; i < s->nact; i++) {
      int j = (int)((double)s->nact * mt_flat01(&s->rng));
      int t = k[i];
      k[i] = k[j];
      k[j] = t;
    }
  }
}

/* getcell_I (MDcode/cell_list+forces.c:24-28) */
static int getcell(const ora_sys *s, int ix, int iy, int iz) {
  return ((ix + s->ncx * 3) % s->ncx) + ((iy + s->ncy * 3) % s->ncy) * s->ncx +
         ((iz + s->ncz * 3) % s->ncz) * s->ncx * s->ncy;
}

/* pair distance^2 in absolute units with the reference's minimum image
 * (MDcode/cell_list+forces.c:89-98) */
static double pair_dr2(const ora_sys *s, int a, int b) {
  double dx = s->x[a] - s->x[b], dy = s->y[a] - s->y[b], dz = s->z[a] - s->z[b];
  if (dx < -HALF_LENGTH) dx += LENGTH;
  if (dx > HALF_LENGTH) dx -= LENGTH;
  if (dy < -HALF_LENGTH) dy += LENGTH;
  if (dy > HALF_LENGTH) dy -= LENGTH;
  if (dz < -HALF_LENGTH) dz += LENGTH;
  if (dz > HALF_LENGTH) dz -= LENGTH;
  return (dx * dx + dy * dy + dz * dz) * s->L * s->L;
}

static double list_cut_sq(const ora_sys *s, int ta, int tb) {
  if (s->list_mode == 0) return CELL_CUT * CELL_CUT;
  double rc = 2.5 * SIGMA[ta][tb] + SKIN;
  return rc * rc;
}

static void consider(ora_sys *s, int a, int b) {
  if (pair_dr2(s, a, b) < list_cut_sq(s, s->type[a], s->type[b])) iv_push(&s->nb[a], b);
}

/* update_cell_list (MDcode/cell_list+forces.c:58-148) at one rank. */
void ora_rebuild(ora_sys *s) {
  s->maxD = 0.0;
  for (int c = 0; c < s->ncell; c++) s->cells[c].n = 0;
  for (int i = 0; i < s->n; i++) s->nb[i].n = 0;
  /* binning, ascending i (:71-80); out-of-range indices are clamped */
  for (int i = 0; i < s->n; i++) {
    double fx = floor(s->x[i] * s->invx), fy = floor(s->y[i] * s->invy),
           fz = floor(s->z[i] * s->invz);
    if (fx >= s->ncx) fx = s->ncx - 1;
    if (fy >= s->ncy) fy = s->ncy - 1;
    if (fz >= s->ncz) fz = s->ncz - 1;
    if (fx < 0) fx = 0;
    if (fy < 0) fy = 0;
    if (fz < 0) fz = 0;
    int c = (int)(fx + fy * s->ncx + fz * s->ncx * s->ncy);
    iv_push(&s->cells[c], i);
  }
  for (int c = 0; c < s->ncell; c++) s->cell_count[c] = s->cells[c].n;
  /* intra-cell pairs j<k in in-cell order (:82-105) */
  for (int c = 0; c < s->ncell; c++) {
    const ivec *cl = &s->cells[c];
    for (int j = 0; j < cl->n - 1; j++)
      for (int k = j + 1; k < cl->n; k++) consider(s, cl->v[j], cl->v[k]);
  }
  int full = s->ncx >= 3 && s->ncy >= 3 && s->ncz >= 3;
  if (full) {
    /* the 13 half-neighbour cells of maps() (:32-54), visited per cell in
     * ascending cell order (:107-140) */
    static const int off[13][3] = {{1, 0, 0},  {1, 1, 0},  {0, 1, 0},  {-1, 1, 0}, {1, 0, -1},
                                   {1, 1, -1}, {0, 1, -1}, {-1, 1, -1}, {1, 0, 1}, {1, 1, 1},
                                   {0, 1, 1},  {-1, 1, 1}, {0, 0, 1}};
    for (int c = 0; c < s->ncell; c++) {
      if (s->cells[c].n == 0) continue;
      int ix = c % s->ncx, iy = (c / s->ncx) % s->ncy, iz = c / (s->ncx * s->ncy);
      for (int m = 0; m < 13; m++) {
        int c2 = getcell(s, ix + off[m][0], iy + off[m][1], iz + off[m][2]);
        const ivec *a = &s->cells[c], *b = &s->cells[c2];
        if (b->n == 0) continue;
        for (int i = 0; i < a->n; i++)
          for (int j = 0; j < b->n; j++) consider(s, a->v[i], b->v[j]);
      }
    }
  } else {
    /* fewer than 3 cells on a side: the 26 offsets repeat cells, so visit
     * every distinct pair of distinct cells (c < c2) once instead */
    for (int c = 0; c < s->ncell; c++) {
      int ix = c % s->ncx, iy = (c / s->ncx) % s->ncy, iz = c / (s->ncx * s->ncy);
      int seen[27], ns = 0;
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            int c2 = getcell(s, ix + dx, iy + dy, iz + dz);
            if (c2 <= c) continue;
            int dup = 0;
            for (int t = 0; t < ns; t++) dup |= seen[t] == c2;
            if (dup) continue;
            seen[ns++] = c2;
            const ivec *a = &s->cells[c], *b = &s->cells[c2];
            for (int i = 0; i < a->n; i++)
              for (int j = 0; j < b->n; j++) consider(s, a->v[i], b->v[j]);
          }
    }
  }
  /* (:141-146) */
  for (int i = 0; i < s->n; i++) {
    s->xold[i] = s->xu[i];
    s->yold[i] = s->yu[i];
    s->zold[i] = s->zu[i];
  }
}

/* calculate_forces (MDcode/cell_list+forces.c:153-227) at one rank (factor 1) */
static void compute_forces(ora_sys *s) {
  double pe = 0.0, vir = 0.0, viract = 0.0, L = s->L;
  for (int i = 0; i < s->n; i++) s->Fx[i] = s->Fy[i] = s->Fz[i] = 0.0;
  for (int i = 0; i < s->n; i++) {
    int A = s->type[i];
    const ivec *l = &s->nb[i];
    for (int k = 0; k < l->n; k++) {
      int j = l->v[k], B = s->type[j];
      double dx = s->x[i] - s->x[j], dy = s->y[i] - s->y[j], dz = s->z[i] - s->z[j];
      if (dx < -HALF_LENGTH) dx += LENGTH;
      if (dx > HALF_LENGTH) dx -= LENGTH;
      if (dy < -HALF_LENGTH) dy += LENGTH;
      if (dy > HALF_LENGTH) dy -= LENGTH;
      if (dz < -HALF_LENGTH) dz += LENGTH;
      if (dz > HALF_LENGTH) dz -= LENGTH;
      double dr2 = (dx * dx + dy * dy + dz * dz) * L * L;
      double eps = EPSILON[A][B], sig = SIGMA[A][B];
      double rs2 = dr2 / (sig * sig);
      if (rs2 < LCUT_SQR) {
        double s2 = 1.0 / rs2;
        double s6 = s2 * s2 * s2;
        pe += 1.0 * 4.0 * eps * ((s6 * (s6 - 1.0)) + C0 + C2 * rs2);
        double grad = 8.0 * eps * (6.0 * s6 * (s6 - 0.5) / dr2 - C2 / (sig * sig));
        s->Fx[i] += grad * dx * L;
        s->Fy[i] += grad * dy * L;
        s->Fz[i] += grad * dz * L;
        s->Fx[j] -= grad * dx * L;
        s->Fy[j] -= grad * dy * L;
        s->Fz[j] -= grad * dz * L;
        vir += 1.0 * grad * dr2;
      }
    }
  }
  for (int i = 0; i < s->n; i++) {
    int a = s->act[i];
    if (a != -1) {
      s->Fx[i] += s->f0 * (double)s->kx[a];
      s->Fy[i] += s->f0 * (double)s->ky[a];
      s->Fz[i] += s->f0 * (double)s->kz[a];
      viract += s->f0 * ((double)s->kx[a] * s->xu[i] + (double)s->ky[a] * s->yu[i] +
                         (double)s->kz[a] * s->zu[i]);
    }
  }
  s->pe = pe;
  s->vir = vir / (3.0e0);
  s->viract = viract;
}

void ora_forces(ora_sys *s, double *F, double *out3) {
  compute_forces(s);
  if (F)
    for (int i = 0; i < s->n; i++) {
      F[3 * i] = s->Fx[i];
      F[3 * i + 1] = s->Fy[i];
      F[3 * i + 2] = s->Fz[i];
    }
  if (out3) {
    out3[0] = s->pe;
    out3[1] = s->vir;
    out3[2] = s->viract;
  }
}

/* applypbc1 (MDcode/time_evolve.c:15-26) */
static void wrap(double *v) {
  while (*v >= LENGTH) *v -= LENGTH;
  while (*v < 0.0) *v += LENGTH;
}

/* U1Propagator (MDcode/time_evolve.c:527-557) */
static void u1(ora_sys *s) {
  for (int i = 0; i < s->n; i++) {
    double dx = s->px[i] * TIME_STEP, dy = s->py[i] * TIME_STEP, dz = s->pz[i] * TIME_STEP;
    s->x[i] += dx * s->invL;
    s->xu[i] += dx * s->invL;
    s->y[i] += dy * s->invL;
    s->yu[i] += dy * s->invL;
    s->z[i] += dz * s->invL;
    s->zu[i] += dz * s->invL;
  }
  for (int i = 0; i < s->n; i++) {
    wrap(&s->x[i]);
    wrap(&s->y[i]);
    wrap(&s->z[i]);
  }
  double m = 0.0;
  for (int i = 0; i < s->n; i++) {
    double dx = s->xu[i] - s->xold[i], dy = s->yu[i] - s->yold[i], dz = s->zu[i] - s->zold[i];
    double t = dx * dx + dy * dy + dz * dz;
    if (m < t) m = t;
  }
  m *= s->L * s->L;
  s->maxD = m;
}

/* U2Propagator (MDcode/time_evolve.c:558-567) */
static void u2(ora_sys *s) {
  for (int i = 0; i < s->n; i++) {
    s->px[i] += s->Fx[i] * HALF_TIME_STEP;
    s->py[i] += s->Fy[i] * HALF_TIME_STEP;
    s->pz[i] += s->Fz[i] * HALF_TIME_STEP;
  }
}

/* U3Propagator (MDcode/time_evolve.c:568-577) */
static void u3(ora_sys *s, double t) {
  for (int i = 0; i < s->n; i++) {
    s->px[i] = s->px[i] * exp(-t * s->p_eta[0] / s->q[0]);
    s->py[i] = s->py[i] * exp(-t * s->p_eta[0] / s->q[0]);
    s->pz[i] = s->pz[i] * exp(-t * s->p_eta[0] / s->q[0]);
  }
  for (int i = 0; i < NHC_M; i++) s->eta[i] = s->eta[i] + t * s->p_eta[i] / s->q[i];
}

/* U4Propagator (MDcode/time_evolve.c:578-609): chain sweep jStart..jEnd */
static void u4(ora_sys *s, double t, int j0, int j1) {
  int dj = j0 > j1 ? -1 : 1;
  int j = j0;
  double gj = 0.0;
  do {
    if (j == 0) {
      double kb = 0.0;
      for (int i = 0; i < s->n; i++)
        kb += s->px[i] * s->px[i] + s->py[i] * s->py[i] + s->pz[i] * s->pz[i];
      gj = kb;
      s->ke = gj;
      gj -= s->dof * s->T;
    } else {
      gj = (s->p_eta[j - 1] * s->p_eta[j - 1]) / s->q[j - 1] - s->T;
    }
    if (j == NHC_M - 1) {
      s->p_eta[j] = s->p_eta[j] + t * gj;
    } else {
      double xx = t * s->p_eta[j + 1] / s->q[j + 1];
      s->p_eta[j] = s->p_eta[j] * exp(-xx) + t * gj * (1.0 - exp(-xx)) / xx;
    }
    j = j + dj;
  } while (j - dj != j1);
}

static int maybe_rebuild(ora_sys *s) {
  if (s->rebuild_factor * s->maxD > SKIN * SKIN) {
    ora_rebuild(s);
    return 1;
  }
  return 0;
}

/* AdvanceTimeNVTNoseHoover (MDcode/time_evolve.c:495-526) */
static int nvt_step(ora_sys *s) {
  u4(s, TIME_STEP * 0.25, NHC_M - 1, 0);
  u3(s, TIME_STEP * 0.50);
  u4(s, TIME_STEP * 0.25, 0, NHC_M - 1);
  u2(s);
  u1(s);
  double maxd = s->maxD;
  int rb = maybe_rebuild(s);
  s->maxD = maxd;
  compute_forces(s);
  u2(s);
  u4(s, TIME_STEP * 0.25, NHC_M - 1, 0);
  u3(s, TIME_STEP * 0.50);
  u4(s, TIME_STEP * 0.25, 0, NHC_M - 1);
  s->ke = s->ke * 0.5;
  s->inst_T = 2.0 * s->ke / s->dof;
  return rb;
}

/* fixDrift (MDcode/initialise.c:104-138): subtract the mean momentum, the
 * sums taken over the particles in index order, one component at a time */
void ora_fix_drift(ora_sys *s) {
  double P[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < s->n; i++) {
    P[0] += s->px[i];
    P[1] += s->py[i];
    P[2] += s->pz[i];
  }
  for (int k = 0; k < 3; k++) P[k] = P[k] / (double)s->n;
  for (int i = 0; i < s->n; i++) {
    s->px[i] -= P[0];
    s->py[i] -= P[1];
    s->pz[i] -= P[2];
  }
}

/* run() loop body (MDcode/main.c:244-265): ShuffleActDirec every TAU_per
 * steps, the step, and fixDrift after every 100000th step when do_drift */
int ora_run(ora_sys *s, long start, int nsteps, int do_shuffle, int do_drift) {
  int rebuilds = 0;
  for (long i = start; i < start + nsteps; i++) {
    if (do_shuffle && !(i % s->tau_p)) ora_shuffle(s);
    rebuilds += nvt_step(s);
    if (do_drift && i % 100000 == 0) ora_fix_drift(s);
  }
  return rebuilds;
}

/* calculate_temp (MDcode/initialise.c:153-164) */
static double inst_temp(ora_sys *s) {
  double kb = 0.0;
  for (int i = 0; i < s->n; i++) kb += s->px[i] * s->px[i] + s->py[i] * s->py[i] + s->pz[i] * s->pz[i];
  s->ke = kb * 0.5;
  s->inst_T = 2.0 * s->ke / s->dof;
  return s->inst_T;
}

/* adjustInitialTemp (MDcode/initialise.c:141-151); returns inst_T after */
double ora_adjust_temp(ora_sys *s, double T) {
  double xi = sqrt(T / inst_temp(s));
  for (int i = 0; i < s->n; i++) {
    s->px[i] = s->px[i] * xi;
    s->py[i] = s->py[i] * xi;
    s->pz[i] = s->pz[i] * xi;
  }
  return inst_temp(s);
}

/* coldstart / breakxal (MDcode/initialise.c:166-201): rescale to T_start,
 * rebuild and compute forces, then while T has not reached T_end (T < T_end
 * heating, T > T_end cooling): rescale to T, one NVE leap-frog step,
 * T +- time_step * rate.  Returns the number of ramp steps. */
long ora_ramp(ora_sys *s, double T_start, double T_end, double rate) {
  double T = ora_adjust_temp(s, T_start);
  const int heat = T_end > T_start;
  ora_rebuild(s);
  compute_forces(s);
  long k = 0;
  while (heat ? T < T_end : T > T_end) {
    inst_temp(s);
    ora_adjust_temp(s, T);
    ora_run_nve(s, 1);
    if (heat)
      T += TIME_STEP * rate;
    else
      T -= TIME_STEP * rate;
    k++;
  }
  return k;
}

/* advance_time_NVEFrog (MDcode/time_evolve.c:104-171) */
int ora_run_nve(ora_sys *s, int nsteps) {
  int rebuilds = 0;
  for (int st = 0; st < nsteps; st++) {
    u2(s);
    u1(s);
    double maxd = s->maxD;
    rebuilds += maybe_rebuild(s);
    s->maxD = maxd;
    compute_forces(s);
    double kb = 0.0;
    for (int i = 0; i < s->n; i++) {
      s->px[i] += s->Fx[i] * HALF_TIME_STEP;
      s->py[i] += s->Fy[i] * HALF_TIME_STEP;
      s->pz[i] += s->Fz[i] * HALF_TIME_STEP;
      kb += s->px[i] * s->px[i] + s->py[i] * s->py[i] + s->pz[i] * s->pz[i];
    }
    s->ke = 0.5 * kb;
    s->inst_T = 2.0 * s->ke / s->dof;
  }
  return rebuilds;
}

void ora_get_scalars(const ora_sys *s, double *out6) {
  out6[0] = s->pe;
  out6[1] = s->ke;
  out6[2] = s->vir;
  out6[3] = s->viract;
  out6[4] = s->inst_T;
  out6[5] = s->maxD;
}

int ora_get_cells(const ora_sys *s, int *dims, int *counts, int *members) {
  dims[0] = s->ncx;
  dims[1] = s->ncy;
  dims[2] = s->ncz;
  int m = 0;
  for (int c = 0; c < s->ncell; c++) {
    if (counts) counts[c] = s->cells[c].n;
    if (members)
      for (int j = 0; j < s->cells[c].n; j++) members[m++] = s->cells[c].v[j];
  }
  return s->ncell;
}

long ora_get_neighbors(const ora_sys *s, int *counts, int *pairs) {
  long m = 0;
  for (int i = 0; i < s->n; i++) {
    if (counts) counts[i] = s->nb[i].n;
    for (int k = 0; k < s->nb[i].n; k++) {
      if (pairs) {
        pairs[2 * m] = i;
        pairs[2 * m + 1] = s->nb[i].v[k];
      }
      m++;
    }
  }
  return m;
}

/* prepareSavingArray (MDcode/main.c:62-119): origins k*(run/numOrigins);
 * offsets 1, then *factor with integer truncation (+1 when that does not
 * advance), kept while below runLength; then sorted and de-duplicated. */
static int cmp_u64(const void *a, const void *b) {
  unsigned long long x = *(const unsigned long long *)a, y = *(const unsigned long long *)b;
  return (x > y) - (x < y);
}
int ora_log_schedule(unsigned long long run_length, int num_origins, double factor,
                     unsigned long long *out, int cap) {
  unsigned long long lin = run_length / (unsigned long long)num_origins;
  unsigned long long maxi = run_length;
  size_t n = 0, ncap = 1024;
  unsigned long long *v = (unsigned long long *)malloc(ncap * sizeof(*v));
  for (unsigned long long k = 0; k < (unsigned long long)num_origins; k++) {
    if (n == ncap) v = (unsigned long long *)realloc(v, (ncap *= 2) * sizeof(*v));
    v[n++] = k * lin;
    unsigned long long off = 1;
    while (off < maxi) {
      unsigned long long idx = k * lin + off;
      if (idx < run_length) {
        if (n == ncap) v = (unsigned long long *)realloc(v, (ncap *= 2) * sizeof(*v));
        v[n++] = idx;
      }
      if ((unsigned long long)(off * factor) == off)
        off++;
      else
        off = (unsigned long long)((double)off * factor);
    }
  }
  /* shellSort (MDcode/main.c:17-41) is the 1-based Numerical Recipes routine
   * but is called on the 0-based array: it sorts v[1..n], i.e. it leaves v[0]
   * (= 0) in place and pulls in the element one past the end, which is zero
   * in a fresh allocation.  The net effect is that one copy of the largest
   * value among v[1..n-1] is replaced by 0, a duplicate of v[0]. */
  if (n >= 2) {
    size_t imax = 1;
    for (size_t i = 2; i < n; i++)
      if (v[i] > v[imax]) imax = i;
    v[imax] = 0;
  }
  qsort(v, n, sizeof(*v), cmp_u64);
  int m = 0;
  for (size_t i = 0; i < n; i++)
    if (i == 0 || v[i] != v[i - 1]) {
      if (m < cap) out[m] = v[i];
      m++;
    }
  free(v);
  return m;
}
