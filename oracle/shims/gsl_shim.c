/*
 * GSL shim implementation — oracle test infrastructure (see gsl/gsl_rng.h).
 * MT19937 per Matsumoto & Nishimura (1998): 624-word state, twist with the
 * matrix A of the paper, tempering by the paper's (u,s,b,t,c,l) parameters.
 */
#include "gsl/gsl_rng.h"
#include "gsl/gsl_randist.h"
#include <math.h>
#include <stdlib.h>

static const gsl_rng_type mt_type = {19937};
const gsl_rng_type *gsl_rng_mt19937 = &mt_type;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *t) {
  (void)t;
  gsl_rng *r = (gsl_rng *)calloc(1, sizeof(gsl_rng));
  gsl_rng_set(r, 5489UL);
  return r;
}

void gsl_rng_set(gsl_rng *r, unsigned long int seed) {
  if (seed == 0) seed = 4357; /* GSL's mt19937 takes seed 0 as 4357 */
  r->mt[0] = (unsigned int)(seed & 0xffffffffUL);
  for (int i = 1; i < 624; i++) {
    unsigned int p = r->mt[i - 1];
    r->mt[i] = 1812433253U * (p ^ (p >> 30)) + (unsigned int)i;
  }
  r->idx = 624;
}

static void twist(gsl_rng *r) {
  for (int i = 0; i < 624; i++) {
    unsigned int y = (r->mt[i] & 0x80000000U) | (r->mt[(i + 1) % 624] & 0x7fffffffU);
    unsigned int v = r->mt[(i + 397) % 624] ^ (y >> 1);
    if (y & 1U) v ^= 0x9908b0dfU;
    r->mt[i] = v;
  }
  r->idx = 0;
}

unsigned long int gsl_rng_get(gsl_rng *r) {
  if (r->idx >= 624) twist(r);
  unsigned int y = r->mt[r->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680U;
  y ^= (y << 15) & 0xefc60000U;
  y ^= y >> 18;
  return y;
}

double gsl_rng_uniform(gsl_rng *r) { return (double)gsl_rng_get(r) / 4294967296.0; }

double gsl_ran_flat(gsl_rng *r, double a, double b) {
  double u = gsl_rng_uniform(r);
  return a * (1.0 - u) + b * u;
}

/* Off the hot path (MDcode/initialise.c:13-17, used only by the Brownian
 * integrators).  Box-Muller is enough for the oracle. */
double gsl_ran_gaussian_ziggurat(gsl_rng *r, double sigma) {
  double u1 = 1.0 - gsl_rng_uniform(r), u2 = gsl_rng_uniform(r);
  return sigma * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}
