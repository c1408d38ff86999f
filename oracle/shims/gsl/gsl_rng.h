/*
 * Minimal GSL random-number shim — test infrastructure for the oracle only.
 *
 * The reference (MDcode/initialise.c:5-21, active.c:59-71) draws from GSL's
 * MT19937 generator through gsl_rng_alloc / gsl_rng_set / gsl_ran_flat.  GSL is
 * not installed here, so this shim supplies those calls.  The generator is the
 * Mersenne Twister written from its published description (Matsumoto &
 * Nishimura, ACM TOMACS 8(1), 1998).  Bit parity with GSL's stream is not
 * needed: every seed in the reference derives from time(), so no reference
 * run is reproducible and parity tests hand identical active directions and
 * thermostat momenta to both sides instead.
 */
#ifndef ACG_ORACLE_GSL_RNG_H
#define ACG_ORACLE_GSL_RNG_H
typedef struct { int id; } gsl_rng_type;
typedef struct {
  unsigned int mt[624];
  int idx;
} gsl_rng;
extern const gsl_rng_type *gsl_rng_mt19937;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *t);
void gsl_rng_set(gsl_rng *r, unsigned long int seed);
unsigned long int gsl_rng_get(gsl_rng *r);
double gsl_rng_uniform(gsl_rng *r);
#endif
