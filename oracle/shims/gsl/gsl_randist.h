/* Minimal GSL distribution shim — oracle test infrastructure (see gsl_rng.h). */
#ifndef ACG_ORACLE_GSL_RANDIST_H
#define ACG_ORACLE_GSL_RANDIST_H
#include "gsl/gsl_rng.h"
double gsl_ran_flat(gsl_rng *r, double a, double b);
double gsl_ran_gaussian_ziggurat(gsl_rng *r, double sigma);
#endif
