/* Project-written stand-in for GSL's random-distribution header (test oracle
 * build only). The reference draws move types with
 * gsl_ran_bernoulli(MCRng, 0.5) (simulation engine/src/Replica.cpp:388). */
#ifndef REMC_ORACLE_STUB_GSL_RANDIST_H
#define REMC_ORACLE_STUB_GSL_RANDIST_H
#include "gsl_rng.h"
static inline unsigned int gsl_ran_bernoulli(gsl_rng* r, double p) {
  return gsl_rng_uniform(r) < p ? 1u : 0u;
}
#endif
