/* Project-written stand-in for GSL's quasi-random header (test oracle build
 * only). The reference includes it but every call is commented out
 * (simulation engine/src/Replica.cpp:384). */
#ifndef REMC_ORACLE_STUB_GSL_QRNG_H
#define REMC_ORACLE_STUB_GSL_QRNG_H
struct gsl_qrng { int unused; };
#endif
