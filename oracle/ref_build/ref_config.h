/*
 * ref_config.h -- forced pre-include for compiling the reference's CPU path.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference selects its backend in
 * include/config.h:13-23 (USE_MPI on, USE_GPU off, USE_DOUBLE).  There is no
 * MPI here, so this header is force-included (g++ -include) ahead of every
 * reference translation unit.  It defines the same include guard and the
 * same public names (Float, PREC, VERSION_*) for a single-process
 * double-precision CPU build, after which the reference's config.h is a no-op.
 */
#ifndef INCLUDED_CONFIG
#define INCLUDED_CONFIG

#define VERSION_MAJOR 2
#define VERSION_MINOR 7
#define VERSION_SUB 6
#define VERSION_STR "nrCPS_v2_7_6"

#define USE_DOUBLE
const int PREC = 15;
typedef double Float;

#endif
