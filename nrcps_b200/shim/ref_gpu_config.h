/*
 * ref_gpu_config.h -- forced pre-include for building the reference's class
 * layer in its GPU configuration against libnrcps_b200.
 *
 * The reference selects backends in include/config.h:13-33 (USE_MPI,
 * USE_GPU, precision, BLOCKS/THREADS).  This header defines the same guard
 * and names for a single-process FP64 GPU build, so that the reference's
 * common translation units (the .C files directly under each src module)
 * compile with their USE_GPU paths, and the shims in this directory stand
 * in for the modules' cuda units.
 */
#ifndef INCLUDED_CONFIG
#define INCLUDED_CONFIG

#define VERSION_MAJOR 2
#define VERSION_MINOR 7
#define VERSION_SUB 6
#define VERSION_STR "nrCPS_v2_7_6"

#define USE_GPU
#define USE_DOUBLE
#define BLOCKS 128
#define THREADS 112
const int PREC = 15;
typedef double Float;

#endif
