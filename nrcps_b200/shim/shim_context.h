// shim_context.h -- the one libnrcps_b200 context of a process using the
// reference's class API, and the reference's error path for its failures.
#ifndef NRCPS_SHIM_CONTEXT_H
#define NRCPS_SHIM_CONTEXT_H

#include "nrcps_b200.h"

nrcps_context* nrcps_shim_context();
// Translates a non-OK status into ERR.General(fname, ...), which prints and
// exits as every failure in the reference does (src/utils/error.C:36-46).
void nrcps_shim_check(nrcps_status st, const char* fname);

#endif
