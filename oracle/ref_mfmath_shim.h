/* Forced include for the mfmath build of the translated reference
 * (TEST INFRASTRUCTURE ONLY): the reference's exp/log/erf calls go to the
 * solver's own functions, so this build and the GPU path use identical
 * transcendentals and can be compared bit for bit. */
#pragma once
#include <math.h>
#include "../3d-mfcfd_b200/csrc/mfmath.h"
#define exp(x) mf_exp(x)
#define log(x) mf_log(x)
#define erf(x) mf_erf(x)
