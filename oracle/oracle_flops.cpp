/*
 * oracle_flops.cpp - the oracle built with counting FP64 arithmetic -- TEST
 * INFRASTRUCTURE ONLY.
 *
 * Compiles mfcfd_oracle.cpp with every `double` a CountedDouble
 * (flop_counter.h) and marks the phases of fpi_solver, so a run gives the
 * FP64 operations per phase that the restated reference performs.  The C
 * API is the oracle's own (liboracle_flops.so exports the same oracle_*
 * functions) plus oracle_flops_get / oracle_flops_reset.
 */
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <vector>

#include "flop_counter.h"

FlopTally g_flops[FLOP_PHASES];
int g_flop_phase = 0;

// phases: 0 conserved vector + q variables, 1 q-derivatives + time step,
// 2 flux residual, 3 D_inv (forward sweep's), 4 forward sweep (LdelU and
// the increments), 5 backward sweep (UdelU and the increments), 6 state
// update and residual, 7 anything else (the backward sweep's recomputation
// of D_inv, set-up, bookkeeping)
#define ORACLE_PHASE(k) (g_flop_phase = (k))
#define double CountedDouble
#include "mfcfd_oracle.cpp"
#undef double

extern "C" {

void oracle_flops_reset() {
    for (auto &t : g_flops) t = FlopTally();
    g_flop_phase = 7;
}

// out: FLOP_PHASES rows of 9 counts (add, mul, div, sqrt, fma, exp, log, erf, pow)
void oracle_flops_get(int64_t *out) {
    for (int p = 0; p < FLOP_PHASES; ++p) {
        const FlopTally &t = g_flops[p];
        const int64_t row[9] = {t.add, t.mul, t.div, t.sqrt, t.fma, t.exp_calls, t.log_calls, t.erf_calls,
                                t.pow_calls};
        std::memcpy(out + 9 * p, row, sizeof row);
    }
}

}  // extern "C"
