/*
 * oracle/ref_shim/src/ref_eos_table.cpp -- test infrastructure (CPU checker).
 *
 * Replaces the reference translation unit rhic/src/EquationOfState.cpp in the
 * "table" builds of oracle/_ref: the same five functions
 * (old_cpu-vah_code/include/EquationOfState.h:19-27), answered from the
 * tabulated crossover EoS that the test hands in with vref_set_eos_table().
 * The reference has no tabulated EoS; swapping this TU is how the reference's
 * own time step is run on the 3+1D workloads' EoS.
 */
#include "../include/DynamicalVariables.h"
#include "../include/EquationOfState.h"

#include "vo_eos.h"

extern const double *vref_eos_table;

PRECISION equilibriumPressure(PRECISION e) { return vo_table_lookup(vref_eos_table, e).p; }

PRECISION speedOfSoundSquared(PRECISION e) { return vo_table_lookup(vref_eos_table, e).cs2; }

PRECISION effectiveTemperature(PRECISION e) { return vo_table_lookup(vref_eos_table, e).T; }

/* Inverse of T(e) by bisection in ln e (only the reference's initial
 * conditions and driver printout use it; never on the time step). */
PRECISION equilibriumEnergyDensity(PRECISION T) {
    double lo = -60.0, hi = 60.0;
    for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (vo_table_lookup(vref_eos_table, exp(mid)).T < T) lo = mid; else hi = mid;
    }
    return exp(0.5 * (lo + hi));
}

/* de/dT = s / c_s^2 with s = (e + p) / T. */
PRECISION derivativeEnergyDensityWithRespectToTemperature(PRECISION T) {
    double e = equilibriumEnergyDensity(T);
    vo_eos_point r = vo_table_lookup(vref_eos_table, e);
    return (e + r.p) / T / r.cs2;
}
