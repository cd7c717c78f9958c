/*
 * Force-included into the "table" build of the reference's SourceTerms.cpp,
 * whose zeta/s(T) (SourceTerms.cpp:36-44) the build recipe redirects to the
 * crossover zeta/s of the 3+1D workloads. Test infrastructure only.
 */
#ifndef VREF_ZETA_H
#define VREF_ZETA_H
extern "C" double vref_zeta_over_s(double T);
#endif
