/*
 * CPU-only stand-in for the reference header rhic/include/HydroParameters.h.
 *
 * Test infrastructure: used only to compile the reference's own CPU sources
 * into oracle/_ref/. The shipped header includes DynamicalVariables.cuh, whose
 * typedefs clash with the CPU DynamicalVariables.h; this stand-in declares the
 * same struct (rhic/include/HydroParameters.h:15-21, field order and types are
 * part of the reference's plugin interface) without that include.
 */
#ifndef HYDROPARAMETERS_H_
#define HYDROPARAMETERS_H_

#include <libconfig.h>

struct HydroParameters {
    double initialProperTimePoint;
    double shearViscosityToEntropyDensity;
    double freezeoutTemperatureGeV;
    int initializePimunuNavierStokes;
};

void loadHydroParameters(config_t *cfg, const char *configDirectory, void *params);

#endif
