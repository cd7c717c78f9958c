/*
 * vah_plugin.h -- the reference's driver/plugin surface over libvah
 * (libvah_host.so and the gpu-vah executable).
 *
 * Keeps the reference's input surface so it is a drop-in: the three
 * parameter structs with the reference's field order and types, the
 * <dir>/{lattice,ic,hydro}.properties files with the same keys and defaults,
 * the run() plugin entry point and the .dat output writer.
 */
#ifndef VAH_PLUGIN_H
#define VAH_PLUGIN_H

#ifdef __cplusplus
extern "C" {
#endif

/* rhic/include/LatticeParameters.h:17-31 */
struct LatticeParameters {
    int numLatticePointsX;
    int numLatticePointsY;
    int numLatticePointsRapidity;
    int numComputationalLatticePointsX;
    int numComputationalLatticePointsY;
    int numComputationalLatticePointsRapidity;
    int numProperTimePoints;
    double latticeSpacingX;
    double latticeSpacingY;
    double latticeSpacingRapidity;
    double latticeSpacingProperTime;
};

/* rhic/include/InitialConditionParameters.h:13-27 */
struct InitialConditionParameters {
    int initialConditionType;
    int numberOfNucleonsPerNuclei;
    double initialEnergyDensity;
    double scatteringCrossSectionNN;
    double impactParameter;
    double fractionOfBinaryCollisions;
    double rapidityVariance;
    double rapidityMean;
};

/* rhic/include/HydroParameters.h:15-21 */
struct HydroParameters {
    double initialProperTimePoint;
    double shearViscosityToEntropyDensity;
    double freezeoutTemperatureGeV;
    int initializePimunuNavierStokes;
};

/* Loaders: <configDirectory>/{lattice,ic,hydro}.properties with the
 * reference's keys and defaults (LatticeParameters.cpp:21-53,
 * InitialConditionParameters.cpp:24-52, HydroParameters.cpp:16-36). A missing
 * file keeps the defaults and prints the reference's warning on stderr.
 * Lookups are type-strict like libconfig without auto-conversion: a key whose
 * literal is an integer does not satisfy a floating-point lookup (and vice
 * versa), so the default is kept. Return 0, or 1 when the file was missing. */
int vah_load_lattice_parameters(const char *configDirectory, struct LatticeParameters *out);
int vah_load_initial_condition_parameters(const char *configDirectory, struct InitialConditionParameters *out);
int vah_load_hydro_parameters(const char *configDirectory, struct HydroParameters *out);

/* FileIO.cpp:14-59: <dir>/<name>_<t %.3f>.dat, one line
 * "%.3f\t%.3f\t%.3f\t%.8f\n" (x, y, eta, value) per interior cell, eta outer,
 * x inner. `var` is a full ghosted array. Returns 0, or -1 if the file could
 * not be written. */
int vah_output(const double *var, double t, const char *pathToOutDir, const char *name,
               const struct LatticeParameters *lattice);

/* HydroPlugin.cpp:130-242 on the GPU: initial conditions, nt+1 RK2 steps,
 * state copied back and written every 10 steps. Physics, EoS and precision
 * options come from the environment (VAH_PHYSICS = ideal|pimunu|pimunu_pi,
 * VAH_EOS = conformal|table, VAH_DEVICE); the defaults match the reference's
 * CPU build (PIMUNU off, conformal EoS). Returns 0 or a VAH_ERR_* code. */
int vah_run_plugin(void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory,
                   const char *outputDir);

#ifdef __cplusplus
}

/* The reference's plugin symbol (rhic/include/HydroPlugin.h:11, C++
 * linkage), so the reference's main (Run.cpp:34-36) links unchanged. */
void run(void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory,
         const char *outputDir);
#endif

#endif
