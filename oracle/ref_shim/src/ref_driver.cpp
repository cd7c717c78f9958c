/*
 * oracle/ref_shim/src/ref_driver.cpp -- test infrastructure (CPU checker).
 *
 * A C API over the reference's own CPU time step, compiled together with the
 * reference sources (old_cpu-vah_code/src/*.cpp and
 * rhic/src/AnisotropicDistributionFunctions.cpp) straight from the reference
 * tree into oracle/_ref/libvahref_<variant>.so. The reference keeps its state
 * in process globals (DynamicalVariables.h:119-121) and ships no CPU driver;
 * this file plays the part of HydroPlugin.cpp:130-242 for the CPU path:
 * allocate, fill, step with rungeKutta2 + setCurrentConservedVariables,
 * read back. Field ids follow include/vah.h (VAH_F_*).
 */
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../include/DynamicalVariables.h"
#include "../include/LatticeParameters.h"
#include "../include/HydroParameters.h"
#include "../include/FullyDiscreteKurganovTadmorScheme.h"

#include "vo_eos.h"

static struct LatticeParameters g_lat;
static struct HydroParameters g_hydro;
static int g_len = 0;

/* EoS table handed in by the test (table builds only) and the zeta/s the
 * patched SourceTerms.cpp calls (see oracle/Makefile). */
const double *vref_eos_table = 0;
extern "C" double vref_zeta_over_s(double T) { return vo_zeta_crossover(T); }

extern "C" int vref_num_conserved(void) { return NUMBER_CONSERVED_VARIABLES; }

static void free_conserved(CONSERVED_VARIABLES *c) {
    if (!c) return;
    free(c->ttt); free(c->ttx); free(c->tty); free(c->ttn); free(c->pl);
#ifdef PIMUNU
    free(c->pitt); free(c->pitx); free(c->pity); free(c->pitn); free(c->pixx);
    free(c->pixy); free(c->pixn); free(c->piyy); free(c->piyn); free(c->pinn);
#endif
#ifdef PI
    free(c->Pi);
#endif
    free(c);
}

static void free_velocity(FLUID_VELOCITY *v) {
    if (!v) return;
    free(v->ut); free(v->ux); free(v->uy); free(v->un);
    free(v);
}

extern "C" void vref_free(void) {
    if (!g_len) return;
    free_conserved(q); free_conserved(Q); free_conserved(qS);
    free_velocity(u); free_velocity(up); free_velocity(uS);
    free(e); free(p);
    PRECISION **vd = (PRECISION **)validityDomain;
    for (size_t k = 0; k < sizeof(VALIDITY_DOMAIN) / sizeof(PRECISION *); ++k) free(vd[k]);
    free(validityDomain);
    free(fTSol_X1); free(fTSol_Y1); free(fTSol_1);
    free(fTSol_X2); free(fTSol_Y2); free(fTSol_2);
    q = Q = qS = 0; u = up = uS = 0; e = p = 0; validityDomain = 0;
    g_len = 0;
}

/* The reference's validity arrays (VALIDITY_DOMAIN, DynamicalVariables.h:86-117),
 * member k in declaration order; checkValidity fills them at the end of every
 * rungeKutta2 (FullyDiscreteKurganovTadmorScheme.cpp:791). */
extern "C" PRECISION *vref_validity(int k) {
    if (!validityDomain || k < 0 || (size_t)k >= sizeof(VALIDITY_DOMAIN) / sizeof(PRECISION *)) return 0;
    return ((PRECISION **)validityDomain)[k];
}

/* Allocate the reference globals for an nx*ny*nz interior grid (2 ghost
 * layers per side, LatticeParameters.cpp:45-47). */
extern "C" int vref_init(int nx, int ny, int nz, double dx, double dy, double dz,
                         double dt, double etabar, double t0) {
    vref_free();
    g_lat.numLatticePointsX = nx;
    g_lat.numLatticePointsY = ny;
    g_lat.numLatticePointsRapidity = nz;
    g_lat.numComputationalLatticePointsX = nx + N_GHOST_CELLS;
    g_lat.numComputationalLatticePointsY = ny + N_GHOST_CELLS;
    g_lat.numComputationalLatticePointsRapidity = nz + N_GHOST_CELLS;
    g_lat.numProperTimePoints = 0;
    g_lat.latticeSpacingX = dx;
    g_lat.latticeSpacingY = dy;
    g_lat.latticeSpacingRapidity = dz;
    g_lat.latticeSpacingProperTime = dt;
    g_hydro.initialProperTimePoint = t0;
    g_hydro.shearViscosityToEntropyDensity = etabar;
    g_hydro.freezeoutTemperatureGeV = 0.155;
    g_hydro.initializePimunuNavierStokes = 0;
    g_len = (nx + 4) * (ny + 4) * (nz + 4);
    allocateHostMemory(g_len);
    return g_len;
}

extern "C" void vref_set_eos_table(const double *tab) { vref_eos_table = tab; }

/* Pointer to the current array behind a field id (valid until the next
 * step, which swaps q<->Q and u<->up). */
extern "C" double *vref_field(int id) {
    switch (id) {
    case 0: return q->ttt;
    case 1: return q->ttx;
    case 2: return q->tty;
    case 3: return q->ttn;
    case 4: return q->pl;
#ifdef PIMUNU
    case 5: return q->pitt;
    case 6: return q->pitx;
    case 7: return q->pity;
    case 8: return q->pitn;
    case 9: return q->pixx;
    case 10: return q->pixy;
    case 11: return q->pixn;
    case 12: return q->piyy;
    case 13: return q->piyn;
    case 14: return q->pinn;
#endif
#ifdef PI
    case 15: return q->Pi;
#endif
    case 16: return e;
    case 17: return p;
    case 18: return u->ut;
    case 19: return u->ux;
    case 20: return u->uy;
    case 21: return u->un;
    case 22: return up->ut;
    case 23: return up->ux;
    case 24: return up->uy;
    case 25: return up->un;
    /* inversion-failure flags of the last step (FullyDiscreteKurganovTadmorScheme.cpp:189-190) */
    case 32: return fTSol_X1;
    case 33: return fTSol_Y1;
    case 34: return fTSol_1;
    case 35: return fTSol_X2;
    case 36: return fTSol_Y2;
    case 37: return fTSol_2;
    default: return 0;
    }
}

/* The reference's own primitive -> conserved initialisation
 * (DynamicalVariables.cpp:197-287; P_L = 0.0154483 e hard-coded). */
extern "C" void vref_set_conserved(double t) { setConservedVariables(t, &g_lat); }

/* DynamicalVariables.cpp:349-356 on the current state. */
extern "C" void vref_set_ghost_cells(void) { setGhostCells(q, e, p, u, &g_lat); }

/* One time step exactly as HydroPlugin.cpp:223,230 drive it. */
extern "C" void vref_step(double t, double dt) {
    rungeKutta2(t, dt, q, Q, &g_lat, &g_hydro);
    setCurrentConservedVariables();
}

/* n steps from t0; returns wall seconds (CLOCK_MONOTONIC). */
extern "C" double vref_run(double t0, double dt, int n) {
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    for (int k = 0; k < n; ++k) {
        rungeKutta2(t0 + k * dt, dt, q, Q, &g_lat, &g_hydro);
        setCurrentConservedVariables();
    }
    clock_gettime(CLOCK_MONOTONIC, &b);
    return (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
}
