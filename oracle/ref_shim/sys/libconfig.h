/*
 * Minimal stand-in for libconfig's header (libconfig is not installed here).
 *
 * Test infrastructure: the reference's rhic/include/LatticeParameters.h:11
 * includes <libconfig.h> only to name config_t in a loader declaration; the
 * hot-path sources never call libconfig. Nothing here is linked into the
 * product.
 */
#ifndef VAH_REF_SHIM_LIBCONFIG_H
#define VAH_REF_SHIM_LIBCONFIG_H

typedef struct config_t {
    int unused;
} config_t;

#endif
