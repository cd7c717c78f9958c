// vah_kernels.cuh -- kernel launch interface shared by vah_kernels.cu and vah_api.cu.
#pragma once

#include <cuda_runtime.h>

#include "vah_stage.cuh"

namespace vah {

// One fused RK stage over all interior cells.
template <typename S>
cudaError_t launch_stage(const StageArgs<S> &a, int physics, cudaStream_t stream);

// One RK stage on the face/cell split: face launches (x, y[, z]) then the
// cell launch; a.H (and a.HR when exact) must point at the face buffers.
// exact = the reference's per-cell face evaluation.
template <typename S>
cudaError_t launch_stage_split(const StageArgs<S> &a, int physics, bool exact, cudaStream_t stream);

// A set of device field pointers, passed to kernels by value.
template <typename S>
struct FieldSet {
    S *f[32];
    int n;
};

// Primitive -> conserved over the interior (setConservedVariables):
// q = 16 conserved slots, u/up = 4 velocity components each.
template <typename S>
cudaError_t launch_set_conserved(const FieldSet<S> &q, const FieldSet<S> &u, const FieldSet<S> &up, const S *e,
                                 int physics, int nx, int ny, int nz, double t, int pl_from_field,
                                 cudaStream_t stream);

// Interior primitives for a fresh event: p = EoS(e), u = (1,0,0,0),
// pi = Pi = 0, P_L = p (q[4]).
template <typename S>
cudaError_t launch_init_primitives(const FieldSet<S> &q, const FieldSet<S> &u, const S *e, S *p, const Eos &eos,
                                   int nx, int ny, int nz, cudaStream_t stream);

// Reference ghost fill, three passes with its loop ranges (setGhostCells).
template <typename S>
cudaError_t launch_ghosts(const FieldSet<S> &fields, int nx, int ny, int nz, cudaStream_t stream);

}  // namespace vah
