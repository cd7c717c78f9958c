// vah_kernels.cuh -- kernel launch interface shared by vah_kernels.cu and vah_api.cu.
#pragma once

#include <cuda_runtime.h>

#include "vah_stage.cuh"
#include "vah_validity.cuh"

namespace vah {

// One fused RK stage over all interior cells.
template <typename S>
cudaError_t launch_stage(const StageArgs<S> &a, int physics, cudaStream_t stream);

// ---- face/cell split: launch kinds and their tunable launch configuration --
// Kinds of launch in one split stage: the face launches per axis, then the
// cell launch. Each has a block shape (bx x by = kSplitThreads threads, x
// fastest) and a register-cap variant minb: the compiler must fit minb
// resident blocks per SM, i.e. at most 65536 / (128 minb) registers per
// thread (face: 3, 4, 5 -> 168, 128, 96-102; cell: 2, 3, 4 -> 255, 168, 128).
enum SplitKind { kFaceX = 0, kFaceY = 1, kFaceZ = 2, kCell = 3, kNumSplitKinds = 4 };
constexpr int kSplitThreads = 128;

struct KindConfig {
    int bx, by, minb;
};
struct SplitConfig {
    KindConfig k[kNumSplitKinds];
};

// The autotuner's search space per kind (block shapes x register caps).
constexpr int kNumShapes = 2;
constexpr int kShapes[kNumShapes][2] = {{32, 4}, {64, 2}};
constexpr int kNumMinb = 3;
constexpr int kFaceMinb[kNumMinb] = {3, 4, 5};
constexpr int kCellMinb[kNumMinb] = {2, 3, 4};

inline bool valid_kind_config(int kind, const KindConfig &c) {
    if (kind < 0 || kind >= kNumSplitKinds || c.bx * c.by != kSplitThreads) return false;
    bool shape = false, minb = false;
    for (int s = 0; s < kNumShapes; ++s) shape |= c.bx == kShapes[s][0] && c.by == kShapes[s][1];
    for (int m = 0; m < kNumMinb; ++m) minb |= c.minb == (kind == kCell ? kCellMinb[m] : kFaceMinb[m]);
    return shape && minb;
}

// Candidates of one kind, in a fixed order; returns their number.
inline int split_candidates(int kind, KindConfig *out, int max) {
    int n = 0;
    for (int s = 0; s < kNumShapes; ++s)
        for (int m = 0; m < kNumMinb; ++m)
            if (n < max) out[n++] = {kShapes[s][0], kShapes[s][1], kind == kCell ? kCellMinb[m] : kFaceMinb[m]};
    return n;
}

// Untuned default: the best of the candidates on the 121x121x81 shear+bulk
// table-EoS event (faces capped at 128 registers, cells at 168).
inline SplitConfig default_split_config() {
    SplitConfig c;
    for (int k = 0; k < kNumSplitKinds; ++k) c.k[k] = {32, 4, k == kCell ? 3 : 4};
    return c;
}

// One launch of one split kind (a.H, and a.HR when exact, must point at the
// face buffers). exact = the reference's per-cell face evaluation.
template <typename S>
cudaError_t launch_split_kind(const StageArgs<S> &a, int physics, bool exact, int kind, const KindConfig &c,
                              cudaStream_t stream);

// One RK stage on the face/cell split: face launches (x, y[, z]) then the
// cell launch, with the given (or the default) launch configuration.
template <typename S>
cudaError_t launch_stage_split(const StageArgs<S> &a, int physics, bool exact, const SplitConfig &c,
                               cudaStream_t stream);
template <typename S>
cudaError_t launch_stage_split(const StageArgs<S> &a, int physics, bool exact, cudaStream_t stream);

// Validity diagnostics of every interior cell after a step.
template <typename S>
cudaError_t launch_validity(const ValidityArgs<S> &a, int physics, cudaStream_t stream);

// A set of device field pointers, passed to kernels by value.
template <typename S>
struct FieldSet {
    S *f[32];
    int n;
};

// The set-up launches below index cell (i, j, k) of the ghosted grid at
// i + pitch (j + (ny + 4) k): pitch = nx + 4 in the reference layout, or the
// padded pitch of the tile layout.
// Primitive -> conserved over the interior (setConservedVariables):
// q = 16 conserved slots, u/up = 4 velocity components each.
template <typename S>
cudaError_t launch_set_conserved(const FieldSet<S> &q, const FieldSet<S> &u, const FieldSet<S> &up, const S *e,
                                 int physics, int nx, int ny, int nz, int pitch, double t, int pl_from_field,
                                 cudaStream_t stream);

// Interior primitives for a fresh event: p = EoS(e), u = (1,0,0,0),
// pi = Pi = 0, P_L = p (q[4]).
template <typename S>
cudaError_t launch_init_primitives(const FieldSet<S> &q, const FieldSet<S> &u, const S *e, S *p, const Eos &eos,
                                   int nx, int ny, int nz, int pitch, cudaStream_t stream);

// Reference ghost fill, three passes with its loop ranges (setGhostCells).
template <typename S>
cudaError_t launch_ghosts(const FieldSet<S> &fields, int nx, int ny, int nz, int pitch, cudaStream_t stream);
// One pass of it (0: x, 1: y, 2: eta): on 2+1D lattices the eta pass fills the
// eta ghost layers that the steps leave to the reader.
template <typename S>
cudaError_t launch_ghost_pass(const FieldSet<S> &fields, int nx, int ny, int nz, int pitch, int pass,
                              cudaStream_t stream);

}  // namespace vah
