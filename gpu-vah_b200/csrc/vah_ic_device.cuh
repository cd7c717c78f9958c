// vah_ic_device.cuh -- the workloads' initial energy densities generated on
// the GPU (the host generators are vah_ic.cpp; the device ones follow the same
// definitions and, for the MC-Glauber collision, the same random streams).
//
// MC-Glauber: one block samples both nuclei (a thread per nucleus walking its
// splitmix64 stream exactly as the host sampler does), flags the participants
// in parallel and compacts them in the host's order (nucleus A's, then B's);
// a grid then deposits their Gaussians per transverse cell.
// Optical Glauber: the Woods-Saxon thickness T(r) by Simpson in z on a table
// of radii (a thread per radius), its normalisation to A nucleons, then
// N_part/2 and N_coll per transverse cell.
#pragma once

#include <cuda_runtime.h>

namespace vah {

// Participants of one seeded collision into d_pxy (x, y pairs, at most 2A)
// and their number into *d_np, all on the device, on `stream`.
cudaError_t ic_participants_device(double b, double sigma_nn_fm2, int A, double ws_R, double ws_a,
                                   unsigned long long seed, double *d_pxy, int *d_np, cudaStream_t stream);

// v(x, y) = sum of exp(-r^2 / (2 w^2)) over the participants (cut at r = 8 w)
// on an nx * ny grid centred like the lattice, and its maximum (as the bit
// pattern of a non-negative double) into *maxbits (which must start at 0).
cudaError_t ic_deposit_device(const double *d_pxy, const int *d_np, double width, int nx, int ny, double dx,
                              double dy, double *d_v, unsigned long long *maxbits, cudaStream_t stream);

// Optical-Glauber profile v = (1 - x_coll) N_part/2 + x_coll N_coll on the grid,
// and its maximum into *maxbits (which must start at 0). d_tab: scratch of
// kThicknessPoints + 1 doubles.
constexpr int kThicknessPoints = 2048;
cudaError_t ic_optical_device(int nx, int ny, double dx, double dy, double b, double sigma_nn_fm2, int A,
                              double ws_R, double ws_a, double x_coll, double *d_tab, double *d_v,
                              unsigned long long *maxbits, cudaStream_t stream);

// e(x, y, eta) = e_peak v / max v * f(eta) + e_floor into the interior of a
// ghosted field (row pitch `pitch`, ny + 4 rows per plane); a flat floor when
// max v = 0. f(eta) is vah_ic_longitudinal's profile (flat for |eta| <
// eta_flat, Gaussian tails of width sigma_eta, eta centred on the lattice with
// spacing dz), 1 when nz = 1.
template <typename S>
cudaError_t ic_fill_device(const double *d_v, const unsigned long long *maxbits, int nx, int ny, int nz, int pitch,
                           double dz, double eta_flat, double sigma_eta, double e_peak, double e_floor, S *e,
                           cudaStream_t stream);

}  // namespace vah
