// Host-side launchers of the kernels that live in their own translation units (compiled in
// parallel): the three sweep directions of k_flux and the chemistry kernels.
#pragma once
#include <cuda_runtime.h>
#include "ocfd_flow.cuh"

namespace ocfd {
// one sweep direction; group = 0 for the flow fluxes, else the species per block of a scalar
// sweep over ngroups x group species (1 or 3); character selects the characteristic-space flow
// flux (IF_Scheme_Character = 1); throws std::runtime_error on a bad scheme id
void launch_flux_x(int scheme, int split, bool sep, int group, int ngroups, bool character, const FluxArgs& a,
                   int nx, int ny, int nz, cudaStream_t st);
void launch_flux_y(int scheme, int split, bool sep, int group, int ngroups, bool character, const FluxArgs& a,
                   int nx, int ny, int nz, cudaStream_t st);
void launch_flux_z(int scheme, int split, bool sep, int group, int ngroups, bool character, const FluxArgs& a,
                   int nx, int ny, int nz, cudaStream_t st);
// the flow fluxes of one sweep direction with the alternative tile shape 1 or 2 (Tile<DIR, TS>),
// each (direction, shape) in its own translation unit; throw on a bad scheme id
#define OCFD_FLUX_TILE_DECL(NAME)                                                                  \
  void NAME(int scheme, int split, bool sep, const FluxArgs& a, int nx, int ny, int nz, cudaStream_t st);
OCFD_FLUX_TILE_DECL(launch_flux_x_t1)
OCFD_FLUX_TILE_DECL(launch_flux_x_t2)
OCFD_FLUX_TILE_DECL(launch_flux_y_t1)
OCFD_FLUX_TILE_DECL(launch_flux_y_t2)
OCFD_FLUX_TILE_DECL(launch_flux_z_t1)
OCFD_FLUX_TILE_DECL(launch_flux_z_t2)
#undef OCFD_FLUX_TILE_DECL
void launch_chem_cells(int ns, long long ncell, double* f, double* Et, double* T, double* p, double* di, double dt2,
                       int nsub, int* nfail, cudaStream_t st);
void launch_chem_batch(int ns, int sms, int n, double* di, double* e, const double* dt, const int* nsub,
                       const int* perm, int* counter, int* nfail, cudaStream_t st);
// the compiled mechanism whose structure the constant block's mechanism has (MECH_H2AIR9), else
// MECH_GENERIC (ocfd_chem.cu)
int mech_match(const DevConst& c);
}  // namespace ocfd
