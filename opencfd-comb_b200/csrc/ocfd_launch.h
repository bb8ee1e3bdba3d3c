// Host-side launchers of the kernels that live in their own translation units (compiled in
// parallel): the three sweep directions of k_flux and the chemistry kernels.
#pragma once
#include <cuda_runtime.h>
#include "ocfd_flow.cuh"

namespace ocfd {
// one sweep direction; throws std::runtime_error on a bad scheme id
void launch_flux_x(int scheme, int split, bool sep, bool scalar, const FluxArgs& a, int nx, int ny, int nz,
                   cudaStream_t st);
void launch_flux_y(int scheme, int split, bool sep, bool scalar, const FluxArgs& a, int nx, int ny, int nz,
                   cudaStream_t st);
void launch_flux_z(int scheme, int split, bool sep, bool scalar, const FluxArgs& a, int nx, int ny, int nz,
                   cudaStream_t st);
void launch_chem_cells(int ns, long long ncell, double* f, double* Et, double* T, double* p, double* di, double dt2,
                       int nsub, int* nfail, cudaStream_t st);
void launch_chem_batch(int ns, int sms, int n, double* di, double* e, const double* dt, const int* nsub,
                       const int* perm, int* counter, int* nfail, cudaStream_t st);
}  // namespace ocfd
