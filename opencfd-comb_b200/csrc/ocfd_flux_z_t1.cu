// Flow fluxes of sweep direction 2 with the alternative tile shape 1 (k_flux, Tile<2, 1>), in
// its own translation unit so that the shapes compile in parallel.
#include "ocfd_flux_launch.cuh"

namespace ocfd {
void launch_flux_z_t1(int scheme, int split, bool sep, const FluxArgs& a, int nx, int ny, int nz,
                      cudaStream_t st) {
  flux_launch::launch_tile<2, 1>(scheme, split, sep, a, nx, ny, nz, st);
}
}  // namespace ocfd
