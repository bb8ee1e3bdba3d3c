// Flow fluxes of sweep direction 0 with the alternative tile shape 2 (k_flux, Tile<0, 2>), in
// its own translation unit so that the shapes compile in parallel.
#include "ocfd_flux_launch.cuh"

namespace ocfd {
void launch_flux_x_t2(int scheme, int split, bool sep, const FluxArgs& a, int nx, int ny, int nz,
                      cudaStream_t st) {
  flux_launch::launch_tile<0, 2>(scheme, split, sep, a, nx, ny, nz, st);
}
}  // namespace ocfd
