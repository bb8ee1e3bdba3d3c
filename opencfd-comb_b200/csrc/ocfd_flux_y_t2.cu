// Flow fluxes of sweep direction 1 with the alternative tile shape 2 (k_flux, Tile<1, 2>), in
// its own translation unit so that the shapes compile in parallel.
#include "ocfd_flux_launch.cuh"

namespace ocfd {
void launch_flux_y_t2(int scheme, int split, bool sep, const FluxArgs& a, int nx, int ny, int nz,
                      cudaStream_t st) {
  flux_launch::launch_tile<1, 2>(scheme, split, sep, a, nx, ny, nz, st);
}
}  // namespace ocfd
