// Flow fluxes of sweep direction 1 with the alternative tile shape 1 (k_flux, Tile<1, 1>), in
// its own translation unit so that the shapes compile in parallel.
#include "ocfd_flux_launch.cuh"

namespace ocfd {
void launch_flux_y_t1(int scheme, int split, bool sep, const FluxArgs& a, int nx, int ny, int nz,
                      cudaStream_t st) {
  flux_launch::launch_tile<1, 1>(scheme, split, sep, a, nx, ny, nz, st);
}
}  // namespace ocfd
