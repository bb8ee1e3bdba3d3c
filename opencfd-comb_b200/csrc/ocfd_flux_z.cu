// Sweep direction 2 of the inviscid flux (k_flux) in its own translation unit.
#include "ocfd_flux_launch.cuh"

namespace ocfd {
void launch_flux_z(int scheme, int split, bool sep, int group, int ngroups, bool character, const FluxArgs& a,
                   int nx, int ny, int nz, cudaStream_t st) {
  flux_launch::launch<2>(scheme, split, sep, group, ngroups, character, a, nx, ny, nz, st);
}
}  // namespace ocfd
