// Launcher of one sweep direction of k_flux, included by the three per-direction translation
// units (compiled in parallel).
#pragma once
#include <stdexcept>
#include "ocfd_flux_char.cuh"
#include "ocfd_launch.h"

namespace ocfd {
namespace flux_launch {
template <int DIR, int TS>
dim3 tile_grid(int nx, int ny, int nz) {
  using T = Tile<DIR, TS>;
  auto nb = [](int n, int b) { return (unsigned)((n + b - 1) / b); };
  if (DIR == 0) return dim3(nb(nx, T::C), nb(ny, T::NL), nz);
  if (DIR == 1) return dim3(nb(nx, T::NL), nb(ny, T::C), nz);
  return dim3(nb(nx, T::NL), nb(nz, T::C), ny);
}
template <int DIR, int SCHEME, int SPLIT, bool SEP, bool SCALAR, int G, int TS = 0>
void go(FluxArgs a, int ngroups, int nx, int ny, int nz, cudaStream_t st) {
  constexpr size_t sm = flux_smem<DIR, SCALAR, G, TS>();
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_flux<DIR, SCHEME, SPLIT, SEP, SCALAR, G, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sm);
    attr = true;
  }
  dim3 grid = tile_grid<DIR, TS>(nx, ny, nz);
  a.nbz = (int)grid.z;
  grid.z *= (unsigned)ngroups;
  k_flux<DIR, SCHEME, SPLIT, SEP, SCALAR, G, TS><<<grid, FLUX_THREADS, sm, st>>>(a);
}
template <int DIR, int SCHEME, int SPLIT, bool SEP>
void go_char(FluxArgs a, int nx, int ny, int nz, cudaStream_t st) {
  constexpr size_t sm = CharTile<DIR>::smem;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_flux_char<DIR, SCHEME, SPLIT, SEP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  dim3 grid = tile_grid<DIR, 0>(nx, ny, nz);
  a.nbz = (int)grid.z;
  k_flux_char<DIR, SCHEME, SPLIT, SEP><<<grid, FLUX_THREADS, sm, st>>>(a);
}
template <int DIR, bool SEP>
void pick(int scheme, int split, int group, int ngroups, bool character, const FluxArgs& a, int nx, int ny, int nz,
          cudaStream_t st) {
#define FX(S)                                                                                      \
  if (scheme == S) {                                                                               \
    if (character && group == 0) {                                                                 \
      if (split == OCFD_SPLIT_SW) go_char<DIR, S, OCFD_SPLIT_SW, SEP>(a, nx, ny, nz, st);          \
      else go_char<DIR, S, OCFD_SPLIT_LLF, SEP>(a, nx, ny, nz, st);                                \
    } else if (group == 3) go<DIR, S, OCFD_SPLIT_SW, SEP, true, 3>(a, ngroups, nx, ny, nz, st);    \
    else if (group == 1) go<DIR, S, OCFD_SPLIT_SW, SEP, true, 1>(a, ngroups, nx, ny, nz, st);      \
    else if (split == OCFD_SPLIT_SW) go<DIR, S, OCFD_SPLIT_SW, SEP, false, 1>(a, 1, nx, ny, nz, st); \
    else go<DIR, S, OCFD_SPLIT_LLF, SEP, false, 1>(a, 1, nx, ny, nz, st);                         \
    return;                                                                                        \
  }
  FX(OCFD_SCHEME_WENO5) FX(OCFD_SCHEME_WENO7) FX(OCFD_SCHEME_OMP6) FX(OCFD_SCHEME_UD7L) FX(OCFD_SCHEME_HYBRID)
#undef FX
  throw std::runtime_error("scheme");
}
template <int DIR>
void launch(int scheme, int split, bool sep, int group, int ngroups, bool character, const FluxArgs& a, int nx,
            int ny, int nz, cudaStream_t st) {
  if (group != 0 && group != 1 && group != 3) throw std::runtime_error("species group");
  if (sep) pick<DIR, true>(scheme, split, group, ngroups, character, a, nx, ny, nz, st);
  else pick<DIR, false>(scheme, split, group, ngroups, character, a, nx, ny, nz, st);
}
// the flow fluxes (no species group, component-wise) with the alternative tile shape TS
template <int DIR, int TS>
void launch_tile(int scheme, int split, bool sep, const FluxArgs& a, int nx, int ny, int nz, cudaStream_t st) {
#define FT(S)                                                                                           \
  if (scheme == S) {                                                                                    \
    if (sep) {                                                                                          \
      if (split == OCFD_SPLIT_SW) go<DIR, S, OCFD_SPLIT_SW, true, false, 1, TS>(a, 1, nx, ny, nz, st);   \
      else go<DIR, S, OCFD_SPLIT_LLF, true, false, 1, TS>(a, 1, nx, ny, nz, st);                        \
    } else {                                                                                            \
      if (split == OCFD_SPLIT_SW) go<DIR, S, OCFD_SPLIT_SW, false, false, 1, TS>(a, 1, nx, ny, nz, st);  \
      else go<DIR, S, OCFD_SPLIT_LLF, false, false, 1, TS>(a, 1, nx, ny, nz, st);                       \
    }                                                                                                   \
    return;                                                                                             \
  }
  FT(OCFD_SCHEME_WENO5) FT(OCFD_SCHEME_WENO7) FT(OCFD_SCHEME_OMP6) FT(OCFD_SCHEME_UD7L) FT(OCFD_SCHEME_HYBRID)
#undef FT
  throw std::runtime_error("scheme");
}
}  // namespace flux_launch
}  // namespace ocfd
