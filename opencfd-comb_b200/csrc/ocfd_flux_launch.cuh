// Launcher of one sweep direction of k_flux, included by the three per-direction translation
// units (compiled in parallel).
#pragma once
#include <stdexcept>
#include "ocfd_flux_char.cuh"
#include "ocfd_launch.h"

namespace ocfd {
namespace flux_launch {
template <int DIR, int SCHEME, int SPLIT, bool SEP, bool SCALAR, int G>
void go(FluxArgs a, int ngroups, int nx, int ny, int nz, cudaStream_t st) {
  constexpr size_t sm = flux_smem<DIR, SCALAR, G>();
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_flux<DIR, SCHEME, SPLIT, SEP, SCALAR, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sm);
    attr = true;
  }
  auto nb = [](int n, int b) { return (unsigned)((n + b - 1) / b); };
  dim3 grid;
  if (DIR == 0) grid = dim3(nb(nx, Tile<0>::C), nb(ny, Tile<0>::NL), nz);
  else if (DIR == 1) grid = dim3(nb(nx, Tile<1>::NL), nb(ny, Tile<1>::C), nz);
  else grid = dim3(nb(nx, Tile<2>::NL), nb(nz, Tile<2>::C), ny);
  a.nbz = (int)grid.z;
  grid.z *= (unsigned)ngroups;
  k_flux<DIR, SCHEME, SPLIT, SEP, SCALAR, G><<<grid, FLUX_THREADS, sm, st>>>(a);
}
template <int DIR, int SCHEME, int SPLIT, bool SEP>
void go_char(FluxArgs a, int nx, int ny, int nz, cudaStream_t st) {
  constexpr size_t sm = CharTile<DIR>::smem;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_flux_char<DIR, SCHEME, SPLIT, SEP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  auto nb = [](int n, int b) { return (unsigned)((n + b - 1) / b); };
  dim3 grid;
  if (DIR == 0) grid = dim3(nb(nx, Tile<0>::C), nb(ny, Tile<0>::NL), nz);
  else if (DIR == 1) grid = dim3(nb(nx, Tile<1>::NL), nb(ny, Tile<1>::C), nz);
  else grid = dim3(nb(nx, Tile<2>::NL), nb(nz, Tile<2>::C), ny);
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
}  // namespace flux_launch
}  // namespace ocfd
