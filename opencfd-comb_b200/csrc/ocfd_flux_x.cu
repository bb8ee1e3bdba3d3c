// Sweep direction 0 of the inviscid flux (k_flux) in its own translation unit.
#include <stdexcept>
#include "ocfd_launch.h"

namespace ocfd {
namespace {
template <int SCHEME, int SPLIT, bool SEP, bool SCALAR>
void go(const FluxArgs& a, int nx, int ny, int nz, cudaStream_t st) {
  constexpr int DIR = 0;
  constexpr size_t sm = flux_smem<DIR, SCALAR>();
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_flux<DIR, SCHEME, SPLIT, SEP, SCALAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  auto nb = [](int n, int b) { return (unsigned)((n + b - 1) / b); };
  dim3 grid;
  if (DIR == 0) grid = dim3(nb(nx, Tile<0>::C), nb(ny, Tile<0>::NL), nz);
  else if (DIR == 1) grid = dim3(nb(nx, Tile<1>::NL), nb(ny, Tile<1>::C), nz);
  else grid = dim3(nb(nx, Tile<2>::NL), nb(nz, Tile<2>::C), ny);
  k_flux<DIR, SCHEME, SPLIT, SEP, SCALAR><<<grid, 256, sm, st>>>(a);
}
template <bool SEP, bool SCALAR>
void pick(int scheme, int split, const FluxArgs& a, int nx, int ny, int nz, cudaStream_t st) {
#define FX(S)                                                                \
  if (scheme == S) {                                                         \
    if constexpr (SCALAR) {                                                  \
      go<S, OCFD_SPLIT_SW, SEP, SCALAR>(a, nx, ny, nz, st);                  \
    } else {                                                                 \
      if (split == OCFD_SPLIT_SW) go<S, OCFD_SPLIT_SW, SEP, SCALAR>(a, nx, ny, nz, st); \
      else go<S, OCFD_SPLIT_LLF, SEP, SCALAR>(a, nx, ny, nz, st);            \
    }                                                                        \
    return;                                                                  \
  }
  FX(OCFD_SCHEME_WENO5) FX(OCFD_SCHEME_WENO7) FX(OCFD_SCHEME_OMP6) FX(OCFD_SCHEME_UD7L) FX(OCFD_SCHEME_HYBRID)
#undef FX
  throw std::runtime_error("scheme");
}
}  // namespace

void launch_flux_x(int scheme, int split, bool sep, bool scalar, const FluxArgs& a, int nx, int ny, int nz,
                   cudaStream_t st) {
  if (sep) {
    if (scalar) pick<true, true>(scheme, split, a, nx, ny, nz, st);
    else pick<true, false>(scheme, split, a, nx, ny, nz, st);
  } else {
    if (scalar) pick<false, true>(scheme, split, a, nx, ny, nz, st);
    else pick<false, false>(scheme, split, a, nx, ny, nz, st);
  }
}
}  // namespace ocfd
