// Flow kernels of the OpenCFD-Comb hot path on sm_100a.
//
//  k_flux        one sweep direction of du_inviscous / du_scaler_invis
//                (OCFD_inviscous.f90:47-202, OCFD_scaler_inviscous.f90:1-84): a tile of pencils is
//                split (Steger-Warming / LLF, OCFD_flux_split.f90) into shared memory once per
//                point, every interface of the tile is reconstructed once (WENO5/7, OMP6, UD7L,
//                HYBRID + boundary closures), and the flux difference is combined into du.
//  k_visc_ev     first pass of du_viscous (OCFD_viscous.f90:38-108): CD6/CD8 gradients, stresses,
//                heat flux -> Ev1/Ev2/Ev3.
//  k_visc_div    second pass (OCFD_viscous.f90:114-129): divergence of Ev into du(2..5).
//  k_rk_prims    OCFD_time_adv_RK3 + comput_flow_variables + Rescaling_di + comput_T_P.
//  k_repair_et   handle_NegativeEt replay (OCFD_handle_NegativeT.f90).
//  k_bc_*        OCFD_bc, ocfd_bc_BoundaryLayer, Flow_Ghost_Extent_2nd.
#pragma once
#include <type_traits>
#include "ocfd_device.cuh"

namespace ocfd {

// per-step error / statistics words (device)
struct DevStatus {
  int neg_count;          // cells with Et <= 0 in the current stage
  int neg_list[16];       // their interior linear indices (first 16)
  int error;              // OCFD_ERR_* raised on the device
  int nan_count;
  int newton_fail;        // Newton T(E) non-converged (chemistry and primitives)
  int chem_bad;           // chemistry: zero Gauss pivot or non-finite result (follows newton_fail)
  unsigned long long neg_total;
};

// ---------------------------------------------------------------- flux splitting at one point
template <int SPLIT>
__device__ __forceinline__ void split_point(double Et1, double p1, double c1, double d1, double u1, double v1,
                                            double w1, double A1, double A2, double A3, double* fp, double* fm) {
  if (SPLIT == OCFD_SPLIT_SW) {
    double gamma = p1 / Et1 + 1.0;
    double tmp1 = 2.0 * (gamma - 1.0);
    double tmp3 = (3.0 - gamma) / (2.0 * (gamma - 1.0));
    double ss = sqrt(A1 * A1 + A2 * A2 + A3 * A3);
    double ss1 = 1.0 / ss;
    double ak1 = A1 * ss1, ak2 = A2 * ss1, ak3 = A3 * ss1;
    double vs = A1 * u1 + A2 * v1 + A3 * w1;
    double E1 = vs, E2 = vs - c1 * ss, E3 = vs + c1 * ss;
    double E1P = (E1 + fabs(E1)) * 0.5, E2P = (E2 + fabs(E2)) * 0.5, E3P = (E3 + fabs(E3)) * 0.5;
    double E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
    double tmp0 = d1 / (2.0 * gamma);
    double uc1 = u1 - c1 * ak1, uc2 = u1 + c1 * ak1;
    double vc1 = v1 - c1 * ak2, vc2 = v1 + c1 * ak2;
    double wc1 = w1 - c1 * ak3, wc2 = w1 + c1 * ak3;
    double vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.5;
    double vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.5;
    double vv = (gamma - 1.0) * (u1 * u1 + v1 * v1 + w1 * w1);
    double W2 = tmp3 * c1 * c1;
    fp[0] = tmp0 * (tmp1 * E1P + E2P + E3P);
    fp[1] = tmp0 * (tmp1 * E1P * u1 + E2P * uc1 + E3P * uc2);
    fp[2] = tmp0 * (tmp1 * E1P * v1 + E2P * vc1 + E3P * vc2);
    fp[3] = tmp0 * (tmp1 * E1P * w1 + E2P * wc1 + E3P * wc2);
    fp[4] = tmp0 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
    fm[0] = tmp0 * (tmp1 * E1M + E2M + E3M);
    fm[1] = tmp0 * (tmp1 * E1M * u1 + E2M * uc1 + E3M * uc2);
    fm[2] = tmp0 * (tmp1 * E1M * v1 + E2M * vc1 + E3M * vc2);
    fm[3] = tmp0 * (tmp1 * E1M * w1 + E2M * wc1 + E3M * wc2);
    fm[4] = tmp0 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
  } else {
    double ss = sqrt(A1 * A1 + A2 * A2 + A3 * A3);
    double un = A1 * u1 + A2 * v1 + A3 * w1;
    double lam = fabs(un) + ss * c1;
    double E0 = Et1 + 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1);
    fp[0] = 0.5 * (d1 * un + lam * d1);
    fp[1] = 0.5 * (d1 * u1 * un + A1 * p1 + lam * d1 * u1);
    fp[2] = 0.5 * (d1 * v1 * un + A2 * p1 + lam * d1 * v1);
    fp[3] = 0.5 * (d1 * w1 * un + A3 * p1 + lam * d1 * w1);
    fp[4] = 0.5 * ((E0 + p1) * un + lam * E0);
    fm[0] = 0.5 * (d1 * un - lam * d1);
    fm[1] = 0.5 * (d1 * u1 * un + A1 * p1 - lam * d1 * u1);
    fm[2] = 0.5 * (d1 * v1 * un + A2 * p1 - lam * d1 * v1);
    fm[3] = 0.5 * (d1 * w1 * un + A3 * p1 - lam * d1 * w1);
    fm[4] = 0.5 * ((E0 + p1) * un - lam * E0);
  }
}

// Tile shapes: C cells along the sweep x NL pencils. x sweeps run along the contiguous index, so
// a tile is a long chunk of few lines; y / z sweeps put NL contiguous i-lines side by side and a
// chunk along j / k. Every shape makes the split phase (C + 8 points of NL pencils) a whole
// number of 256-thread rounds. TS = 0 is the default shape; TS = 1, 2 are the alternatives the
// tile autotuner times for the flow sweeps of a given grid (a tile shape changes which block
// computes an interface, never its arithmetic, so every shape gives bit-identical fluxes):
//   x: (C, NL) = (56, 4), (120, 2), (24, 8)        y / z: (24, 16), (24, 8), (56, 8)
// MINB is the resident-block target given to the register allocator (3 x 256 threads per SM;
// the shared memory of one tile, at most 42 KB for x and 73 KB for the y / z shapes 0 and 1,
// also fits 3 times; the 79 KB of y / z shape 2 fits twice).
constexpr int FLUX_THREADS = 256, FLUX_TILE_SHAPES = 3;
template <int DIR, int TS = 0>
struct Tile {
  static constexpr int C = DIR == 0 ? (TS == 0 ? 56 : TS == 1 ? 120 : 24) : (TS == 2 ? 56 : 24);
  static constexpr int NL = DIR == 0 ? (TS == 0 ? 4 : TS == 1 ? 2 : 8) : (TS == 0 ? 16 : 8);
  static constexpr int MINB = (DIR != 0 && TS == 2) ? 2 : 3;
};

// NC components per point: the five flow fluxes, or G species of a scalar sweep
template <int DIR, int NC_, int TS = 0>
struct FluxTile {
  static constexpr int C = Tile<DIR, TS>::C, NL = Tile<DIR, TS>::NL, P = C + 8, NC = NC_;
  // pencil pitch in shared memory: odd along x, so that the lanes of a warp that read the same
  // point of different pencils fall in different banks
  static constexpr int PS = DIR == 0 ? P + 1 : P;
  static constexpr int NCS = 2 * NC;        // (component, sign) pairs: plus components, then minus
  static constexpr int NI = (C + 1) * NL;   // interfaces of a tile
  // UD7L runs: R consecutive interfaces of one pencil per item (R divides the C + 1 interfaces)
  static constexpr int R = (C + 1) % 3 == 0 ? 3 : ((C + 1) % 5 == 0 ? 5 : (C + 1) % 11 == 0 ? 11 : 1);
  static_assert((P * NL) % FLUX_THREADS == 0, "split phase must fill whole rounds");
  static constexpr size_t smem = sizeof(double) * (size_t)(NCS * PS * NL + NCS * NI) + sizeof(int) * (2 * NI + 4);
};

struct FluxArgs {
  const double *d, *u, *v, *w, *p, *Et;  // halo arrays
  const double* fs;                      // species densities di (Ns x H) for SCALAR sweeps
  const double* Rh;                      // hybrid sensor (halo array)
  double* out;                           // du (5 x N) or Dus of every species (Ns x N)
  int nbz;                               // blocks along the third grid dimension per species group
  Geo g;
};

// interface i of a pencil of n cells lies where a boundary closure of OCFD2d_flux1/2 may apply
// to the positive or the negative flux (OCFD_inviscous.f90:209-362)
__device__ __forceinline__ bool closure_zone(int i, int n, int dir) {
  const int ka = max(-cC.Ka1, -cC.Ka2), kb = max(cC.Kb1, cC.Kb2);
  return (cC.bound[dir][0] == 1 && cC.sb[2 * dir] != -1 && i <= ka) ||
         (cC.bound[dir][1] == 1 && cC.sb[2 * dir + 1] != -1 && i >= n - kb + 1);
}

// UD7L for either sign with one code path: the negative flux reads the stencil mirrored, and
// both sums keep the reference's term order (OCFD_Schemes_1.f90 UD7L P / M)
template <int VS>
__device__ __forceinline__ double ud7l_signed(const double* v, bool plus) {
  const double* U = cC.UD7L;
  const double* w = plus ? v - 3 * VS : v + 4 * VS;
  const int s = plus ? VS : -VS;
  return U[0] * w[0] + U[1] * w[s] + U[2] * w[2 * s] + U[3] * w[3 * s] + U[4] * w[4 * s] + U[5] * w[5 * s] +
         U[6] * w[6 * s] + U[7] * w[7 * s];
}

// One sweep direction of the inviscid flux for a tile of NL pencils x C cells, in three phases:
//  1. split fluxes of the C + 8 points of every pencil into shared memory (one point per thread);
//     for HYBRID the same threads classify the tile's interfaces: those that take UD7L away from
//     a boundary closure are marked fast, the rest go to a shared-memory work list;
//  2. interface fluxes, one (component, sign, interface) item per thread: fast interfaces run
//     UD7L, then the listed ones run the general reconstruction (closures, WENO5/7, OMP6), so a
//     warp never carries the WENO branches for the lanes that need only UD7L;
//  3. flux difference (hh(i) - hh(i-1)) / d, combined into du as the reference does per sweep.
// SCALAR sweeps (du_scaler_invis, OCFD_scaler_inviscous.f90) carry G species per block: the
// split velocity is formed once per point for the group, and blockIdx.z also selects the group.
// resident-block target of the species sweeps: their tiles carry 3 species instead of 5 flow
// components, so four blocks fit in shared memory; 4 (at most 64 registers) measured 1.5 %
// faster than 3 on the 9-species jet
#ifndef OCFD_SCALAR_FLUX_MINB
#define OCFD_SCALAR_FLUX_MINB 4
#endif
template <int DIR, int SCHEME, int SPLIT, bool SEP, bool SCALAR, int G = 1, int TS = 0>
__global__ void __launch_bounds__(FLUX_THREADS, SCALAR ? OCFD_SCALAR_FLUX_MINB : Tile<DIR, TS>::MINB) k_flux(FluxArgs a) {
  using T = FluxTile<DIR, SCALAR ? G : 5, TS>;
  constexpr int C = T::C, NL = T::NL, P = T::P, PS = T::PS, NC = T::NC, NCS = T::NCS, NI = T::NI;
  constexpr bool HYB = SCHEME == OCFD_SCHEME_HYBRID;
  constexpr int VS = DIR == 0 ? 1 : NL;  // stride of consecutive sweep points in shared memory
  extern __shared__ double smem[];
  double* sf = smem;                // [NCS][PS x NL] split fluxes
  double* sh = sf + NCS * PS * NL;  // [NCS][NI] interface fluxes
  int* squeue = reinterpret_cast<int*>(sh + NCS * NI);  // listed interfaces: scm << 16 | interface
  int* sfast = squeue + NI;                             // 1 = UD7L fast path
  int* sqn = sfast + NI;                                // list length
  // point p of pencil l, interface t of pencil l
  auto sidx = [&](int cs, int p, int l) { return DIR == 0 ? (cs * NL + l) * PS + p : (cs * P + p) * NL + l; };
  auto iidx = [&](int t, int l) { return DIR == 0 ? l * (C + 1) + t : t * NL + l; };

  const int n = DIR == 0 ? cC.nx : (DIR == 1 ? cC.ny : cC.nz);
  const int s0 = (DIR == 0 ? blockIdx.x : blockIdx.y) * C + 1;  // first cell of the chunk
  const int l0 = DIR == 0 ? blockIdx.y * NL + 1 : blockIdx.x * NL + 1;
  const int grp = SCALAR ? (int)blockIdx.z / a.nbz : 0;
  const int bz = (SCALAR ? (int)blockIdx.z - grp * a.nbz : (int)blockIdx.z) + 1;
  const double* fsg = SCALAR ? a.fs + (size_t)grp * G * cC.H : nullptr;
  double* outg = SCALAR ? a.out + (size_t)grp * G * cC.N : a.out;
  const int nl_max = DIR == 0 ? cC.ny : cC.nx;
  const int ncell = min(C, n - s0 + 1);
  const int stride = hstride(DIR);
  auto coords = [&](int s, int l, int& i, int& j, int& k) {
    if (DIR == 0) { i = s; j = l0 + l; k = bz; }
    else if (DIR == 1) { i = l0 + l; j = s; k = bz; }
    else { i = l0 + l; j = bz; k = s; }
  };
  if (HYB) {
    if (threadIdx.x == 0) *sqn = 0;
    __syncthreads();
  }

  // phase 1 (uniform trip count: the warp-wide ballot below needs every lane)
  for (int base = 0; base < P * NL; base += FLUX_THREADS) {
    const int idx = base + threadIdx.x;
    int p, l;
    if (DIR == 0) { p = idx % P; l = idx / P; }
    else { l = idx % NL; p = idx / NL; }
    const int s = s0 - 4 + p;
    const bool line_ok = l0 + l <= nl_max;
    double fp[NC], fm[NC];
    if (line_ok && p < ncell + 8) {
      int i, j, k;
      coords(s, l, i, j, k);
      const int q = hidx(i, j, k);
      double A1, A2, A3;
      metric_dir<SEP>(a.g, DIR, i, j, k, q, A1, A2, A3);
      if constexpr (SCALAR) {
        double vs = A1 * __ldg(a.u + q) + A2 * __ldg(a.v + q) + A3 * __ldg(a.w + q);
#pragma unroll
        for (int c = 0; c < NC; c++) {
          double fsq = __ldg(fsg + (size_t)c * cC.H + q);
          fp[c] = 0.5 * (vs + fabs(vs)) * fsq;
          fm[c] = 0.5 * (vs - fabs(vs)) * fsq;
        }
      } else {
        double pp = __ldg(a.p + q), et = __ldg(a.Et + q), dd = __ldg(a.d + q);
        double gamma = pp / et + 1.0;
        double cc = sqrt(gamma * pp / dd);  // comput_cc
        split_point<SPLIT>(et, pp, cc, dd, __ldg(a.u + q), __ldg(a.v + q), __ldg(a.w + q), A1, A2, A3, fp, fm);
      }
    } else {
#pragma unroll
      for (int c = 0; c < NC; c++) fp[c] = fm[c] = 0.0;
    }
#pragma unroll
    for (int c = 0; c < NC; c++) {
      sf[sidx(c, p, l)] = fp[c];
      sf[sidx(NC + c, p, l)] = fm[c];
    }
    if (HYB) {
      // interface t = p - 3 lies between this point's cell and the next one
      const int t = p - 3;
      bool listed = false;
      int scm = 1;
      if (line_ok && t >= 0 && t <= ncell) {
        const int ig = s0 - 1 + t;
        int i, j, k;
        coords(ig, l, i, j, k);
        const int q = hidx(i, j, k);
        scm = hybrid_index(fmax(__ldg(a.Rh + q), __ldg(a.Rh + q + stride)));
        listed = scm != 1 || closure_zone(ig, n, DIR);
        sfast[iidx(t, l)] = listed ? 0 : 1;
      }
      const unsigned m = __ballot_sync(0xffffffffu, listed);
      if (m) {
        const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
        int pos = 0;
        if (lane == leader) pos = atomicAdd(sqn, __popc(m));
        pos = __shfl_sync(0xffffffffu, pos, leader);
        if (listed) squeue[pos + __popc(m & ((1u << lane) - 1u))] = (scm << 16) | iidx(t, l);
      }
    }
  }
  __syncthreads();

  // the y / z sweeps add into du: load this thread's phase-3 cells now, so the loads are in
  // flight during phase 2
  constexpr int R3 = (C * NL + FLUX_THREADS - 1) / FLUX_THREADS;
  const long long N = cC.N;
  double pre[R3][NC];
  if (DIR != 0) {
#pragma unroll
    for (int r = 0; r < R3; r++) {
      const int idx = threadIdx.x + r * FLUX_THREADS;
      int t, l;
      if (DIR == 0) { t = idx % C; l = idx / C; }
      else { l = idx % NL; t = idx / NL; }
      if (idx < C * NL && l0 + l <= nl_max && t < ncell) {
        int i, j, k;
        coords(s0 + t, l, i, j, k);
        const int nn = nidx(i, j, k);
#pragma unroll
        for (int c = 0; c < NC; c++) pre[r][c] = outg[(size_t)c * N + nn];
      }
    }
  }

  // phase 2: numerical fluxes at interfaces s0-1 .. s0-1+ncell
  const int nq = HYB ? *sqn : 0;
  const int nfast = NCS * NI;
  auto decode = [&](int it, int& t, int& l) {
    if (DIR == 0) { t = it % (C + 1); l = it / (C + 1); }
    else { l = it % NL; t = it / NL; }
  };
  // one (component, sign, interface) item; false when the item is not this pass's work
  auto item_flux = [&](int idx, double& h, int& dst) -> bool {
    const int cs = idx / NI, it = idx - cs * NI;
    int t, l;
    decode(it, t, l);
    if (l0 + l > nl_max || t > ncell) return false;
    if (HYB && !sfast[it]) return false;
    const double* v = sf + sidx(cs, t + 3, l);
    const bool plus = cs < NC;
    if (HYB) {
      h = ud7l_signed<VS>(v, plus);
    } else {
      const int ig = s0 - 1 + t;  // reference interface index hh(ig), between cells ig and ig+1
      h = plus ? interface_flux<SCHEME, true, VS>(v, ig, n, DIR, 0) : interface_flux<SCHEME, false, VS>(v, ig, n, DIR, 0);
    }
    dst = cs * NI + it;
    return true;
  };
  if constexpr (HYB && T::R > 1) {
    // fast interfaces: UD7L in runs of R consecutive interfaces of one pencil and (component,
    // sign). The R + 7 split fluxes of a run are loaded once at fixed offsets and the R sums are
    // independent FP64 chains; each sum keeps ud7l_signed's term order (the minus flux reads the
    // stencil mirrored). Plus items come first, so only one warp mixes the two signs.
    constexpr int R = T::R, NR = (C + 1) / R, NH = NC * NL * NR;
    const double* U = cC.UD7L;
    for (int it = threadIdx.x; it < 2 * NH; it += FLUX_THREADS) {
      const bool plus = it < NH;
      const int jt = plus ? it : it - NH;
      int c, l, r;
      if (DIR == 0) {  // lanes across pencils (odd pitch: no bank conflicts)
        const int cl = jt % (NC * NL);
        r = jt / (NC * NL); c = cl / NL; l = cl - c * NL;
      } else {         // lanes along the contiguous i-lines
        l = jt % NL;
        const int rc = jt / NL;
        r = rc % NR; c = rc / NR;
      }
      const int cs = plus ? c : NC + c, t0 = r * R;
      const double* x = sf + sidx(cs, t0, l);
      double w[R + 7];
#pragma unroll
      for (int m = 0; m < R + 7; m++) w[m] = x[m * VS];
      double h[R];
      if (plus) {
#pragma unroll
        for (int q = 0; q < R; q++)
          h[q] = U[0] * w[q] + U[1] * w[q + 1] + U[2] * w[q + 2] + U[3] * w[q + 3] + U[4] * w[q + 4] +
                 U[5] * w[q + 5] + U[6] * w[q + 6] + U[7] * w[q + 7];
      } else {
#pragma unroll
        for (int q = 0; q < R; q++)
          h[q] = U[0] * w[q + 7] + U[1] * w[q + 6] + U[2] * w[q + 5] + U[3] * w[q + 4] + U[4] * w[q + 3] +
                 U[5] * w[q + 2] + U[6] * w[q + 1] + U[7] * w[q];
      }
      const bool line_ok = l0 + l <= nl_max;
#pragma unroll
      for (int q = 0; q < R; q++) {
        const int ii = iidx(t0 + q, l);
        if (line_ok && t0 + q <= ncell && sfast[ii]) sh[cs * NI + ii] = h[q];
      }
    }
  } else if constexpr (!HYB && SCHEME == OCFD_SCHEME_WENO5) {
    // WENO5 in runs of R = 3 consecutive interfaces of one pencil and (component, sign), items
    // laid out like the UD7L runs above: the R + 4 split fluxes of a run are loaded once, and the
    // second-difference terms of the smoothness indicators, which neighbouring interfaces share,
    // are formed once per point (each the expression the single-interface form evaluates, so the
    // results are the same). A run that touches a boundary closure, or the last run of a pencil
    // when 3 does not divide its C + 1 interfaces, goes interface by interface. (Runs of 5 made
    // the 64-register species sweeps spill.)
    constexpr int R = 3, NR = (C + R) / R, NH = NC * NL * NR;
    auto run = [&](auto plus_c, int cs, int t0, int l) {
      constexpr bool PLUS = decltype(plus_c)::value;
      double* hs = sh + cs * NI;
      const int tl = min(t0 + R - 1, ncell);
      if (t0 + R - 1 > C || closure_zone(s0 - 1 + t0, n, DIR) || closure_zone(s0 - 1 + tl, n, DIR)) {
        for (int t = t0; t <= tl; t++)
          hs[iidx(t, l)] = interface_flux<SCHEME, PLUS, VS>(sf + sidx(cs, t + 3, l), s0 - 1 + t, n, DIR, 0);
        return;
      }
      // flux+: f(i0-2) .. f(i0+R+1); flux-: f(i0-1) .. f(i0+R+2), i0 the run's first left cell
      const double* x = sf + sidx(cs, t0 + (PLUS ? 1 : 2), l);
      double w[R + 4], D[R + 3];
#pragma unroll
      for (int m = 0; m < R + 4; m++) w[m] = x[m * VS];
#pragma unroll
      for (int m = 1; m < R + 3; m++) D[m] = PLUS ? w5d(w[m - 1], w[m], w[m + 1]) : w5d(w[m + 1], w[m], w[m - 1]);
#pragma unroll
      for (int q = 0; q < R; q++) {
        const double h = PLUS ? weno5P_v(w[q], w[q + 1], w[q + 2], w[q + 3], w[q + 4], D[q + 3], D[q + 2], D[q + 1])
                              : weno5M_v(w[q], w[q + 1], w[q + 2], w[q + 3], w[q + 4], D[q + 1], D[q + 2], D[q + 3]);
        if (t0 + q <= ncell) hs[iidx(t0 + q, l)] = h;
      }
    };
    for (int it = threadIdx.x; it < 2 * NH; it += FLUX_THREADS) {
      const bool plus = it < NH;
      const int jt = plus ? it : it - NH;
      int c, l, r;
      if (DIR == 0) {  // lanes across pencils (odd pitch: no bank conflicts)
        const int cl = jt % (NC * NL);
        r = jt / (NC * NL); c = cl / NL; l = cl - c * NL;
      } else {         // lanes along the contiguous i-lines
        l = jt % NL;
        const int rc = jt / NL;
        r = rc % NR; c = rc / NR;
      }
      if (l0 + l > nl_max || r * R > ncell) continue;
      if (plus) run(std::true_type{}, c, r * R, l);
      else run(std::false_type{}, NC + c, r * R, l);
    }
  } else {
    // two independent items per iteration, so that their dependent FP64 chains overlap
    for (int idx = threadIdx.x; idx < nfast; idx += 2 * FLUX_THREADS) {
      double ha = 0.0, hb = 0.0;
      int da = 0, db = 0;
      const bool oa = item_flux(idx, ha, da);
      const bool ob = idx + FLUX_THREADS < nfast && item_flux(idx + FLUX_THREADS, hb, db);
      if (oa) sh[da] = ha;
      if (ob) sh[db] = hb;
    }
  }
  if (HYB) {  // listed interfaces: general reconstruction (closures, WENO7 / WENO5)
    for (int r = threadIdx.x; r < NCS * nq; r += FLUX_THREADS) {
      const int nqd = nq > 0 ? nq : 1;
      const int cs = r / nqd;
      const int e = squeue[r - cs * nqd];
      const int it = e & 0xffff, scm = e >> 16;
      int t, l;
      decode(it, t, l);
      const double* v = sf + sidx(cs, t + 3, l);
      const int ig = s0 - 1 + t;
      sh[cs * NI + it] = cs < NC ? interface_flux<SCHEME, true, VS>(v, ig, n, DIR, scm)
                                 : interface_flux<SCHEME, false, VS>(v, ig, n, DIR, scm);
    }
  }
  __syncthreads();

  // phase 3: flux difference into du
  const double h1 = cC.h1[DIR];
#pragma unroll
  for (int r = 0; r < R3; r++) {
    const int idx = threadIdx.x + r * FLUX_THREADS;
    int t, l;
    if (DIR == 0) { t = idx % C; l = idx / C; }
    else { l = idx % NL; t = idx / NL; }
    if (idx >= C * NL || l0 + l > nl_max || t >= ncell) continue;
    int i, j, k;
    coords(s0 + t, l, i, j, k);
    const int nn = nidx(i, j, k);
    double ajac = 0.0;
    if (DIR == 2) ajac = metric_jac<SEP>(a.g, i, j, k, hidx(i, j, k));
    const int i0 = iidx(t, l), i1 = iidx(t + 1, l);
#pragma unroll
    for (int c = 0; c < NC; c++) {
      const double* hp = sh + c * NI;
      const double* hm = sh + (NC + c) * NI;
      double val = (hp[i1] - hp[i0] + hm[i1] - hm[i0]) * h1;
      double* o = outg + (size_t)c * N + nn;
      if (DIR == 0) *o = val;
      else if (DIR == 1) *o = pre[r][c] + val;
      else *o = -(pre[r][c] + val) * ajac;
    }
    if (DIR == 2 && !SCALAR && cC.if_mass_force == 1) {
      int q = hidx(i, j, k);
      double dd = a.d[q];
      double* o = a.out + nn;
      o[N] = o[N] + dd * cC.mass_force[0];
      o[2 * N] = o[2 * N] + dd * cC.mass_force[1];
      o[3 * N] = o[3 * N] + dd * cC.mass_force[2];
      o[4 * N] = o[4 * N] + dd * (a.u[q] * cC.mass_force[0] + a.v[q] * cC.mass_force[1] + a.w[q] * cC.mass_force[2]);
    }
  }
}

template <int DIR, bool SCALAR, int G = 1, int TS = 0>
constexpr size_t flux_smem() {
  return FluxTile<DIR, SCALAR ? G : 5, TS>::smem;
}

// ---------------------------------------------------------------- CD6 / CD8 derivative
// OCFD_dx0/dy0/dz0 (OCFD_dxyz_viscous.f90) at sweep index ii of n; f(m) is the value m points
// away along the direction. CD = 6 or 8 fixes the interior scheme at compile time, CD = 0 reads
// it from the constant block; every variant evaluates the same expressions.
template <int CD, class F>
__device__ __forceinline__ double cdiff_g(F f, int dir, int ii, int n) {
  const bool cd8 = CD == 8 || (CD == 0 && cC.cd8_on);
  if (!cC.iper[dir]) {
    const double h2 = cC.h2x[dir], h12 = cC.h12x[dir];
    if (ii == 1) return (-3.0 * f(0) + 4.0 * f(1) - f(2)) / h2;
    if (ii == 2) return (f(1) - f(-1)) / h2;
    if (ii == 3) return (8.0 * (f(1) - f(-1)) - (f(2) - f(-2))) / h12;
    if (ii == n) return (f(-2) - 4.0 * f(-1) + 3.0 * f(0)) / h2;
    if (ii == n - 1) return (f(1) - f(-1)) / h2;
    if (ii == n - 2) return (8.0 * (f(1) - f(-1)) - (f(2) - f(-2))) / h12;
    if (cd8 && (ii == 4 || ii == n - 3)) {
      const double* a = cC.cd6[dir];
      return a[0] * (f(3) - f(-3)) + a[1] * (f(2) - f(-2)) + a[2] * (f(1) - f(-1));
    }
  }
  if (CD == 6 || !cd8) {
    const double* a = cC.cd6[dir];
    return a[0] * (f(3) - f(-3)) + a[1] * (f(2) - f(-2)) + a[2] * (f(1) - f(-1));
  }
  if constexpr (CD != 6) {
    const double* c = cC.cd8[dir];
    return c[0] * (f(1) - f(-1)) + c[1] * (f(2) - f(-2)) + c[2] * (f(3) - f(-3)) + c[3] * (f(4) - f(-4));
  }
  return 0.0;
}
__device__ __forceinline__ double cdiff(const double* __restrict__ f, int q, int dir, int ii, int n) {
  const int s = hstride(dir);
  return cdiff_g<0>([&](int m) { return f[q + m * s]; }, dir, ii, n);
}
// true when cdiff takes its interior formula at sweep index ii of n in direction dir (periodic,
// or away from the one-sided and reduced closures of both faces)
__device__ __forceinline__ bool cdiff_interior(int dir, int ii, int n) {
  if (cC.iper[dir]) return true;
  const int e = cC.cd8_on ? 4 : 3;
  return ii > e && ii < n + 1 - e;
}
// d fx / dx, d fy / dy, d fz / dz at (i, j, k) / q with cdiff's expressions; a cell whose three
// directions are all interior (most cells) takes one straight-line path, so the 18 (CD6) or 24
// (CD8) stencil loads are issued together instead of behind each direction's closure branches
__device__ __forceinline__ void cdiff3(const double* __restrict__ fx, const double* __restrict__ fy,
                                       const double* __restrict__ fz, int q, int i, int j, int k, double& dk,
                                       double& di, double& ds) {
  if (cdiff_interior(0, i, cC.nx) && cdiff_interior(1, j, cC.ny) && cdiff_interior(2, k, cC.nz)) {
    const int sy = hstride(1), sz = hstride(2);
    if (cC.cd8_on) {
      auto c8 = [&](const double* __restrict__ f, int dir, int s) {
        const double* c = cC.cd8[dir];
        const double fm1 = __ldg(f + q - s), fp1 = __ldg(f + q + s), fm2 = __ldg(f + q - 2 * s), fp2 = __ldg(f + q + 2 * s);
        const double fm3 = __ldg(f + q - 3 * s), fp3 = __ldg(f + q + 3 * s), fm4 = __ldg(f + q - 4 * s), fp4 = __ldg(f + q + 4 * s);
        return c[0] * (fp1 - fm1) + c[1] * (fp2 - fm2) + c[2] * (fp3 - fm3) + c[3] * (fp4 - fm4);
      };
      dk = c8(fx, 0, 1); di = c8(fy, 1, sy); ds = c8(fz, 2, sz);
    } else {
      auto c6 = [&](const double* __restrict__ f, int dir, int s) {
        const double* a = cC.cd6[dir];
        const double fm1 = __ldg(f + q - s), fp1 = __ldg(f + q + s), fm2 = __ldg(f + q - 2 * s), fp2 = __ldg(f + q + 2 * s);
        const double fm3 = __ldg(f + q - 3 * s), fp3 = __ldg(f + q + 3 * s);
        return a[0] * (fp3 - fm3) + a[1] * (fp2 - fm2) + a[2] * (fp1 - fm1);
      };
      dk = c6(fx, 0, 1); di = c6(fy, 1, sy); ds = c6(fz, 2, sz);
    }
    return;
  }
  dk = cdiff(fx, q, 0, i, cC.nx);
  di = cdiff(fy, q, 1, j, cC.ny);
  ds = cdiff(fz, q, 2, k, cC.nz);
}

// interior cell of a linear thread index (32-bit arithmetic: the library rejects grids whose
// halo arrays reach 2^31 elements, and 64-bit division is emulated in software on the GPU)
// FAST: the divisions by nx and ny as multiply-high and shift (fast_div); k_transport keeps the
// hardware-emulated division, with which it measured faster (the magic-number form cost it 6-10 %
// per launch, 1.48 against 1.63 ms on 384x256x32 cells)
template <bool FAST = true>
__device__ __forceinline__ bool cell_of(long long t64, int& i, int& j, int& k) {
  if (t64 >= cC.N) return false;
  const unsigned t = (unsigned)t64, nx = (unsigned)cC.nx, ny = (unsigned)cC.ny;
  const unsigned r = FAST ? fast_div(t, nx, cC.mx, cC.sx) : t / nx;
  i = (int)(t - r * nx) + 1;
  const unsigned s = FAST ? fast_div(r, ny, cC.my, cC.sy) : r / ny;
  j = (int)(r - s * ny) + 1;
  k = (int)s + 1;
  return true;
}

// the cell of linear index t in slab order (DevConst::jt): tiles of jt rows, each plane by plane;
// consecutive threads still take consecutive i (a warp reads one row), and every cell is visited
// once, so kernels give the same values in either order
__device__ __forceinline__ bool cell_of_slab(long long t64, int& i, int& j, int& k) {
  if (t64 >= cC.N) return false;
  const unsigned t = (unsigned)t64, nx = (unsigned)cC.nx, jt = (unsigned)cC.jt;
  const unsigned tile = jt * nx * (unsigned)cC.nz, slab = jt * nx;
  const unsigned tj = fast_div(t, tile, cC.m_tile, cC.s_tile);
  const unsigned r = t - tj * tile;
  const unsigned k0 = fast_div(r, slab, cC.m_slab, cC.s_slab);
  const unsigned r2 = r - k0 * slab;
  const unsigned jj = fast_div(r2, nx, cC.mx, cC.sx);
  i = (int)(r2 - jj * nx) + 1;
  j = (int)(tj * jt + jj) + 1;
  k = (int)k0 + 1;
  return true;
}

struct ViscArgs {
  const double *d, *u, *v, *w, *T, *di;
  const double *amu, *amk;        // precomputed transport (NS > 1) or nullptr
  const double *qpx, *qpy, *qpz;  // species enthalpy fluxes (NS > 1) or nullptr
  double* ev[3][4];               // Ev1, Ev2, Ev3 (halo arrays)
  int kc;                         // k planes marched by one block (grid.z = ceil(nz / kc))
  Geo g;
};

// stresses, heat flux and Ev1..Ev3 at one cell from its twelve derivatives g[m][dir] of
// (u, v, w, T) along (xi, eta, zeta) (OCFD_viscous.f90:60-108)
template <int NS, bool SEP>
__device__ __forceinline__ void visc_point(const ViscArgs& a, int i, int j, int k, const double (&g)[4][3], double uq,
                                           double vq, double wq, double Tq) {
  const int q = hidx(i, j, k), nn = nidx(i, j, k);
  double A[9], A1[9];
  metric_all<SEP>(a.g, i, j, k, q, A, A1);
  // A: Akx Aky Akz Aix Aiy Aiz Asx Asy Asz
  double ux = g[0][0] * A[0] + g[0][1] * A[3] + g[0][2] * A[6];
  double vx = g[1][0] * A[0] + g[1][1] * A[3] + g[1][2] * A[6];
  double wx = g[2][0] * A[0] + g[2][1] * A[3] + g[2][2] * A[6];
  double Tx = g[3][0] * A[0] + g[3][1] * A[3] + g[3][2] * A[6];
  double uy = g[0][0] * A[1] + g[0][1] * A[4] + g[0][2] * A[7];
  double vy = g[1][0] * A[1] + g[1][1] * A[4] + g[1][2] * A[7];
  double wy = g[2][0] * A[1] + g[2][1] * A[4] + g[2][2] * A[7];
  double Ty = g[3][0] * A[1] + g[3][1] * A[4] + g[3][2] * A[7];
  double uz = g[0][0] * A[2] + g[0][1] * A[5] + g[0][2] * A[8];
  double vz = g[1][0] * A[2] + g[1][1] * A[5] + g[1][2] * A[8];
  double wz = g[2][0] * A[2] + g[2][1] * A[5] + g[2][2] * A[8];
  double Tz = g[3][0] * A[2] + g[3][1] * A[5] + g[3][2] * A[8];
  double div = ux + vy + wz;
  double amu1, amuk;
  if constexpr (NS > 1) {  // from k_transport
    amu1 = a.amu[nn];
    amuk = a.amk[nn];
  } else {  // comput_Amu_Amk_AMD inline (Comput_flow_variables.f90:69-98)
    double d0[NS], Xi[NS], X0 = 0.0;
#pragma unroll
    for (int m = 0; m < NS; m++) {
      d0[m] = a.di[(size_t)m * cC.H + q];
      Xi[m] = d0[m] / cC.Mi[m];
      X0 = X0 + Xi[m];
    }
#pragma unroll
    for (int m = 0; m < NS; m++) Xi[m] = Xi[m] / X0;
    amu1 = dev_viscosity<NS>(Tq, Xi);
    double cp = dev_Cp<NS>(a.d[q], d0, Tq);
    amuk = dev_conductivity<NS>(amu1, cp, Tq, Xi);
  }
  const double tmp2_3 = 2.0 / 3.0;
  double s11 = (2.0 * ux - tmp2_3 * div) * amu1;
  double s22 = (2.0 * vy - tmp2_3 * div) * amu1;
  double s33 = (2.0 * wz - tmp2_3 * div) * amu1;
  double s12 = (uy + vx) * amu1, s13 = (uz + wx) * amu1, s23 = (vz + wy) * amu1;
  double qx = 0.0, qy = 0.0, qz = 0.0;
  if constexpr (NS > 1) { qx = a.qpx[nn]; qy = a.qpy[nn]; qz = a.qpz[nn]; }
  double E1 = uq * s11 + vq * s12 + wq * s13 + amuk * Tx + qx;
  double E2 = uq * s12 + vq * s22 + wq * s23 + amuk * Ty + qy;
  double E3 = uq * s13 + vq * s23 + wq * s33 + amuk * Tz + qz;
#pragma unroll
  for (int dd = 0; dd < 3; dd++) {
    double B1 = A1[3 * dd], B2 = A1[3 * dd + 1], B3 = A1[3 * dd + 2];
    a.ev[dd][0][q] = B1 * s11 + B2 * s12 + B3 * s13;
    a.ev[dd][1][q] = B1 * s12 + B2 * s22 + B3 * s23;
    a.ev[dd][2][q] = B1 * s13 + B2 * s23 + B3 * s33;
    a.ev[dd][3][q] = B1 * E1 + B2 * E2 + B3 * E3;
  }
}

// asynchronous 8-byte global -> shared copies (cp.async, completed per thread by commit/wait
// groups); an invalid source fills the destination with zeros and reads nothing
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// k_visc_ev as a 2.5-D stencil: a VE_TX x VE_TY tile of (i, j) columns marches along a chunk of
// kc planes in k (VE_KC by default; the tile autotuner times the VE_KC_CHOICES). The x / y
// neighbours of (u, v, w, T) come from a shared-memory copy of the current plane with an
// HZ-point halo, the z neighbours from a ring of the tile's own columns, so each value is read
// from global memory about (kc + 2 HZ) / kc times per sweep instead of once per stencil use.
// The copies of plane k+1 (and ring plane k+HZ+1) are in flight while plane k is computed: the
// halo plane is double-buffered and the ring has 2 HZ + 2 slots. HZ = 3 for CD6, 4 for CD8.
#ifndef OCFD_VE_MINB
#define OCFD_VE_MINB 2  // resident blocks per SM given to the register allocator
#endif
constexpr int VE_TX = 32, VE_TY = 8, VE_KC = 16, VE_THREADS = VE_TX * VE_TY;
constexpr int VE_KC_CHOICES[4] = {8, 16, 32, 64};
template <int HZ>
struct VeTile {
  static constexpr int W = VE_TX + 2 * HZ, HH = VE_TY + 2 * HZ, PL = W * HH;  // halo plane
  static constexpr int RS = 2 * HZ + 2;                                         // ring slots
  static constexpr size_t smem = sizeof(double) * (size_t)(2 * 4 * PL + RS * 4 * VE_THREADS);
};

template <int NS, bool SEP, int HZ>
__global__ void __launch_bounds__(VE_THREADS, OCFD_VE_MINB) k_visc_ev(ViscArgs a) {
  using TT = VeTile<HZ>;
  constexpr int W = TT::W, PL = TT::PL, RS = TT::RS, CD = HZ == 3 ? 6 : 8;
  extern __shared__ double smem[];
  double* pl = smem;                 // [2][4][HH][W]: u, v, w, T of planes k, k+1 with the halo
  double* ring = smem + 2 * 4 * PL;  // [RS][4][VE_THREADS]: planes k-HZ .. k+HZ+1, own columns
  const int tid = threadIdx.x, tx = tid % VE_TX, ty = tid / VE_TX;
  const int i0 = blockIdx.x * VE_TX + 1, j0 = blockIdx.y * VE_TY + 1, k0 = blockIdx.z * a.kc + 1;
  const int i = i0 + tx, j = j0 + ty;
  const int k1 = min(k0 + a.kc - 1, cC.nz);
  const int imax = cC.nx + OCFD_L, jmax = cC.ny + OCFD_L;  // last index of the halo arrays
  const bool in_array = i <= imax && j <= jmax;
  const bool active = i <= cC.nx && j <= cC.ny;
  const double* fl[4] = {a.u, a.v, a.w, a.T};
  auto ring_issue = [&](int kk) {  // kk >= 1 - HZ
    double* r = ring + ((kk + 4 * RS) % RS) * 4 * VE_THREADS + tid;
    const int q = in_array ? hidx(i, j, kk) : 0;
#pragma unroll
    for (int f = 0; f < 4; f++) cp_async8(r + f * VE_THREADS, fl[f] + q, in_array);
  };
  auto plane_issue = [&](int k, int b) {
    double* dst = pl + b * 4 * PL;
#pragma unroll
    for (int it = 0; it < (PL + VE_THREADS - 1) / VE_THREADS; it++) {
      const int r = tid + it * VE_THREADS;
      if (r < PL) {
        const int yy = r / W, xx = r - yy * W;
        const int ii = i0 - HZ + xx, jj = j0 - HZ + yy;
        const bool ok = ii <= imax && jj <= jmax;
        const int q = ok ? hidx(ii, jj, k) : 0;
#pragma unroll
        for (int f = 0; f < 4; f++) cp_async8(dst + f * PL + r, fl[f] + q, ok);
      }
    }
  };
  for (int kk = k0 - HZ; kk <= k0 + HZ; kk++) ring_issue(kk);
  plane_issue(k0, 0);
  cp_async_commit();

  for (int k = k0; k <= k1; k++) {
    const int b = (k - k0) & 1;
    if (k < k1) {  // prefetch the next plane
      ring_issue(k + HZ + 1);
      plane_issue(k + 1, b ^ 1);
    }
    cp_async_commit();
    cp_async_wait<1>();  // everything but the prefetch has landed
    __syncthreads();
    if (active) {
      int sl[2 * HZ + 1];  // ring slot of plane k + m at sl[m + HZ]
      {
        int c = (k - HZ + 4 * RS) % RS;
#pragma unroll
        for (int m = 0; m <= 2 * HZ; m++) {
          sl[m] = c;
          c = c + 1 == RS ? 0 : c + 1;
        }
      }
      const double* cur = pl + b * 4 * PL;
      double g[4][3];
#pragma unroll
      for (int f = 0; f < 4; f++) {
        const double* row = cur + f * PL + (ty + HZ) * W + tx + HZ;
        g[f][0] = cdiff_g<CD>([&](int m) { return row[m]; }, 0, i, cC.nx);
        g[f][1] = cdiff_g<CD>([&](int m) { return row[m * W]; }, 1, j, cC.ny);
        g[f][2] = cdiff_g<CD>([&](int m) { return ring[(sl[m + HZ] * 4 + f) * VE_THREADS + tid]; }, 2, k, cC.nz);
      }
      const double* c0 = cur + (ty + HZ) * W + tx + HZ;
      visc_point<NS, SEP>(a, i, j, k, g, c0[0], c0[PL], c0[2 * PL], c0[3 * PL]);
    }
    __syncthreads();  // plane buffer b and ring slot k-HZ are refilled next
  }
}

struct DivArgs {
  const double* ev[12];  // Ev1 (4), Ev2 (4), Ev3 (4) halo arrays, periodic halos exchanged
  double* du;
  int kc;                // k planes marched by one block
  Geo g;
};

// k_visc_div on the same marching tiles as k_visc_ev: Ev1 is differentiated along x from a
// plane copy with an x halo, Ev2 along y from a plane copy with a y halo, Ev3 along z from a
// ring of the tile's columns (double-buffered planes, 2 HZ + 2 ring slots, next plane in flight);
// du(2..5) += (dEv1/dxi + dEv2/deta + dEv3/dzeta) * Jac (OCFD_viscous.f90:114-129).
template <int HZ>
struct VdTile {
  static constexpr int W = VE_TX + 2 * HZ, HH = VE_TY + 2 * HZ;
  static constexpr int PX = VE_TY * W, PY = HH * VE_TX, RS = 2 * HZ + 2;
  static constexpr size_t smem = sizeof(double) * (size_t)(2 * 4 * (PX + PY) + RS * 4 * VE_THREADS);
};

template <bool SEP, int HZ>
__global__ void __launch_bounds__(VE_THREADS, 2) k_visc_div(DivArgs a) {
  using TT = VdTile<HZ>;
  constexpr int W = TT::W, PX = TT::PX, PY = TT::PY, RS = TT::RS, CD = HZ == 3 ? 6 : 8;
  extern __shared__ double smem[];
  double* pb = smem;                        // [2][ [4][VE_TY][W] Ev1 | [4][HH][VE_TX] Ev2 ]
  double* ring = smem + 2 * 4 * (PX + PY);  // [RS][4][VE_THREADS]: Ev3 of planes k-HZ .. k+HZ+1
  const int tid = threadIdx.x, tx = tid % VE_TX, ty = tid / VE_TX;
  const int i0 = blockIdx.x * VE_TX + 1, j0 = blockIdx.y * VE_TY + 1, k0 = blockIdx.z * a.kc + 1;
  const int i = i0 + tx, j = j0 + ty;
  const int k1 = min(k0 + a.kc - 1, cC.nz);
  const int imax = cC.nx + OCFD_L, jmax = cC.ny + OCFD_L;
  const bool in_array = i <= imax && j <= jmax;
  const bool active = i <= cC.nx && j <= cC.ny;
  auto ring_issue = [&](int kk) {
    double* r = ring + ((kk + 4 * RS) % RS) * 4 * VE_THREADS + tid;
    const int q = in_array ? hidx(i, j, kk) : 0;
#pragma unroll
    for (int m = 0; m < 4; m++) cp_async8(r + m * VE_THREADS, a.ev[8 + m] + q, in_array);
  };
  auto plane_issue = [&](int k, int b) {
    double* px = pb + b * 4 * (PX + PY);
    double* py = px + 4 * PX;
#pragma unroll
    for (int it = 0; it < (PX + VE_THREADS - 1) / VE_THREADS; it++) {
      const int r = tid + it * VE_THREADS;
      if (r < PX) {
        const int yy = r / W, xx = r - yy * W;
        const int ii = i0 - HZ + xx, jj = j0 + yy;
        const bool ok = ii <= imax && jj <= jmax;
        const int q = ok ? hidx(ii, jj, k) : 0;
#pragma unroll
        for (int m = 0; m < 4; m++) cp_async8(px + m * PX + r, a.ev[m] + q, ok);
      }
    }
#pragma unroll
    for (int it = 0; it < (PY + VE_THREADS - 1) / VE_THREADS; it++) {
      const int r = tid + it * VE_THREADS;
      if (r < PY) {
        const int yy = r / VE_TX, xx = r - yy * VE_TX;
        const int ii = i0 + xx, jj = j0 - HZ + yy;
        const bool ok = ii <= imax && jj <= jmax;
        const int q = ok ? hidx(ii, jj, k) : 0;
#pragma unroll
        for (int m = 0; m < 4; m++) cp_async8(py + m * PY + r, a.ev[4 + m] + q, ok);
      }
    }
  };
  for (int kk = k0 - HZ; kk <= k0 + HZ; kk++) ring_issue(kk);
  plane_issue(k0, 0);
  cp_async_commit();

  const long long N = cC.N;
  // du(2..5) of the current and the next plane in registers: the next plane's loads are in
  // flight while the current one is computed
  double duc[4], dun[4];
  if (active) {
    const int nn = nidx(i, j, k0);
#pragma unroll
    for (int m = 0; m < 4; m++) duc[m] = a.du[(size_t)(m + 1) * N + nn];
  }
  for (int k = k0; k <= k1; k++) {
    const int b = (k - k0) & 1;
    if (k < k1) {
      ring_issue(k + HZ + 1);
      plane_issue(k + 1, b ^ 1);
      if (active) {
        const int nn = nidx(i, j, k + 1);
#pragma unroll
        for (int m = 0; m < 4; m++) dun[m] = a.du[(size_t)(m + 1) * N + nn];
      }
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    if (active) {
      int sl[2 * HZ + 1];
      {
        int c = (k - HZ + 4 * RS) % RS;
#pragma unroll
        for (int m = 0; m <= 2 * HZ; m++) {
          sl[m] = c;
          c = c + 1 == RS ? 0 : c + 1;
        }
      }
      const double* px = pb + b * 4 * (PX + PY);
      const double* py = px + 4 * PX;
      const double ajac = metric_jac<SEP>(a.g, i, j, k, hidx(i, j, k));
      const int nn = nidx(i, j, k);
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const double* rx = px + m * PX + ty * W + tx + HZ;
        const double* ry = py + m * PY + (ty + HZ) * VE_TX + tx;
        double uk = cdiff_g<CD>([&](int o) { return rx[o]; }, 0, i, cC.nx);
        double ui = cdiff_g<CD>([&](int o) { return ry[o * VE_TX]; }, 1, j, cC.ny);
        double us = cdiff_g<CD>([&](int o) { return ring[(sl[o + HZ] * 4 + m) * VE_THREADS + tid]; }, 2, k, cC.nz);
        a.du[(size_t)(m + 1) * N + nn] = duc[m] + (uk + ui + us) * ajac;
      }
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 4; m++) duc[m] = dun[m];
  }
}

// resident-block target of the per-cell k_visc_div: it waits on its stencil loads, so a fifth
// block per SM (48 registers, about 20 bytes spilled to L1) measured 4 % faster than four (55
// registers); six (40 registers, 50 bytes spilled) gained nothing
#ifndef OCFD_VDIV_MINB
#define OCFD_VDIV_MINB 5
#endif
// per-cell form of k_visc_div (the autotuner's k chunk 0): one thread per cell, every stencil
// value read through the read-only cache; the same expressions as the marching form
template <bool SEP, int HZ>
__global__ void __launch_bounds__(256, OCFD_VDIV_MINB) k_visc_div_pc(DivArgs a) {
  constexpr int CD = HZ == 3 ? 6 : 8;
  int i, j, k;
  if (!cell_of_slab((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const int q = hidx(i, j, k), nn = nidx(i, j, k);
  const int sy = hstride(1), sz = hstride(2);
  const long long N = cC.N;
  double duc[4];
#pragma unroll
  for (int m = 0; m < 4; m++) duc[m] = a.du[(size_t)(m + 1) * N + nn];
  const double ajac = metric_jac<SEP>(a.g, i, j, k, q);
  // an interior cell (most cells) takes cdiff3's straight-line path: each component's 18 (CD6) or
  // 24 (CD8) stencil loads are issued together; the closures of the end planes go per direction
  const bool inner = cdiff_interior(0, i, cC.nx) && cdiff_interior(1, j, cC.ny) && cdiff_interior(2, k, cC.nz);
#pragma unroll
  for (int m = 0; m < 4; m++) {
    double uk, ui, us;
    if (inner) {
      cdiff3(a.ev[m], a.ev[4 + m], a.ev[8 + m], q, i, j, k, uk, ui, us);
    } else {
      const double* e1 = a.ev[m] + q;
      const double* e2 = a.ev[4 + m] + q;
      const double* e3 = a.ev[8 + m] + q;
      uk = cdiff_g<CD>([&](int o) { return __ldg(e1 + o); }, 0, i, cC.nx);
      ui = cdiff_g<CD>([&](int o) { return __ldg(e2 + o * sy); }, 1, j, cC.ny);
      us = cdiff_g<CD>([&](int o) { return __ldg(e3 + o * sz); }, 2, k, cC.nz);
    }
    a.du[(size_t)(m + 1) * N + nn] = duc[m] + (uk + ui + us) * ajac;
  }
}

// ---------------------------------------------------------------- species: viscous part
// du_scaler_viscous (OCFD_scaler_viscous.f90:4-79) for every species of a stage at once. The
// reference loops over species, each pass using du(:,:,:,1) and Ev1 as scratch; no species reads
// another's result within a stage except the enthalpy-flux sums Qp, which are accumulated here in
// the reference's species order, so the batched form computes the same numbers.
// ci = fs / d over the full halo range first (blockIdx.y = species)
static __global__ void k_ci(const double* di, const double* d, double* ci, long long H) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t o = (size_t)blockIdx.y * H;
  if (t < H) ci[o + t] = di[o + t] / d[t];
}
// One thread per (cell, species): a block is 32 consecutive cells (threadIdx.x) x NS species
// (threadIdx.y), so every species' loads are coalesced and the NS stencil evaluations of a cell
// run in parallel. The enthalpy-flux sums Qp go through shared memory and are added by the
// species-0 thread in species order.
// resident blocks per SM given to the register allocator of the (cell, species) kernels: 3 (at
// most 75 registers at 9 species) instead of the 90-94 the compiler picks alone, which allowed
// only two 288-thread blocks; measured on the 9-species jet: species work 424 -> 294 ms per step.
// k_scal_ev at 4 (56 registers, 120-280 bytes spilled) made the jet step 2 % slower
#ifndef OCFD_SPECIES_MINB
#define OCFD_SPECIES_MINB 3
#endif
template <int NS, bool SEP>
__global__ void __launch_bounds__(32 * NS, OCFD_SPECIES_MINB) k_scal_ev(const double* ci, const double* d, const double* T,
                                                     const double* amd, double* qpx, double* qpy, double* qpz,
                                                     double* e1, double* e2, double* e3, Geo g) {
  __shared__ double sq[3][NS][32];
  const int ks = threadIdx.y, lane = threadIdx.x;
  int i, j, k;
  const bool ok = cell_of_slab((long long)blockIdx.x * 32 + lane, i, j, k);
  int nn = 0;
  if (ok) {
    const int q = hidx(i, j, k);
    nn = nidx(i, j, k);
    const long long H = cC.H, N = cC.N;
    // every species' thread evaluates its cell's metrics (the same values): the FP64 pipe has room
    // for the repeated work, and the block does not wait for one warp at a barrier
    double A[9], A1[9];
    metric_all<SEP>(g, i, j, k, q, A, A1);
    const double* c = ci + (size_t)ks * H;
    double uk, ui, us;
    cdiff3(c, c, c, q, i, j, k, uk, ui, us);
    double hi = dev_hi(ks, T[q]);
    double cix = uk * A[0] + ui * A[3] + us * A[6];
    double ciy = uk * A[1] + ui * A[4] + us * A[7];
    double ciz = uk * A[2] + ui * A[5] + us * A[8];
    double dD = d[q] * amd[(size_t)ks * N + nn];
    double E1 = dD * cix, E2 = dD * ciy, E3 = dD * ciz;
    sq[0][ks][lane] = E1 * hi;
    sq[1][ks][lane] = E2 * hi;
    sq[2][ks][lane] = E3 * hi;
    const size_t o = (size_t)ks * H + q;
    e1[o] = E1 * A1[0] + E2 * A1[1] + E3 * A1[2];
    e2[o] = E1 * A1[3] + E2 * A1[4] + E3 * A1[5];
    e3[o] = E1 * A1[6] + E2 * A1[7] + E3 * A1[8];
  }
  __syncthreads();
  if (ok && ks == 0) {
    // Qp = 0 before the first species, then Qp = Qp + flux * h_k
    double qx = 0.0 + sq[0][0][lane], qy = 0.0 + sq[1][0][lane], qz = 0.0 + sq[2][0][lane];
#pragma unroll
    for (int m = 1; m < NS; m++) {
      qx = qx + sq[0][m][lane];
      qy = qy + sq[1][m][lane];
      qz = qz + sq[2][m][lane];
    }
    qpx[nn] = qx;
    qpy[nn] = qy;
    qpz[nn] = qz;
  }
}
// resident-block target of k_scal_div: its threads wait on strided stencil loads, so 7 blocks of
// 9 species (32 registers, about 150 bytes spilled to L1; 63 of 64 warps) measured 18 % faster
// than the 5 blocks that 40 registers allow
#ifndef OCFD_SCAL_DIV_MINB
#define OCFD_SCAL_DIV_MINB 7
#endif
// RK: the species RK update (k_scal_rk's expressions on the finished Dus value, which then stays in
// a register instead of making a round trip through HBM; nothing else reads Dus afterwards)
template <int NS, bool SEP, bool RK = false>
__global__ void __launch_bounds__(32 * NS, OCFD_SCAL_DIV_MINB) k_scal_div(const double* e1, const double* e2,
                                                                          const double* e3, double* dus, Geo g,
                                                                          int krk = 0, double dt = 0.0,
                                                                          const double* din = nullptr,
                                                                          double* di = nullptr) {
  const int ks = threadIdx.y;
  int i, j, k;
  const bool ok = cell_of_slab((long long)blockIdx.x * 32 + threadIdx.x, i, j, k);
  if (!ok) return;
  const int q = hidx(i, j, k), nn = nidx(i, j, k);
  const double jac = metric_jac<SEP>(g, i, j, k, q);  // every species' thread (no barrier)
  const size_t o = (size_t)ks * cC.H;
  double uk, ui, us;
  cdiff3(e1 + o, e2 + o, e3 + o, q, i, j, k, uk, ui, us);
  double* du = dus + (size_t)ks * cC.N + nn;
  const double d1 = *du + (uk + ui + us) * jac;
  if constexpr (RK) {  // Scalar_time_adv_RK3 (OCFD_Time_Adv.f90:134-166)
    const double ra[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0}, rb[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
    const size_t oh = o + q, on = (size_t)ks * cC.N + nn;
    if (krk == 1) di[oh] = din[on] + dt * d1;
    else di[oh] = ra[krk - 1] * din[on] + rb[krk - 1] * (di[oh] + dt * d1);
  } else {
    *du = d1;
  }
}
// Scalar_time_adv_RK3 (OCFD_Time_Adv.f90:134-166), blockIdx.y = species
static __global__ void k_scal_rk(int krk, double dt, const double* dus, const double* din, double* di) {
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const size_t oh = (size_t)blockIdx.y * cC.H, on = (size_t)blockIdx.y * cC.N;
  const int q = hidx(i, j, k), nn = nidx(i, j, k);
  const double ra[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0}, rb[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
  if (krk == 1) di[oh + q] = din[on + nn] + dt * dus[on + nn];
  else di[oh + q] = ra[krk - 1] * din[on + nn] + rb[krk - 1] * (di[oh + q] + dt * dus[on + nn]);
}

// comput_Amu_Amk_AMD for NS > 1 (Comput_flow_variables.f90:69-98; comput_vis_coeff,
// comput_thermal_conductivity, comput_diffusion_coeff of TRANSPORT_modules.f90:259-426).
// One thread per (cell, species): a block is 32 consecutive cells (threadIdx.x) x NS species
// (threadIdx.y). The per-species exponentials, the Wilke rows and the NS (NS-1) / 2 distinct
// binary-diffusion pairs are spread over a cell's NS threads; every sum is taken from shared
// memory in the reference's order. The divisions and square roots of the pair terms are
// restated as products (square roots of the viscosities per species, reciprocal pair constants
// from the host, 1 / D2 as exp(-poly) * 1e4, 1 / kappa_k formed by species k's thread): the same
// quantities up to last-place rounding, which the transcendental functions of this path already
// make inexact against the oracle. ln T is formed once per cell; the species pairs come from a
// table.
// k_transport runs one block more than k_scal_ev: at 4 blocks of 9 species it needs 56 registers
// and spills only 32 bytes (k_scal_ev would spill 120-280), measured 504 -> 495.5 ms per jet step
#ifndef OCFD_TRANSPORT_MINB
#define OCFD_TRANSPORT_MINB 4
#endif
template <int NS>
__global__ void __launch_bounds__(32 * NS, OCFD_TRANSPORT_MINB) k_transport(const double* d, const double* T, const double* p,
                                                       const double* di, double* amu, double* amk, double* amd) {
  constexpr int NP = NS * (NS - 1) / 2;
  __shared__ double sX[NS][32], sD0[NS][32], sMu[NS][32], sK[NS][32], sW[NS][32], sD2[NP > 0 ? NP : 1][32];
  __shared__ double sSq[NS][32], sRs[NS][32];  // sqrt(mu_k), 1 / sqrt(mu_k)
  __shared__ double sKr[NS][32], sL[32];       // 1 / kappa_k; ln T of the cell (formed once)
  const int ks = threadIdx.y, lane = threadIdx.x;
  int i, j, k;
  const bool ok = cell_of<false>((long long)blockIdx.x * 32 + lane, i, j, k);
  const int q = ok ? hidx(i, j, k) : 0, nn = ok ? nidx(i, j, k) : 0;
  const double Tq = ok ? T[q] : 300.0;
  if (ok) {
    const double d0 = di[(size_t)ks * cC.H + q];
    sD0[ks][lane] = d0;
#if OCFD_FMA_BUILD
    sX[ks][lane] = d0 * cC.rMi[ks];  // d0 / Mi up to rounding
#else
    sX[ks][lane] = d0 / cC.Mi[ks];
#endif
  }
  if (ks == NS - 1) sL[lane] = log(Tq);
  __syncthreads();
  {
    double X0 = 0.0;
#pragma unroll
    for (int m = 0; m < NS; m++) X0 = X0 + sX[m][lane];
    sW[ks][lane] = sX[ks][lane] / X0;  // mole fraction of species ks
  }
  __syncthreads();
  double Xi[NS];
#pragma unroll
  for (int m = 0; m < NS; m++) Xi[m] = sW[m][lane];
  const double L = sL[lane];
  if (cC.flag_vis != 0) {
    const double muk = exp(cC.mu_an[ks][0] + cC.mu_an[ks][1] * L + cC.mu_an[ks][2] * q2(L) + cC.mu_an[ks][3] * q3(L)) * 0.1;
    sMu[ks][lane] = muk;
    const double sq = sqrt(muk);
    sSq[ks][lane] = sq;
    sRs[ks][lane] = 1.0 / sq;
  }
  if (cC.flag_cond != 0) {
    const double kk = exp(cC.k_an[ks][0] + cC.k_an[ks][1] * L + cC.k_an[ks][2] * q2(L) + cC.k_an[ks][3] * q3(L)) * 1.0e-5;
    sK[ks][lane] = kk;
    sKr[ks][lane] = 1.0 / kk;  // the species' own thread forms the reciprocal for the harmonic sum
  }
  if (cC.flag_diff != 0) {
    for (int pi = ks; pi < NP; pi += NS) {  // pair pi = (a, b), a < b, enumerated a-major
      const int a = cC.pair_a[pi], b = cC.pair_b[pi];
      // 1 / D2 of the pair: exp(-poly) * 1e4 (the reciprocal of exp(poly) * 1e-4 up to rounding)
      sD2[pi][lane] =
          exp(-(cC.d_an[a][b][0] + cC.d_an[a][b][1] * L + cC.d_an[a][b][2] * q2(L) + cC.d_an[a][b][3] * q3(L))) * 1.0e4;
    }
  }
  __syncthreads();
  // viscosity: Wilke row ks (or Sutherland)
  double mu;
  if (cC.flag_vis == 0) {
    const double TA = 288.15, TC = 110.4;
    mu = cC.amu0 * sqrt(q3(Tq / TA)) * (TA + TC) / (TC + Tq);
  } else {
    // Wilke's phi_kj = (1 + sqrt(mu_k / mu_j) (M_j / M_k)^(1/4))^2 / sqrt(8 (1 + M_k / M_j)), with
    // the square roots of the viscosities taken once per species and the pair constants'
    // reciprocals precomputed (the same quantities up to rounding; TRANSPORT_modules.f90:259-300)
    const double muk = sMu[ks][lane], sqk = sSq[ks][lane];
    double pk0 = 0.0;
#pragma unroll
    for (int jj = 0; jj < NS; jj++) {
      double s1 = 1.0 + sqk * sRs[jj][lane] * cC.wk_c[ks][jj];
      double pkj = q2(s1) * cC.wk_binv[ks][jj];
      pk0 = pk0 + Xi[jj] * pkj;
    }
    sW[ks][lane] = Xi[ks] * muk / pk0;
    __syncthreads();
    mu = 0.0;
#pragma unroll
    for (int m = 0; m < NS; m++) mu = mu + sW[m][lane];
  }
  if (!ok) return;
  if (ks == 0) {
    double cp;
    {
      double dd[NS];
#pragma unroll
      for (int m = 0; m < NS; m++) dd[m] = sD0[m][lane];
      cp = dev_Cp<NS>(d[q], dd, Tq);
    }
    double kk;
    if (cC.flag_cond == 0) {
      kk = mu * cp / cC.pr;
    } else {
      double a1 = 0.0, a2 = 0.0;
#pragma unroll
      for (int m = 0; m < NS; m++) {
        a1 = a1 + Xi[m] * sK[m][lane];
        a2 = a2 + Xi[m] * sKr[m][lane];  // X_m / kappa_m as X_m (1 / kappa_m): the same up to the last place
      }
      kk = 0.5 * (a1 + 1.0 / a2);
    }
    amu[nn] = mu;
    amk[nn] = kk;
  }
  double ad;
  if (cC.flag_diff == 0) {
    double d0 = 0.0;
#pragma unroll
    for (int m = 0; m < NS; m++) d0 = d0 + Xi[m] * cC.Mi[m];
    ad = mu * (1.0 - Xi[ks] * cC.Mi[ks] / d0) / ((1.0 - Xi[ks]) * cC.sc * d[q] + 1.0e-20);
  } else {
    double ds = 0.0;
#pragma unroll
    for (int jj = 0; jj < NS; jj++) {
      if (jj == ks) continue;
      ds = ds + Xi[jj] * sD2[cC.pair_of[ks][jj]][lane];  // sD2 holds 1 / D2
    }
#if OCFD_FMA_BUILD
    ad = (1.0 - Xi[ks]) * 1.013e5 / ((ds + 1.0e-20) * p[q]);  // one division; the same up to rounding
#else
    ad = (1.0 - Xi[ks]) / (ds + 1.0e-20) * 1.013e5 / p[q];
#endif
  }
  amd[(size_t)ks * cC.N + nn] = ad;
}

// ---------------------------------------------------------------- halo exchange (single rank)
// exchange_boundary_x/y/z (OCFD_mpi.f90:201-236): in a periodic direction the LAP face planes
// wrap around; a non-periodic face halo is left untouched (MPI_PROC_NULL).
struct ExchArgs {
  double* f[24];
  int nf;
  int dirmask;  // which directions to exchange (bit d)
};
static __global__ void k_exchange(ExchArgs a) {
  // thread grid: x = face point, y = field
  const int fidx = blockIdx.y;
  if (fidx >= a.nf) return;
  double* f = a.f[fidx];
  const int L = OCFD_L;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nxz = L * cC.ny * cC.nz, nyz = L * cC.nx * cC.nz, nzz = L * cC.nx * cC.ny;
  if ((a.dirmask & 1) && cC.iper[0] && t < nxz) {
    int l = t % L, j = (t / L) % cC.ny + 1, k = t / L / cC.ny + 1;
    f[hidx(cC.nx + 1 + l, j, k)] = f[hidx(1 + l, j, k)];
    f[hidx(1 - L + l, j, k)] = f[hidx(cC.nx + 1 - L + l, j, k)];
  }
  if ((a.dirmask & 2) && cC.iper[1] && t < nyz) {
    int i = t % cC.nx + 1, l = (t / cC.nx) % L, k = t / cC.nx / L + 1;
    f[hidx(i, cC.ny + 1 + l, k)] = f[hidx(i, 1 + l, k)];
    f[hidx(i, 1 - L + l, k)] = f[hidx(i, cC.ny + 1 - L + l, k)];
  }
  if ((a.dirmask & 4) && cC.iper[2] && t < nzz) {
    int i = t % cC.nx + 1, j = (t / cC.nx) % cC.ny + 1, l = t / cC.nx / cC.ny;
    f[hidx(i, j, cC.nz + 1 + l)] = f[hidx(i, j, 1 + l)];
    f[hidx(i, j, 1 - L + l)] = f[hidx(i, j, cC.nz + 1 - L + l)];
  }
}

static __global__ void k_copy(const double* src, double* dst, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = src[t];
}

// comput_Rhybrid, shock sensor 1 (OCFD_SetHybrid.f90:34-43) and forced patches (:80-102)
static __global__ void k_sensor1(const double* p, double* Rh, int npatch, const int* patches) {
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const int q = hidx(i, j, k), sy = cC.HX, sz = cC.HX * cC.HY;
  double r = fabs((p[q - 1] - 2.0 * p[q] + p[q + 1]) / (p[q - 1] + 2.0 * p[q] + p[q + 1])) +
             fabs((p[q - sy] - 2.0 * p[q] + p[q + sy]) / (p[q - sy] + 2.0 * p[q] + p[q + sy])) +
             fabs((p[q - sz] - 2.0 * p[q] + p[q + sz]) / (p[q - sz] + 2.0 * p[q] + p[q + sz]));
  for (int m = 0; m < npatch; m++) {
    const int* b = patches + 6 * m;
    if (i >= b[0] && i <= b[1] && j >= b[2] && j <= b[3] && k >= b[4] && k <= b[5]) r = r + 100.0;
  }
  Rh[q] = r;
}
// sensor 2 (|grad p| / mean): gradient magnitude, then scaled by the host-reduced mean
template <bool SEP>
__global__ void k_sensor2(const double* p, double* Rh, double* partial, Geo g) {
  int i, j, k;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0.0;
  if (cell_of(t, i, j, k)) {
    const int q = hidx(i, j, k);
    double pk = cdiff(p, q, 0, i, cC.nx), pi = cdiff(p, q, 1, j, cC.ny), ps = cdiff(p, q, 2, k, cC.nz);
    double A[9], A1[9];
    metric_all<SEP>(g, i, j, k, q, A, A1);
    double px = pk * A[0] + pi * A[3] + ps * A[6];
    double py = pk * A[1] + pi * A[4] + ps * A[7];
    double pz = pk * A[2] + pi * A[5] + ps * A[8];
    r = sqrt(px * px + py * py + pz * pz);
    Rh[q] = r;
  }
  // deterministic block partial sums (fixed tree order)
  __shared__ double sh[256];
  sh[threadIdx.x] = r;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}
static __global__ void k_sensor2_scale(double* Rh, const double* partial, int nblk, int npatch, const int* patches) {
  // every block re-derives the same total in the same order (deterministic)
  __shared__ double tot;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s = s + partial[b];
    double dp_av = s / (1.0 * cC.nx * cC.ny * cC.nz);
    tot = 1.0 / (dp_av + 1.0e-30);
  }
  __syncthreads();
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const int q = hidx(i, j, k);
  double r = Rh[q] * tot;
  for (int m = 0; m < npatch; m++) {
    const int* b = patches + 6 * m;
    if (i >= b[0] && i <= b[1] && j >= b[2] && j <= b[3] && k >= b[4] && k <= b[5]) r = r + 100.0;
  }
  Rh[q] = r;
}

// ---------------------------------------------------------------- RK3 + primitive variables
struct PrimArgs {
  double* f;
  const double *fn, *du;
  double *d, *u, *v, *w, *T, *p, *Et;  // Et = buffer written this stage
  double* di;
  DevStatus* st;
  int krk;  // 1..3 RK stage; 0 = no update (start-up conversion only)
  double dt;
};
// KRK (1..3, or 0 for the start-up conversion) is a template parameter, so that every stage's
// loads are straight-line code issued together
template <int NS, int KRK>
__global__ void __launch_bounds__(256) k_rk_prims(PrimArgs a) {
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const int q = hidx(i, j, k), nn = nidx(i, j, k);
  const long long N = cC.N;
  double f[5], fo[5], g[5], e[5];
#pragma unroll
  for (int m = 0; m < 5; m++) {
    const size_t o = (size_t)m * N + nn;
    if (KRK >= 1) fo[m] = __ldg(a.fn + o);
    if (KRK >= 1) g[m] = __ldg(a.du + o);
    if (KRK != 1) e[m] = a.f[o];
  }
#pragma unroll
  for (int m = 0; m < 5; m++) {
    if (KRK == 1) f[m] = fo[m] + a.dt * g[m];
    else if (KRK == 2) f[m] = (3.0 / 4.0) * fo[m] + (1.0 / 4.0) * (e[m] + a.dt * g[m]);
    else if (KRK == 3) f[m] = (1.0 / 3.0) * fo[m] + (2.0 / 3.0) * (e[m] + a.dt * g[m]);
    else f[m] = e[m];
    if (KRK != 0) a.f[(size_t)m * N + nn] = f[m];
  }
  double dd = f[0];
  double uu = f[1] / f[0], vv = f[2] / f[0], ww = f[3] / f[0];
  double et = f[4] - (f[1] * uu + f[2] * vv + f[3] * ww) * 0.5;
  a.d[q] = dd; a.u[q] = uu; a.v[q] = vv; a.w[q] = ww;
  a.Et[q] = et;
  if (!(et > 0.0)) {
    if (et <= 0.0) {
      int slot = atomicAdd(&a.st->neg_count, 1);
      if (slot < 16) a.st->neg_list[slot] = nn;
    } else {
      atomicAdd(&a.st->nan_count, 1);
    }
  }
  // Rescaling_di: di >= 0 and sum(di) = d
  double di0[NS];
  double d0 = 0.0;
#pragma unroll
  for (int m = 0; m < NS; m++) {
    double x = a.di[(size_t)m * cC.H + q];
    if (x < 0.0) x = 0.0;
    di0[m] = x;
    d0 = d0 + x;
  }
  double tmp = dd / d0;
#pragma unroll
  for (int m = 0; m < NS; m++) {
    di0[m] = di0[m] * tmp;
    a.di[(size_t)m * cC.H + q] = di0[m];
  }
  double TT = dev_T<NS>(di0, et, &a.st->newton_fail);
  a.T[q] = TT;
  a.p[q] = dev_P<NS>(di0, TT);
}

// handle_NegativeEt replayed in loop order: a repaired cell averages its six neighbours, taking
// this pass's value for interior neighbours earlier in (i,j,k) order and the previous value
// (other Et buffer) for later ones and for halo points. More than 10 such cells stop the run.
template <int NS>
__global__ void k_repair_et(double* f, double* Et_new, const double* Et_old, double* T, double* p, const double* di,
                            DevStatus* st) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int cnt = st->neg_count;
  if (cnt == 0) return;
  st->neg_total += (unsigned long long)cnt;
  if (cnt > 10) {
    st->error = OCFD_ERR_NEGATIVE_ET;
    st->neg_count = 0;
    return;
  }
  int lst[16];
  for (int m = 0; m < cnt; m++) lst[m] = st->neg_list[m];
  for (int a = 1; a < cnt; a++)  // insertion sort into loop order
    for (int b = a; b > 0 && lst[b - 1] > lst[b]; b--) { int t = lst[b]; lst[b] = lst[b - 1]; lst[b - 1] = t; }
  for (int m = 0; m < cnt; m++) {
    int nn = lst[m];
    int i = nn % cC.nx + 1, j = (nn / cC.nx) % cC.ny + 1, k = nn / cC.nx / cC.ny + 1;
    auto nb = [&](int ii, int jj, int kk) {
      bool inside = ii >= 1 && ii <= cC.nx && jj >= 1 && jj <= cC.ny && kk >= 1 && kk <= cC.nz;
      int qq = hidx(ii, jj, kk);
      if (inside && nidx(ii, jj, kk) < nn) return Et_new[qq];
      return Et_old[qq];
    };
    int q = hidx(i, j, k);
    double e0 = Et_new[q];
    double e1 = (nb(i + 1, j, k) + nb(i - 1, j, k) + nb(i, j + 1, k) + nb(i, j - 1, k) + nb(i, j, k + 1) +
                 nb(i, j, k - 1)) /
                6.0;
    Et_new[q] = e1;
    f[4 * cC.N + nn] = f[4 * cC.N + nn] + (e1 - e0);
    double d0[NS];
    for (int s = 0; s < NS; s++) d0[s] = di[(size_t)s * cC.H + q];
    double TT = dev_T<NS>(d0, e1, &st->newton_fail);
    T[q] = TT;
    p[q] = dev_P<NS>(d0, TT);
  }
  st->neg_count = 0;
}

// ---------------------------------------------------------------- boundary conditions
struct BcArgs {
  double *f, *d, *u, *v, *w, *T, *p, *Et, *di;
  const double *inlet, *upper, *wall_pertb;
  const int* nonref;
  int inlet_kind, upper_kind, outlet, jet_iflag;
  double ht, Tw, xinit, disA;
  const double* X;  // Axx (halo array) for the wall start
  Geo g;
};

template <int NS>
__device__ __forceinline__ void set_point(const BcArgs& a, int q, const double* vals) {
  a.d[q] = vals[0]; a.u[q] = vals[1]; a.v[q] = vals[2]; a.w[q] = vals[3]; a.T[q] = vals[4];
#pragma unroll
  for (int m = 0; m < NS; m++) a.di[(size_t)m * cC.H + q] = vals[5 + m];
}
// inlet i = 1 (OCFD_BC_Boundarylayers.f90:60-104)
template <int NS>
__global__ void k_bc_inlet(BcArgs a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cC.ny * cC.nz) return;
  int j = t % cC.ny + 1, k = t / cC.ny + 1;
  double vals[5 + NS];
  for (int c = 0; c < 5 + NS; c++) {
    if (a.inlet_kind == 0) vals[c] = a.inlet[c];
    else if (a.inlet_kind == 1) vals[c] = a.inlet[c * cC.ny + (j - 1)];
    else vals[c] = a.inlet[((size_t)c * cC.nz + (k - 1)) * cC.ny + (j - 1)];
  }
  set_point<NS>(a, hidx(1, j, k), vals);
}
// upper j = ny where the point is Dirichlet (:107-144)
template <int NS>
__global__ void k_bc_upper(BcArgs a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cC.nx * cC.nz) return;
  int i = t % cC.nx + 1, k = t / cC.nx + 1;
  if (a.nonref[t] != 0) return;
  double vals[5 + NS];
  for (int c = 0; c < 5 + NS; c++) {
    if (a.upper_kind == 0) vals[c] = a.upper[c];
    else if (a.upper_kind == 1) vals[c] = a.upper[c * cC.nx + (i - 1)];
    else vals[c] = a.upper[((size_t)c * cC.nz + (k - 1)) * cC.nx + (i - 1)];
  }
  set_point<NS>(a, hidx(i, cC.ny, k), vals);
}
// wall j = 1: blowing/suction, isothermal or adiabatic, dp/dy = 0, non-catalytic (:147-201)
template <int NS, bool SEP>
__global__ void k_bc_wall(BcArgs a, const double* ht) {
  a.ht = *ht;  // h(t) lives in device memory so that a captured graph sees each step's value
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cC.nx * cC.nz) return;
  int i = t % cC.nx + 1, k = t / cC.nx + 1;
  int q1 = hidx(i, 1, k), q2 = hidx(i, 2, k), q3 = hidx(i, 3, k);
  if (a.X[q1] < a.xinit) {
    a.d[q1] = a.d[q2]; a.u[q1] = a.u[q2]; a.v[q1] = a.v[q2]; a.w[q1] = a.w[q2]; a.T[q1] = a.T[q2];
    for (int m = 0; m < NS; m++) a.di[(size_t)m * cC.H + q1] = a.di[(size_t)m * cC.H + q2];
    return;
  }
  double A[9], A1[9];
  metric_all<SEP>(a.g, i, 1, k, q1, A, A1);
  double Aix = A[3], Aiy = A[4], Aiz = A[5];
  double tmp = 1.0 / sqrt(Aix * Aix + Aiy * Aiy + Aiz * Aiz);
  double A0 = a.disA * a.ht * a.wall_pertb[t];
  a.u[q1] = A0 * Aix * tmp;
  a.v[q1] = A0 * Aiy * tmp;
  a.w[q1] = A0 * Aiz * tmp;
  double T1 = a.Tw > 0 ? a.Tw : (4.0 * a.T[q2] - a.T[q3]) / 3.0;
  a.T[q1] = T1;
  double di2[NS], di3[NS], di1[NS];
  for (int m = 0; m < NS; m++) {
    di2[m] = a.di[(size_t)m * cC.H + q2];
    di3[m] = a.di[(size_t)m * cC.H + q3];
  }
  double p2 = dev_P<NS>(di2, a.T[q2]);
  double p3 = dev_P<NS>(di3, a.T[q3]);
  double p1 = (4.0 * p2 - p3) / 3.0;
  double d2 = a.d[q2];
  for (int m = 0; m < NS; m++) di1[m] = di2[m] / d2;
  double d1 = dev_dens<NS>(di1, T1, p1);
  a.d[q1] = d1;
  for (int m = 0; m < NS; m++) a.di[(size_t)m * cC.H + q1] = di1[m] * d1;
}
// outlet i = nx, first / second order extrapolation (:203-231)
template <int NS>
__global__ void k_bc_outlet(BcArgs a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cC.ny * cC.nz) return;
  int j = t % cC.ny + 1, k = t / cC.ny + 1;
  int q = hidx(cC.nx, j, k), q1 = hidx(cC.nx - 1, j, k), q2 = hidx(cC.nx - 2, j, k);
  if (a.outlet == 1) {
    a.d[q] = a.d[q1]; a.u[q] = a.u[q1]; a.v[q] = a.v[q1]; a.w[q] = a.w[q1]; a.T[q] = a.T[q1];
    for (int m = 0; m < NS; m++) a.di[(size_t)m * cC.H + q] = a.di[(size_t)m * cC.H + q1];
  } else {
    a.d[q] = 2.0 * a.d[q1] - a.d[q2]; a.u[q] = 2.0 * a.u[q1] - a.u[q2]; a.v[q] = 2.0 * a.v[q1] - a.v[q2];
    a.w[q] = 2.0 * a.w[q1] - a.w[q2]; a.T[q] = 2.0 * a.T[q1] - a.T[q2];
    for (int m = 0; m < NS; m++)
      a.di[(size_t)m * cC.H + q] = 2.0 * a.di[(size_t)m * cC.H + q1] - a.di[(size_t)m * cC.H + q2];
  }
}
// ocfd_bc_jet inlet (OCFD_BC_jet.f90:21-75): 2-D table; Iflag_inlet 0 = Dirichlet, 1 = keep the
// interior pressure where the inflow is subsonic (u < c)
template <int NS>
__global__ void k_bc_jet_inlet(BcArgs a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cC.ny * cC.nz) return;
  int j = t % cC.ny + 1, k = t / cC.ny + 1;
  int q = hidx(1, j, k);
  double vals[5 + NS];
  for (int c = 0; c < 5 + NS; c++) vals[c] = a.inlet[((size_t)c * cC.nz + (k - 1)) * cC.ny + (j - 1)];
  if (a.jet_iflag == 0) {
    set_point<NS>(a, q, vals);
    return;
  }
  a.u[q] = vals[1]; a.v[q] = vals[2]; a.w[q] = vals[3]; a.T[q] = vals[4];
  double T1 = vals[4], d1 = vals[0], di1[NS], ai1[NS], d0 = 0.0;
  for (int m = 0; m < NS; m++) { di1[m] = vals[5 + m]; d0 = d0 + di1[m]; }
  for (int m = 0; m < NS; m++) ai1[m] = di1[m] / d0;
  double p1 = dev_P<NS>(di1, T1);
  double Et1 = dev_E<NS>(di1, T1);
  double gamma = p1 / Et1 + 1.0;
  double c1 = sqrt(gamma * p1 / d1);
  if (vals[1] < c1) {
    double pp = a.p[hidx(2, j, k)];
    a.p[q] = pp;
    double dn = dev_dens<NS>(ai1, T1, pp);
    a.d[q] = dn;
    for (int m = 0; m < NS; m++) a.di[(size_t)m * cC.H + q] = dn * ai1[m];
  } else {
    a.d[q] = d1;
    for (int m = 0; m < NS; m++) a.di[(size_t)m * cC.H + q] = di1[m];
  }
}
// ocfd_bc_jet outlet (:77-93): zeroth-order extrapolation of every primitive
template <int NS>
__global__ void k_bc_jet_outlet(BcArgs a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cC.ny * cC.nz) return;
  int j = t % cC.ny + 1, k = t / cC.ny + 1;
  int q = hidx(cC.nx, j, k), q1 = hidx(cC.nx - 1, j, k);
  a.d[q] = a.d[q1]; a.u[q] = a.u[q1]; a.v[q] = a.v[q1]; a.w[q] = a.w[q1]; a.T[q] = a.T[q1];
  a.p[q] = a.p[q1]; a.Et[q] = a.Et[q1];
  for (int m = 0; m < NS; m++) a.di[(size_t)m * cC.H + q] = a.di[(size_t)m * cC.H + q1];
}

// OCFD_bc lines 33-184: every domain-face cell gets di re-scaled, Et and p re-derived from T and
// f rebuilt, once per face it lies on (edges twice, corners three times, as the sequential face
// loops of the reference do). group 0: i faces; 1: j faces without i faces; 2: k faces only.
template <int NS>
__device__ __forceinline__ void face_apply(const BcArgs& a, int i, int j, int k, int times) {
  const int q = hidx(i, j, k), nn = nidx(i, j, k);
  const long long N = cC.N;
  double dd = a.d[q], uu = a.u[q], vv = a.v[q], ww = a.w[q], TT = a.T[q];
  double di1[NS];
  for (int m = 0; m < NS; m++) di1[m] = a.di[(size_t)m * cC.H + q];
  double et = 0.0, pp = 0.0;
  for (int r = 0; r < times; r++) {
    double d0 = 0.0;
    for (int m = 0; m < NS; m++) d0 = d0 + di1[m];
    double dtmp = dd / d0;
    for (int m = 0; m < NS; m++) di1[m] = di1[m] * dtmp;
    et = dev_E<NS>(di1, TT);
    pp = dev_P<NS>(di1, TT);
  }
  for (int m = 0; m < NS; m++) a.di[(size_t)m * cC.H + q] = di1[m];
  a.Et[q] = et;
  a.p[q] = pp;
  a.f[nn] = dd;
  a.f[N + nn] = dd * uu;
  a.f[2 * N + nn] = dd * vv;
  a.f[3 * N + nn] = dd * ww;
  a.f[4 * N + nn] = et + dd * (uu * uu + vv * vv + ww * ww) * 0.5;
}
template <int NS>
__global__ void k_bc_faces(BcArgs a, int group) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = cC.nx, ny = cC.ny, nz = cC.nz;
  int i, j, k;
  if (group == 0) {
    if (t >= 2 * ny * nz) return;
    i = (t & 1) ? nx : 1;
    int r = t >> 1;
    j = r % ny + 1;
    k = r / ny + 1;
  } else if (group == 1) {
    if (t >= 2 * (nx - 2) * nz) return;
    j = (t & 1) ? ny : 1;
    int r = t >> 1;
    i = r % (nx - 2) + 2;
    k = r / (nx - 2) + 1;
  } else {
    if (t >= 2 * (nx - 2) * (ny - 2)) return;
    k = (t & 1) ? nz : 1;
    int r = t >> 1;
    i = r % (nx - 2) + 2;
    j = r / (nx - 2) + 2;
  }
  int times = (i == 1) + (i == nx) + (j == 1) + (j == ny) + (k == 1) + (k == nz);
  face_apply<NS>(a, i, j, k, times);
}
// Flow_Ghost_Extent_2nd (OCFD_GhostCell.f90:166-364): face halos of faces with Ghost_Cell = 1/2
template <int NS>
__global__ void k_bc_ghost(BcArgs a, int face) {
  const int dir = face / 2, side = face % 2;
  const int n = dir == 0 ? cC.nx : (dir == 1 ? cC.ny : cC.nz);
  const int na = dir == 0 ? cC.ny : cC.nx, nb = dir == 2 ? cC.ny : cC.nz;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na * nb * OCFD_L) return;
  int aa = t % na + 1, l = (t / na) % OCFD_L + 1, bb = t / na / OCFD_L + 1;
  int ig = side == 0 ? 1 - l : n + l, ib = side == 0 ? 1 : n, im = side == 0 ? 2 - ig : 2 * n - ig;
  auto at = [&](int s) {
    if (dir == 0) return hidx(s, aa, bb);
    if (dir == 1) return hidx(aa, s, bb);
    return hidx(aa, bb, s);
  };
  int qg = at(ig), qb = at(ib), qm = at(im);
  const double s1 = 0.8, s2 = 1.2;
  a.u[qg] = 2.0 * a.u[qb] - a.u[qm]; a.v[qg] = 2.0 * a.v[qb] - a.v[qm]; a.w[qg] = 2.0 * a.w[qb] - a.w[qm];
  double dg = 2.0 * a.d[qb] - a.d[qm], Tg = 2.0 * a.T[qb] - a.T[qm];
  if (dg < s1 * a.d[qb]) dg = s1 * a.d[qb];
  if (dg > s2 * a.d[qb]) dg = s2 * a.d[qb];
  if (Tg < s1 * a.T[qb]) Tg = s1 * a.T[qb];
  if (Tg > s2 * a.T[qb]) Tg = s2 * a.T[qb];
  a.d[qg] = dg;
  a.T[qg] = Tg;
  double di1[NS], d0 = 0.0;
  for (int m = 0; m < NS; m++) {
    di1[m] = 2.0 * a.di[(size_t)m * cC.H + qb] - a.di[(size_t)m * cC.H + qm];
    d0 = d0 + di1[m];
  }
  double dtmp = dg / d0;
  for (int m = 0; m < NS; m++) {
    di1[m] = di1[m] * dtmp;
    a.di[(size_t)m * cC.H + qg] = di1[m];
  }
  a.Et[qg] = dev_E<NS>(di1, Tg);
  a.p[qg] = dev_P<NS>(di1, Tg);
}

// start-up: d,u,v,w,T,di from primitive input, Rescaling_di, conserved f (OCFD_init.f90:8-25)
template <int NS>
__global__ void k_init_state(const double* prim5, const double* din, double* f, double* d, double* u, double* v,
                             double* w, double* T, double* di) {
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const int q = hidx(i, j, k), nn = nidx(i, j, k);
  const long long N = cC.N;
  double dd = prim5[nn], uu = prim5[N + nn], vv = prim5[2 * N + nn], ww = prim5[3 * N + nn], TT = prim5[4 * N + nn];
  d[q] = dd; u[q] = uu; v[q] = vv; w[q] = ww; T[q] = TT;
  double di1[NS], d0 = 0.0;
  for (int m = 0; m < NS; m++) {
    double x = din[(size_t)m * N + nn];
    if (x < 0.0) x = 0.0;
    di1[m] = x;
    d0 = d0 + x;
  }
  double tmp = dd / d0;
  for (int m = 0; m < NS; m++) {
    di1[m] = di1[m] * tmp;
    di[(size_t)m * cC.H + q] = di1[m];
  }
  f[nn] = dd;
  f[N + nn] = dd * uu;
  f[2 * N + nn] = dd * vv;
  f[3 * N + nn] = dd * ww;
  double et1 = dev_E<NS>(di1, TT);
  f[4 * N + nn] = et1 + dd * (uu * uu + vv * vv + ww * ww) * 0.5;
}

// show_flow_msg sums with a fixed reduction tree (two passes, deterministic)
template <bool SEP>
__global__ void k_diag(const double* f, const double* d, const double* u, const double* v, const double* w,
                       double* partial, Geo g) {
  __shared__ double s1[256], s2[256];
  int i, j, k;
  double e = 0.0, kk = 0.0;
  if (cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) {
    const int q = hidx(i, j, k), nn = nidx(i, j, k);
    double tmp0 = 1.0 / metric_jac<SEP>(g, i, j, k, q);
    e = f[4 * cC.N + nn] * tmp0;
    kk = d[q] * (u[q] * u[q] + v[q] * v[q] + w[q] * w[q]) * 0.5 * tmp0;
  }
  s1[threadIdx.x] = e;
  s2[threadIdx.x] = kk;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s1[threadIdx.x] = s1[threadIdx.x] + s1[threadIdx.x + s];
      s2[threadIdx.x] = s2[threadIdx.x] + s2[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s1[0];
    partial[2 * blockIdx.x + 1] = s2[0];
  }
}

}  // namespace ocfd
