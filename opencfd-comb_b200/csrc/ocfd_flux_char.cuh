// Characteristic-space inviscid flux (IF_Scheme_Character = 1): du_inviscous_Character and
// flux_charteric of OCFD_inviscous_character.f90:3-319.
//
// Same tiles as k_flux. Phase 1 splits every point into shared memory and also keeps the point
// state (u, v, w, c, p, Et and the metric vector) for the interface averages. Phase 2a: one
// thread per (component m, interface): the split fluxes of the stencil are projected on row m of
// the left eigenvector matrix of the interface-averaged state and reconstructed (scheme and
// boundary closures as in the component-wise sweep), h0(m) = h+ + h-. Phase 2b: row m of the
// right eigenvector matrix maps h0 back (HYBRID interfaces on the linear scheme skip both
// projections); a closed face with the default closure takes the non-reflecting physical flux at
// interfaces 0 and n. Phase 3 forms the flux difference like k_flux.
#pragma once
#include "ocfd_flow.cuh"

namespace ocfd {

// interface-averaged state and the orthonormal frame (n, l, m) of the metric vector
struct CharState {
  double u1, v1, w1, c1, n1, n2, n3, l1, l2, l3, m1, m2, m3, un, ul, um, V2, KK, KK1, X1, Hh;
};
__device__ __forceinline__ CharState char_state(double u1, double v1, double w1, double c1, double p1, double Et1,
                                                double a1, double a2, double a3) {
  CharState s;
  s.u1 = u1; s.v1 = v1; s.w1 = w1; s.c1 = c1;
  double ss = sqrt(a1 * a1 + a2 * a2 + a3 * a3);
  s.n1 = a1 / ss; s.n2 = a2 / ss; s.n3 = a3 / ss;
  if (fabs(s.n3) <= fabs(s.n2)) {
    ss = sqrt(s.n1 * s.n1 + s.n2 * s.n2);
    s.l1 = -s.n2 / ss; s.l2 = s.n1 / ss; s.l3 = 0.0;
  } else {
    ss = sqrt(s.n1 * s.n1 + s.n3 * s.n3);
    s.l1 = -s.n3 / ss; s.l2 = 0.0; s.l3 = s.n1 / ss;
  }
  s.m1 = s.n2 * s.l3 - s.n3 * s.l2;
  s.m2 = s.n3 * s.l1 - s.n1 * s.l3;
  s.m3 = s.n1 * s.l2 - s.n2 * s.l1;
  s.un = u1 * s.n1 + v1 * s.n2 + w1 * s.n3;
  s.ul = u1 * s.l1 + v1 * s.l2 + w1 * s.l3;
  s.um = u1 * s.m1 + v1 * s.m2 + w1 * s.m3;
  s.V2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5;
  double gamma = p1 / Et1 + 1.0;
  s.KK = (gamma - 1.0) / (c1 * c1);
  s.KK1 = s.KK * 0.5;
  s.X1 = 1.0 / (2.0 * c1);
  s.Hh = s.V2 + 1.0 / s.KK;
  return s;
}
// row r of the left (S) eigenvector matrix
__device__ __forceinline__ void char_left_row(const CharState& s, int r, double* o) {
  switch (r) {
    case 0: o[0] = 1.0 - s.KK * s.V2; o[1] = s.KK * s.u1; o[2] = s.KK * s.v1; o[3] = s.KK * s.w1; o[4] = -s.KK; break;
    case 1: o[0] = -s.ul; o[1] = s.l1; o[2] = s.l2; o[3] = s.l3; o[4] = 0.0; break;
    case 2: o[0] = -s.um; o[1] = s.m1; o[2] = s.m2; o[3] = s.m3; o[4] = 0.0; break;
    case 3:
      o[0] = s.KK1 * s.V2 + s.X1 * s.un;
      o[1] = -s.X1 * s.n1 - s.KK1 * s.u1;
      o[2] = -s.X1 * s.n2 - s.KK1 * s.v1;
      o[3] = -s.X1 * s.n3 - s.KK1 * s.w1;
      o[4] = s.KK1;
      break;
    default:
      o[0] = s.KK1 * s.V2 - s.X1 * s.un;
      o[1] = s.X1 * s.n1 - s.KK1 * s.u1;
      o[2] = s.X1 * s.n2 - s.KK1 * s.v1;
      o[3] = s.X1 * s.n3 - s.KK1 * s.w1;
      o[4] = s.KK1;
  }
}
// row r of the right (S1) eigenvector matrix
__device__ __forceinline__ void char_right_row(const CharState& s, int r, double* o) {
  const double c1 = s.c1;
  switch (r) {
    case 0: o[0] = 1.0; o[1] = 0.0; o[2] = 0.0; o[3] = 1.0; o[4] = 1.0; break;
    case 1: o[0] = s.u1; o[1] = s.l1; o[2] = s.m1; o[3] = s.u1 - c1 * s.n1; o[4] = s.u1 + c1 * s.n1; break;
    case 2: o[0] = s.v1; o[1] = s.l2; o[2] = s.m2; o[3] = s.v1 - c1 * s.n2; o[4] = s.v1 + c1 * s.n2; break;
    case 3: o[0] = s.w1; o[1] = s.l3; o[2] = s.m3; o[3] = s.w1 - c1 * s.n3; o[4] = s.w1 + c1 * s.n3; break;
    default: o[0] = s.V2; o[1] = s.ul; o[2] = s.um; o[3] = s.Hh - c1 * s.un; o[4] = s.Hh + c1 * s.un;
  }
}

template <int DIR>
struct CharTile {
  static constexpr int C = Tile<DIR>::C, NL = Tile<DIR>::NL, P = C + 8, NI = (C + 1) * NL;
  static constexpr int NQ = 9;  // u, v, w, c, p, Et, A1, A2, A3
  static constexpr size_t smem = sizeof(double) * (size_t)((10 + NQ) * P * NL + 10 * NI) + sizeof(int) * NI;
};

template <int DIR, int SCHEME, int SPLIT, bool SEP>
__global__ void __launch_bounds__(FLUX_THREADS, 2) k_flux_char(FluxArgs a) {
  using T = CharTile<DIR>;
  constexpr int C = T::C, NL = T::NL, P = T::P, NI = T::NI, NQ = T::NQ;
  constexpr bool HYB = SCHEME == OCFD_SCHEME_HYBRID;
  extern __shared__ double smem[];
  double* sf = smem;                // [10][P x NL]: F+ (5) then F- (5)
  double* sq = sf + 10 * P * NL;    // [NQ][P x NL]: point state
  double* sh0 = sq + NQ * P * NL;   // [5][NI]: h0 in characteristic (or physical) space
  double* shh = sh0 + 5 * NI;       // [5][NI]: interface fluxes
  int* sscm = reinterpret_cast<int*>(shh + 5 * NI);
  auto sidx = [&](int c, int p, int l) { return DIR == 0 ? (c * NL + l) * P + p : (c * P + p) * NL + l; };
  auto iidx = [&](int t, int l) { return DIR == 0 ? l * (C + 1) + t : t * NL + l; };

  const int n = DIR == 0 ? cC.nx : (DIR == 1 ? cC.ny : cC.nz);
  const int s0 = (DIR == 0 ? blockIdx.x : blockIdx.y) * C + 1;
  const int l0 = DIR == 0 ? blockIdx.y * NL + 1 : blockIdx.x * NL + 1;
  const int bz = blockIdx.z + 1;
  const int nl_max = DIR == 0 ? cC.ny : cC.nx;
  const int ncell = min(C, n - s0 + 1);
  const int stride = hstride(DIR);
  auto coords = [&](int s, int l, int& i, int& j, int& k) {
    if (DIR == 0) { i = s; j = l0 + l; k = bz; }
    else if (DIR == 1) { i = l0 + l; j = s; k = bz; }
    else { i = l0 + l; j = bz; k = s; }
  };
  const int b0 = cC.bound[DIR][0], b1 = cC.bound[DIR][1], sb0 = cC.sb[2 * DIR], sb1 = cC.sb[2 * DIR + 1];
  const int ia = (b0 == 0 || sb0 != 0) ? 0 : 1, ib = (b1 == 0 || sb1 != 0) ? n : n - 1;

  // phase 1: split fluxes and state of every point, hybrid index of every interface
  for (int idx = threadIdx.x; idx < P * NL; idx += FLUX_THREADS) {
    int p, l;
    if (DIR == 0) { p = idx % P; l = idx / P; }
    else { l = idx % NL; p = idx / NL; }
    const bool line_ok = l0 + l <= nl_max;
    double fp[5], fm[5], st[NQ];
    if (line_ok && p < ncell + 8) {
      int i, j, k;
      coords(s0 - 4 + p, l, i, j, k);
      const int q = hidx(i, j, k);
      double A1, A2, A3;
      metric_dir<SEP>(a.g, DIR, i, j, k, q, A1, A2, A3);
      double pp = __ldg(a.p + q), et = __ldg(a.Et + q), dd = __ldg(a.d + q);
      double uu = __ldg(a.u + q), vv = __ldg(a.v + q), ww = __ldg(a.w + q);
      double gamma = pp / et + 1.0;
      double cc = sqrt(gamma * pp / dd);  // comput_cc
      split_point<SPLIT>(et, pp, cc, dd, uu, vv, ww, A1, A2, A3, fp, fm);
      st[0] = uu; st[1] = vv; st[2] = ww; st[3] = cc; st[4] = pp; st[5] = et; st[6] = A1; st[7] = A2; st[8] = A3;
    } else {
#pragma unroll
      for (int c = 0; c < 5; c++) fp[c] = fm[c] = 0.0;
#pragma unroll
      for (int c = 0; c < NQ; c++) st[c] = 0.0;
    }
#pragma unroll
    for (int c = 0; c < 5; c++) {
      sf[sidx(c, p, l)] = fp[c];
      sf[sidx(5 + c, p, l)] = fm[c];
    }
#pragma unroll
    for (int c = 0; c < NQ; c++) sq[sidx(c, p, l)] = st[c];
    const int t = p - 3;
    if (line_ok && t >= 0 && t <= ncell) {
      int scm = 0;
      if (HYB) {
        int i, j, k;
        coords(s0 - 1 + t, l, i, j, k);
        const int q = hidx(i, j, k);
        scm = hybrid_index(fmax(__ldg(a.Rh + q), __ldg(a.Rh + q + stride)));
      }
      sscm[iidx(t, l)] = scm;
    }
  }
  __syncthreads();

  auto state_at = [&](int t, int l) {  // interface t lies between points t+3 and t+4
    const int pa = sidx(0, t + 3, l), pb = sidx(0, t + 4, l), cs = P * NL;
    auto avg = [&](int c) { return (sq[c * cs + pa] + sq[c * cs + pb]) * 0.5; };
    return char_state(avg(0), avg(1), avg(2), avg(3), avg(4), avg(5), avg(6), avg(7), avg(8));
  };

  // phase 2a: h0(m) at interfaces ia..ib
  for (int idx = threadIdx.x; idx < 5 * NI; idx += FLUX_THREADS) {
    const int m = idx / NI, it = idx - m * NI;
    int t, l;
    if (DIR == 0) { t = it % (C + 1); l = it / (C + 1); }
    else { l = it % NL; t = it / NL; }
    const int ig = s0 - 1 + t;
    if (l0 + l > nl_max || t > ncell || ig < ia || ig > ib) continue;
    const int scm = sscm[it];
    double gp[8], gm[8];  // stencil offsets -3..4
    if (HYB && scm == 1) {
#pragma unroll
      for (int mm = 0; mm < 8; mm++) {
        gp[mm] = sf[sidx(m, t + mm, l)];
        gm[mm] = sf[sidx(5 + m, t + mm, l)];
      }
    } else {
      const CharState s = state_at(t, l);
      double r[5];
      char_left_row(s, m, r);
#pragma unroll
      for (int mm = 0; mm < 8; mm++) {
        const int pt = t + mm;
        gp[mm] = r[0] * sf[sidx(0, pt, l)] + r[1] * sf[sidx(1, pt, l)] + r[2] * sf[sidx(2, pt, l)] +
                 r[3] * sf[sidx(3, pt, l)] + r[4] * sf[sidx(4, pt, l)];
        gm[mm] = r[0] * sf[sidx(5, pt, l)] + r[1] * sf[sidx(6, pt, l)] + r[2] * sf[sidx(7, pt, l)] +
                 r[3] * sf[sidx(8, pt, l)] + r[4] * sf[sidx(9, pt, l)];
      }
    }
    const double h1v = interface_flux<SCHEME, true, 1>(gp + 3, ig, n, DIR, scm);
    const double h2v = interface_flux<SCHEME, false, 1>(gm + 3, ig, n, DIR, scm);
    sh0[m * NI + it] = h1v + h2v;
  }
  __syncthreads();

  // phase 2b: back to physical space; non-reflecting faces
  for (int idx = threadIdx.x; idx < 5 * NI; idx += FLUX_THREADS) {
    const int m = idx / NI, it = idx - m * NI;
    int t, l;
    if (DIR == 0) { t = it % (C + 1); l = it / (C + 1); }
    else { l = it % NL; t = it / NL; }
    const int ig = s0 - 1 + t;
    if (l0 + l > nl_max || t > ncell) continue;
    double h;
    if (ig >= ia && ig <= ib) {
      if (HYB && sscm[it] == 1) {
        h = sh0[m * NI + it];
      } else {
        const CharState s = state_at(t, l);
        double r[5];
        char_right_row(s, m, r);
        h = r[0] * sh0[it] + r[1] * sh0[NI + it] + r[2] * sh0[2 * NI + it] + r[3] * sh0[3 * NI + it] +
            r[4] * sh0[4 * NI + it];
      }
    } else if (ig == 0) {  // point p of cell c is c - s0 + 4
      auto FP = [&](int c) { return sf[sidx(m, c - s0 + 4, l)]; };
      auto FM = [&](int c) { return sf[sidx(5 + m, c - s0 + 4, l)]; };
      h = (2.0 * FP(1) + 5.0 * FP(2) - FP(3) + 2.0 * FM(3) - 7.0 * FM(2) + 11.0 * FM(1)) / 6.0;
    } else {  // ig == n
      auto FP = [&](int c) { return sf[sidx(m, c - s0 + 4, l)]; };
      auto FM = [&](int c) { return sf[sidx(5 + m, c - s0 + 4, l)]; };
      h = (2.0 * FP(n - 2) - 7.0 * FP(n - 1) + 11.0 * FP(n) + 2.0 * FM(n) + 5.0 * FM(n - 1) - FM(n - 2)) / 6.0;
    }
    shh[m * NI + it] = h;
  }
  __syncthreads();

  // phase 3: flux difference into du
  const double h1 = cC.h1[DIR];
  const long long N = cC.N;
  for (int idx = threadIdx.x; idx < C * NL; idx += FLUX_THREADS) {
    int t, l;
    if (DIR == 0) { t = idx % C; l = idx / C; }
    else { l = idx % NL; t = idx / NL; }
    if (l0 + l > nl_max || t >= ncell) continue;
    int i, j, k;
    coords(s0 + t, l, i, j, k);
    const int nn = nidx(i, j, k);
    double ajac = 0.0;
    if (DIR == 2) ajac = metric_jac<SEP>(a.g, i, j, k, hidx(i, j, k));
    const int i0 = iidx(t, l), i1 = iidx(t + 1, l);
#pragma unroll
    for (int c = 0; c < 5; c++) {
      double val = (shh[c * NI + i1] - shh[c * NI + i0]) * h1;
      double* o = a.out + (size_t)c * N + nn;
      if (DIR == 0) *o = val;
      else if (DIR == 1) *o = *o + val;
      else *o = -(*o + val) * ajac;
    }
    if (DIR == 2 && cC.if_mass_force == 1) {
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

}  // namespace ocfd
