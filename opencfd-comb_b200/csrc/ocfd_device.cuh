// Device-side constants and per-point math of the OpenCFD-Comb hot path (sm_100a).
//
// Every routine keeps the reference's evaluation order (left-to-right sums, gfortran's
// integer-power chains, single-precision literals where the Fortran has them) so that, with
// --fmad=false, the kernels reproduce the CPU restatement bit for bit wherever no
// transcendental function (exp/log/pow/sin) is involved.
#pragma once
#include <cstdint>
#include "../../include/ocfd_gpu.h"

#define OCFD_L 4  // halo width LAP
// 1 in the contracted multiply-add build (libocfd_gpu_fma.so): algebraic forms with fewer FP64
// divisions that give the same values up to rounding
#ifndef OCFD_FMA_BUILD
#define OCFD_FMA_BUILD 0
#endif

namespace ocfd {

// ---------------------------------------------------------------- constant memory
struct DevConst {
  int nx, ny, nz, ns;
  // division of a 31-bit cell index by nx and ny as a multiply-high and a shift (magic numbers of
  // fast_divisor, filled by the host)
  unsigned mx, my;
  int sx, sy;
  // slab order of the gather-bound per-cell kernels: tiles of jt rows (a power of two dividing ny),
  // each walked plane by plane (k), so the z neighbours of a cell were read a few planes earlier
  // by the same tile; magic pairs of the slab (jt nx) and tile (jt nx nz) cell counts
  int jt;
  unsigned m_slab, m_tile;
  int s_slab, s_tile;
  int HX, HY, HZ;
  long long H, N;
  int iper[3];
  int bound[3][2];  // Bound_index(side, dir) of set_parameters (OCFD_readpara.f90:360-369)
  int sb[6];        // Scheme_boundary
  int ghost[6];
  int scheme, split, Ka1, Kb1, Ka2, Kb2;
  double UD7L[8];
  double theta1, theta2;
  double h[3], h1[3];      // hx,hy,hz and 1/h
  double cd6[3][3];        // 1/(60h), -3/(20h), 3/(4h)
  double cd8[3][4];        // 0.8/h, -0.2/h, 3.8095e-2/h, -3.5714e-3/h
  double h2x[3], h12x[3];  // 2h, 12h (closures)
  int cd8_on;
  int if_viscous, if_mass_force;
  double mass_force[3];
  int realgas;
  // thermo (read_Spec)
  int n_tct;
  double tct[OCFD_NTCT_MAX], tct_max;
  double Mi[OCFD_MAX_SPEC], Ri[OCFD_MAX_SPEC];
  double rMi[OCFD_MAX_SPEC];  // 1 / Mi (the contracted build's mole numbers)
  double cf[OCFD_MAX_SPEC][OCFD_NTCT_MAX][8];  // A,B,C,D,E,F,G,Ect
  double mratio[OCFD_MAX_SPEC][OCFD_MAX_SPEC];  // Mi(i) / Mi(j), for the implicit-Euler matrix
  // transport
  int flag_vis, flag_cond, flag_diff;
  double amu0, pr, sc;
  double mu_an[OCFD_MAX_SPEC][4], k_an[OCFD_MAX_SPEC][4];
  double d_an[OCFD_MAX_SPEC][OCFD_MAX_SPEC][4];
  // Wilke pair constants of comput_vis_coeff, sqrt(Mi(j)/Mi(k)) and sqrt(8*(1+Mi(k)/Mi(j))):
  // cell-independent, evaluated on the host with the same correctly rounded operations
  double wk_a[OCFD_MAX_SPEC][OCFD_MAX_SPEC], wk_b[OCFD_MAX_SPEC][OCFD_MAX_SPEC];
  // the same pair constants for the multi-species transport kernel: sqrt(wk_a) and 1 / wk_b
  double wk_c[OCFD_MAX_SPEC][OCFD_MAX_SPEC], wk_binv[OCFD_MAX_SPEC][OCFD_MAX_SPEC];
  // species pairs (a, b), a < b, enumerated a-major: pair p = (pair_a[p], pair_b[p])
  unsigned char pair_a[OCFD_MAX_SPEC * (OCFD_MAX_SPEC - 1) / 2], pair_b[OCFD_MAX_SPEC * (OCFD_MAX_SPEC - 1) / 2];
  unsigned char pair_of[OCFD_MAX_SPEC][OCFD_MAX_SPEC];  // the pair number of (a, b) and (b, a)
  // kinetics
  int nreac, rereac, timeadv;
  int const_p;  // batched reactors: hold each reactor's pressure (extension; the reference is constant-volume)
  int af_type[OCFD_MAX_REAC], tr_reac[OCFD_MAX_REAC];
  double fc_troe[OCFD_MAX_REAC];
  double af[OCFD_MAX_REAC][2], bf[OCFD_MAX_REAC][2], ef[OCFD_MAX_REAC][2];
  double ar[OCFD_MAX_REAC], br[OCFD_MAX_REAC], er[OCFD_MAX_REAC];
  double park[OCFD_MAX_REAC][5];
  signed char vf[OCFD_MAX_REAC][OCFD_MAX_SPEC], vr[OCFD_MAX_REAC][OCFD_MAX_SPEC];
  int sgm[OCFD_MAX_REAC];
  double treff[OCFD_MAX_REAC][OCFD_MAX_SPEC];
};

// defined once (ocfd_gpu.cu); the sweep / chemistry translation units share it through
// relocatable device code
#ifdef OCFD_DEFINE_CONST
__constant__ DevConst cC;
#else
extern __constant__ DevConst cC;
#endif

// geometry: either 19 full metric arrays or, for tensor-product grids, three 1-D derivative
// arrays plus the cross derivatives that the one-sided closures of OCFD_dx0/dy0/dz0 leave at the
// non-periodic end planes (e.g. (-3y+4y-y)/(2h) at i = 1 is a rounding residue, not zero).
struct Geo {
  const double* m[19];   // Akx,Aky,Akz,Aix,Aiy,Aiz,Asx,Asy,Asz,Ajac,Akx1..Asz1 (halo layout)
  const double* d1[3];   // dx/dxi(i), dy/deta(j), dz/dzeta(k), halo-inclusive, index s+L-1
  const double* e[6];    // cross terms at the end planes, [side][index+L-1]:
                         //   yi(j), zi(k) at i=1|nx; xj(i), zj(k) at j=1|ny; xk(i), yk(j) at k=1|nz
};
enum { G_AKX = 0, G_AKY, G_AKZ, G_AIX, G_AIY, G_AIZ, G_ASX, G_ASY, G_ASZ, G_AJAC, G_AKX1 };
enum { E_YI = 0, E_ZI, E_XJ, E_ZJ, E_XK, E_YK };

__device__ __forceinline__ int hidx(int i, int j, int k) {
  return (i + OCFD_L - 1) + cC.HX * ((j + OCFD_L - 1) + cC.HY * (k + OCFD_L - 1));
}
__device__ __forceinline__ int nidx(int i, int j, int k) { return (i - 1) + cC.nx * ((j - 1) + cC.ny * (k - 1)); }
// n / d for n < 2^31 with the host's magic pair (m, s) of d (fast_divisor): floor(n m / 2^(32 + s)),
// and n itself for d = 1 (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994: m = ceil(2^(31 + l) / d), l = ceil(log2 d), s = l - 1)
__device__ __forceinline__ unsigned fast_div(unsigned n, unsigned d, unsigned m, int s) {
  return d == 1 ? n : __umulhi(n, m) >> s;
}
// x / N for a small integer N: the division the reference evaluates in the exact build, a
// multiplication by the rounded reciprocal (the same value up to rounding) in the contracted one
template <int N>
__device__ __forceinline__ double divc(double x) {
#if OCFD_FMA_BUILD
  return x * (1.0 / N);
#else
  return x / N;
#endif
}
__device__ __forceinline__ int hstride(int dir) { return dir == 0 ? 1 : (dir == 1 ? cC.HX : cC.HX * cC.HY); }

// gfortran -O3 integer-power chains (GCC powi table): x**3 = x**2*x, x**4 = (x**2)**2, x**5 = x**2*x**3
__device__ __forceinline__ double q2(double x) { return x * x; }
__device__ __forceinline__ double q3(double x) { double a = x * x; return a * x; }
__device__ __forceinline__ double q4(double x) { double a = x * x; return a * a; }
__device__ __forceinline__ double q5(double x) { double a = x * x; double b = a * x; return a * b; }
// libgcc __powidf2: x**n for a run-time integer n (square-and-multiply, then reciprocal)
__device__ __forceinline__ double powi_rt(double x, int m) {
  unsigned n = m < 0 ? -(unsigned)m : (unsigned)m;
  double y = (n & 1u) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n & 1u) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}
__device__ __forceinline__ double fsgn(double x) { return signbit(x) ? -1.0 : 1.0; }

// ---------------------------------------------------------------- metrics
// comput_Jacobian3d (OCFD_mesh.f90:88-98) from the nine coordinate derivatives; for a separable
// grid the cross derivatives are zero except on the non-periodic end planes, where the closure
// residues are looked up, so every point reproduces the reference's 3-D arrays exactly.
__device__ __forceinline__ void sep_derivs(const Geo& g, int i, int j, int k, double& xi, double& yi, double& zi,
                                           double& xj, double& yj, double& zj, double& xk, double& yk, double& zk,
                                           bool& cross) {
  const int L = OCFD_L;
  xi = g.d1[0][i + L - 1];
  yj = g.d1[1][j + L - 1];
  zk = g.d1[2][k + L - 1];
  yi = zi = xj = zj = xk = yk = 0.0;
  const bool bx = !cC.iper[0] && (i == 1 || i == cC.nx);
  const bool by = !cC.iper[1] && (j == 1 || j == cC.ny);
  const bool bz = !cC.iper[2] && (k == 1 || k == cC.nz);
  cross = bx || by || bz;
  if (bx) {
    int s = i == 1 ? 0 : 1;
    yi = g.e[E_YI][s * (cC.ny + 2 * L) + j + L - 1];
    zi = g.e[E_ZI][s * (cC.nz + 2 * L) + k + L - 1];
  }
  if (by) {
    int s = j == 1 ? 0 : 1;
    xj = g.e[E_XJ][s * (cC.nx + 2 * L) + i + L - 1];
    zj = g.e[E_ZJ][s * (cC.nz + 2 * L) + k + L - 1];
  }
  if (bz) {
    int s = k == 1 ? 0 : 1;
    xk = g.e[E_XK][s * (cC.nx + 2 * L) + i + L - 1];
    yk = g.e[E_YK][s * (cC.ny + 2 * L) + j + L - 1];
  }
}
// halo points the reference never fills (non-periodic face halos, edges, corners) keep
// allocate_flow_data's 1.0 in every metric array; they enter the split flux when a face uses
// Scheme_boundary = -1 or 1
__device__ __forceinline__ bool metric_unfilled(int i, int j, int k) {
  const bool ox = i < 1 || i > cC.nx, oy = j < 1 || j > cC.ny, oz = k < 1 || k > cC.nz;
  const int n = (int)ox + (int)oy + (int)oz;
  return n > 1 || (ox && !cC.iper[0]) || (oy && !cC.iper[1]) || (oz && !cC.iper[2]);
}
__device__ __forceinline__ void jac_full(double xi1, double yi1, double zi1, double xj1, double yj1, double zj1,
                                         double xk1, double yk1, double zk1, double* a, double& jac) {
  jac = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1 - zi1 * yj1 * xk1 - yi1 * xj1 * zk1 -
               xi1 * zj1 * yk1);
  a[0] = jac * (yj1 * zk1 - zj1 * yk1);
  a[1] = jac * (zj1 * xk1 - xj1 * zk1);
  a[2] = jac * (xj1 * yk1 - yj1 * xk1);
  a[3] = jac * (yk1 * zi1 - zk1 * yi1);
  a[4] = jac * (zk1 * xi1 - xk1 * zi1);
  a[5] = jac * (xk1 * yi1 - yk1 * xi1);
  a[6] = jac * (yi1 * zj1 - zi1 * yj1);
  a[7] = jac * (zi1 * xj1 - xi1 * zj1);
  a[8] = jac * (xi1 * yj1 - yi1 * xj1);
}
template <bool SEP>
__device__ __forceinline__ void metric_dir(const Geo& g, int dir, int i, int j, int k, int q, double& A1, double& A2,
                                           double& A3) {
  if (SEP) {
    if (metric_unfilled(i, j, k)) {
      A1 = A2 = A3 = 1.0;
      return;
    }
    double xi, yi, zi, xj, yj, zj, xk, yk, zk;
    bool cross;
    sep_derivs(g, i, j, k, xi, yi, zi, xj, yj, zj, xk, yk, zk, cross);
    if (!cross) {
#if OCFD_FMA_BUILD
      // (jac (yj zk)) / jac is yj zk up to rounding: the contracted build skips both divisions
      const double d = dir == 0 ? yj * zk : (dir == 1 ? zk * xi : xi * yj);
#else
      double jac = 1.0 / (xi * yj * zk);
      double a = dir == 0 ? jac * (yj * zk) : (dir == 1 ? jac * (zk * xi) : jac * (xi * yj));
      double d = a / jac;
#endif
      A1 = dir == 0 ? d : 0.0;
      A2 = dir == 1 ? d : 0.0;
      A3 = dir == 2 ? d : 0.0;
    } else {
      double a[9], jac;
      jac_full(xi, yi, zi, xj, yj, zj, xk, yk, zk, a, jac);
      A1 = a[3 * dir] / jac;
      A2 = a[3 * dir + 1] / jac;
      A3 = a[3 * dir + 2] / jac;
    }
  } else {
    A1 = __ldg(g.m[G_AKX1 + 3 * dir] + q);
    A2 = __ldg(g.m[G_AKX1 + 3 * dir + 1] + q);
    A3 = __ldg(g.m[G_AKX1 + 3 * dir + 2] + q);
  }
}
template <bool SEP>
__device__ __forceinline__ double metric_jac(const Geo& g, int i, int j, int k, int q) {
  if (SEP) {
    if (metric_unfilled(i, j, k)) return 1.0;
    double xi, yi, zi, xj, yj, zj, xk, yk, zk;
    bool cross;
    sep_derivs(g, i, j, k, xi, yi, zi, xj, yj, zj, xk, yk, zk, cross);
    if (!cross) return 1.0 / (xi * yj * zk);
    double a[9], jac;
    jac_full(xi, yi, zi, xj, yj, zj, xk, yk, zk, a, jac);
    return jac;
  }
  return __ldg(g.m[G_AJAC] + q);
}
// the nine Akx..Asz and the nine Akx1..Asz1 at one point
template <bool SEP>
__device__ __forceinline__ void metric_all(const Geo& g, int i, int j, int k, int q, double* a, double* a1) {
  if (SEP) {
    if (metric_unfilled(i, j, k)) {
#pragma unroll
      for (int m = 0; m < 9; m++) { a[m] = 1.0; a1[m] = 1.0; }
      return;
    }
    double xi, yi, zi, xj, yj, zj, xk, yk, zk;
    bool cross;
    sep_derivs(g, i, j, k, xi, yi, zi, xj, yj, zj, xk, yk, zk, cross);
    if (!cross) {
      double jac = 1.0 / (xi * yj * zk);
      double akx = jac * (yj * zk), aiy = jac * (zk * xi), asz = jac * (xi * yj);
#pragma unroll
      for (int m = 0; m < 9; m++) { a[m] = 0.0; a1[m] = 0.0; }
      a[0] = akx; a[4] = aiy; a[8] = asz;
#if OCFD_FMA_BUILD
      a1[0] = yj * zk; a1[4] = zk * xi; a1[8] = xi * yj;  // akx / jac etc. up to rounding
#else
      a1[0] = akx / jac; a1[4] = aiy / jac; a1[8] = asz / jac;
#endif
    } else {
      double jac;
      jac_full(xi, yi, zi, xj, yj, zj, xk, yk, zk, a, jac);
#pragma unroll
      for (int m = 0; m < 9; m++) a1[m] = a[m] / jac;
    }
  } else {
#pragma unroll
    for (int m = 0; m < 9; m++) {
      a[m] = __ldg(g.m[m] + q);
      a1[m] = __ldg(g.m[G_AKX1 + m] + q);
    }
  }
}

// ---------------------------------------------------------------- thermodynamics (CHEM_thermdyn.f90)
__device__ __forceinline__ int trange(double T) {
  int jc = 0;
  for (int j = 0; j < cC.n_tct - 1; j++)
    if (T > cC.tct[j]) jc = j + 1;
  return jc;
}
template <int NS>
__device__ __forceinline__ double dev_E(const double* di, double T) {
  if (cC.realgas == 0) {
    double e = 0.0;
#pragma unroll
    for (int k = 0; k < NS; k++) e = e + 2.5 * cC.Ri[k] * di[k] * T;
    return e;
  }
  int jc = trange(T);
  double A1 = 0, B1 = 0, C1 = 0, D1 = 0, E1 = 0, Ec = 0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    const double* c = cC.cf[k][jc];
    double R1 = cC.Ri[k];
    A1 = A1 + (c[0] - 1.0) * R1 * di[k];
    B1 = B1 + c[1] * R1 * di[k];
    C1 = C1 + c[2] * R1 * di[k];
    D1 = D1 + c[3] * R1 * di[k];
    E1 = E1 + c[4] * R1 * di[k];
    Ec = Ec + c[7] * R1 * di[k];
  }
  if (T <= cC.tct_max) return A1 * T + B1 * q2(T) / 2.0 + divc<3>(C1 * q3(T)) + D1 * q4(T) / 4.0 + divc<5>(E1 * q5(T)) + Ec;
  double tm = cC.tct_max;
  double cv2 = A1 + B1 * tm + C1 * q2(tm) + D1 * q3(tm) + E1 * q4(tm);
  return A1 * tm + B1 * q2(tm) / 2.0 + divc<3>(C1 * q3(tm)) + D1 * q4(tm) / 4.0 + divc<5>(E1 * q5(tm)) + Ec + cv2 * (T - tm);
}
template <int NS>
__device__ __forceinline__ double dev_Cp(double d, const double* di, double T) {
  if (cC.realgas == 0) {
    double cp = 0.0;
#pragma unroll
    for (int k = 0; k < NS; k++) cp = cp + 3.5 * cC.Ri[k] * di[k];
    return cp / d;
  }
  int jc = trange(T);
  double A1 = 0, B1 = 0, C1 = 0, D1 = 0, E1 = 0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    const double* c = cC.cf[k][jc];
    double R1 = cC.Ri[k];
    A1 = A1 + c[0] * R1 * di[k];
    B1 = B1 + c[1] * R1 * di[k];
    C1 = C1 + c[2] * R1 * di[k];
    D1 = D1 + c[3] * R1 * di[k];
    E1 = E1 + c[4] * R1 * di[k];
  }
  double t = T <= cC.tct_max ? T : cC.tct_max;
  return (A1 + B1 * t + C1 * q2(t) + D1 * q3(t) + E1 * q4(t)) / d;
}
// the six energy sums of comput_T_rgas for fit range j (CHEM_thermdyn.f90:333-345), species in
// order, so a range's sums are the same numbers whenever they are formed
template <int NS>
__device__ __forceinline__ void e_sums(const double* di, int j, double& a, double& b, double& c, double& d, double& e,
                                       double& g) {
  a = 0; b = 0; c = 0; d = 0; e = 0; g = 0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    const double* cf = cC.cf[k][j];
    double R1 = cC.Ri[k];
    a = a + (cf[0] - 1.0) * R1 * di[k];
    b = b + cf[1] * R1 * di[k];
    c = c + cf[2] * R1 * di[k];
    d = d + cf[3] * R1 * di[k];
    e = e + cf[4] * R1 * di[k];
    g = g + cf[7] * R1 * di[k];
  }
}
// T from internal energy; Newton (tol 1e-3 K, at most 31 iterations) for the fitted gas. The
// reference forms the sums of every fit range first; here the sums of the range the iterate is
// in are formed when it changes (the same values), so nothing is indexed at run time.
template <int NS>
__device__ __forceinline__ double dev_T(const double* di, double Ein, int* nfail) {
  if (cC.realgas == 0) {
    double rcv = 0.0;
#pragma unroll
    for (int k = 0; k < NS; k++) rcv = rcv + 2.5 * cC.Ri[k] * di[k];
    return Ein / rcv;
  }
  double A1, B1, C1, D1, E1, Ec;
  e_sums<NS>(di, 0, A1, B1, C1, D1, E1, Ec);
  int jcur = 0;
  double T1 = Ein / A1, T2 = T1;
  int ks = 0;
  bool conv = false;
  while (ks <= 30) {
    int jc = trange(T1);
    if (jc != jcur) {
      e_sums<NS>(di, jc, A1, B1, C1, D1, E1, Ec);
      jcur = jc;
    }
    double Et1, Ex;
    if (T1 <= cC.tct_max) {
      Et1 = A1 * T1 + B1 * q2(T1) / 2.0 + divc<3>(C1 * q3(T1)) + D1 * q4(T1) / 4.0 + divc<5>(E1 * q5(T1)) + Ec;
      Ex = A1 + B1 * T1 + C1 * q2(T1) + D1 * q3(T1) + E1 * q4(T1);
    } else {
      double tm = cC.tct_max;
      Ex = A1 + B1 * tm + C1 * q2(tm) + D1 * q3(tm) + E1 * q4(tm);
      Et1 = A1 * tm + B1 * q2(tm) / 2.0 + divc<3>(C1 * q3(tm)) + D1 * q4(tm) / 4.0 + divc<5>(E1 * q5(tm)) + Ec +
            Ex * (T1 - tm);
    }
    T2 = T1 - (Et1 - Ein) / Ex;
    ks = ks + 1;
    double err = fabs(T2 - T1);
    T1 = T2;
    if (err < 1.0e-3) { conv = true; break; }
  }
  if (!conv && nfail) atomicAdd(nfail, 1);
  return T2;
}
template <int NS>
__device__ __forceinline__ double dev_P(const double* di, double T) {
  double p = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) p = p + cC.Ri[k] * di[k] * T;
  return p;
}
template <int NS>
__device__ __forceinline__ double dev_dens(const double* ai, double T, double p) {
  double r1 = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) r1 = r1 + cC.Ri[k] * ai[k];
  return p / (T * r1);
}
__device__ __forceinline__ double dev_hi(int k, double T) {
  if (cC.realgas == 0) return 3.5 * cC.Ri[k] * T;
  int jc = trange(T);
  const double* c = cC.cf[k][jc];
  if (T <= cC.tct_max)
    return (c[0] * T + c[1] * q2(T) / 2.0 + divc<3>(c[2] * q3(T)) + c[3] * q4(T) / 4.0 + divc<5>(c[4] * q5(T)) + c[7]) *
           cC.Ri[k];
  double tm = cC.tct_max;
  double cpm = c[0] + c[1] * tm + c[2] * q2(tm) + c[3] * q3(tm) + c[4] * q4(tm);
  return (c[0] * tm + c[1] * q2(tm) / 2.0 + divc<3>(c[2] * q3(tm)) + c[3] * q4(tm) / 4.0 + divc<5>(c[4] * q5(tm)) + c[7] +
          cpm * (T - tm)) *
         cC.Ri[k];
}
// comput_gibbs (CHEM_thermdyn.f90:296-319) of species k in fit range jc = trange(T)
__device__ __forceinline__ double dev_gibbs_jc(int k, int jc, double T, double logT) {
  const double* c = cC.cf[k][jc];
  if (T <= cC.tct_max)
    return c[0] * (1.0 - logT) * T - c[1] * q2(T) / 2.0 - divc<6>(c[2] * q3(T)) - divc<12>(c[3] * q4(T)) -
           divc<20>(c[4] * q5(T)) + c[5] - c[6] * T;
  double tm = cC.tct_max;
  double cpm = c[0] + c[1] * tm + c[2] * q2(tm) + c[3] * q3(tm) + c[4] * q4(tm);
  double hm = c[0] * tm + c[1] * q2(tm) / 2.0 + divc<3>(c[2] * q3(tm)) + c[3] * q4(tm) / 4.0 + divc<5>(c[4] * q5(tm)) + c[5];
  double sm = c[0] * log(tm) + c[1] * tm + c[2] * q2(tm) / 2.0 + divc<3>(c[3] * q3(tm)) + c[4] * q4(tm) / 4.0 + c[6];
  return hm + cpm * (T - tm) - T * (sm + cpm * log(T / tm));
}
__device__ __forceinline__ double dev_gibbs(int k, double T, double logT) { return dev_gibbs_jc(k, trange(T), T, logT); }

// ---------------------------------------------------------------- transport (TRANSPORT_modules.f90)
template <int NS>
__device__ __forceinline__ double dev_viscosity(double T, const double* Xi) {
  if (cC.flag_vis == 0) {
    const double TA = 288.15, TC = 110.4;
    return cC.amu0 * sqrt(q3(T / TA)) * (TA + TC) / (TC + T);
  }
  double L = log(T);
  double mui[NS];
#pragma unroll
  for (int m = 0; m < NS; m++)
    mui[m] = exp(cC.mu_an[m][0] + cC.mu_an[m][1] * L + cC.mu_an[m][2] * q2(L) + cC.mu_an[m][3] * q3(L)) * 0.1;
  double mu = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double pk0 = 0.0;
#pragma unroll
    for (int j = 0; j < NS; j++) {
      double s = 1.0 + sqrt(mui[k] / mui[j] * cC.wk_a[k][j]);
      double pkj = q2(s) / cC.wk_b[k][j];
      pk0 = pk0 + Xi[j] * pkj;
    }
    mu = mu + Xi[k] * mui[k] / pk0;
  }
  return mu;
}
template <int NS>
__device__ __forceinline__ double dev_conductivity(double amu, double cp, double T, const double* Xi) {
  if (cC.flag_cond == 0) return amu * cp / cC.pr;
  double L = log(T);
  double a1 = 0.0, a2 = 0.0;
#pragma unroll
  for (int m = 0; m < NS; m++) {
    double ki = exp(cC.k_an[m][0] + cC.k_an[m][1] * L + cC.k_an[m][2] * q2(L) + cC.k_an[m][3] * q3(L)) * 1.0e-5;
    a1 = a1 + Xi[m] * ki;
    a2 = a2 + Xi[m] / ki;
  }
  return 0.5 * (a1 + 1.0 / a2);
}
template <int NS>
__device__ __forceinline__ void dev_diffusion(double* amd, double amu, double T, double d, double p, const double* Xi) {
  if (cC.flag_diff == 0) {
    double d0 = 0.0;
#pragma unroll
    for (int m = 0; m < NS; m++) d0 = d0 + Xi[m] * cC.Mi[m];
#pragma unroll
    for (int m = 0; m < NS; m++) amd[m] = amu * (1.0 - Xi[m] * cC.Mi[m] / d0) / ((1.0 - Xi[m]) * cC.sc * d + 1.0e-20);
    return;
  }
  double L = log(T);
  // D2(k,j) = D2(min,max) (the reference fills the table symmetrically), so each pair is
  // evaluated once; walking the pairs (a < b) a-major adds to ds(k) the terms j = 0..k-1 and then
  // j = k+1..NS-1, the reference's order for every k
  double ds[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) ds[k] = 0.0;
#pragma unroll
  for (int a = 0; a < NS; a++)
#pragma unroll
    for (int b = a + 1; b < NS; b++) {
      double D2 = exp(cC.d_an[a][b][0] + cC.d_an[a][b][1] * L + cC.d_an[a][b][2] * q2(L) + cC.d_an[a][b][3] * q3(L)) *
                  1.0e-4;
      ds[a] = ds[a] + Xi[b] / D2;
      ds[b] = ds[b] + Xi[a] / D2;
    }
#pragma unroll
  for (int k = 0; k < NS; k++) amd[k] = (1.0 - Xi[k]) / (ds[k] + 1.0e-20) * 1.013e5 / p;
}

// ---------------------------------------------------------------- reconstructions
#if OCFD_FMA_BUILD
// WENO5 nonlinear weights with one division instead of four (contracted build only): the weights
// a_k = C_k / t_k, t_k = (ep + S_k)^2, and their sum are all multiplied by t0 t1 t2, which leaves
// the normalised weights unchanged and differs from the reference's operation order by rounding
// only. With ep = 1e-6 every t_k >= 1e-12, and the products stay in range while the split fluxes
// are below about 1e30 in magnitude.
__device__ __forceinline__ double weno5_fold(double C03, double C13, double C23, double t0, double t1, double t2,
                                             double q0, double q1, double q2_) {
  const double b0 = C03 * (t1 * t2), b1 = C13 * (t0 * t2), b2 = C23 * (t0 * t1);
  return (b0 * q0 + b1 * q1 + b2 * q2_) / (b0 + b1 + b2);
}
#endif
// single interface; v points at the stencil centre v(i) (OCFD_Schemes.f90 / OCFD_Schemes_1.f90).
// VS is the element stride of v (1 when v is contiguous, the line count in shared memory otherwise).
// 13/12 (a - 2 b + c)^2, the second-difference part of a WENO5 smoothness indicator: sub-stencils
// of neighbouring interfaces with the same centre share it (the same expression on the same values)
__device__ __forceinline__ double w5d(double a, double b, double c) { return 13.0 / 12.0 * q2(a - 2.0 * b + c); }
// WENO5 flux+ from its five values and the second-difference terms of its three sub-stencils
// (D0 centred on v1, D1 on v0, D2 on vm1)
__device__ __forceinline__ double weno5P_v(double vm2, double vm1, double v0, double v1, double v2, double D0,
                                           double D1, double D2) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double S0 = D0 + 1.0 / 4.0 * q2(3.0 * v0 - 4.0 * v1 + v2);
  double S1 = D1 + 1.0 / 4.0 * q2(vm1 - v1);
  double S2 = D2 + 1.0 / 4.0 * q2(vm2 - 4.0 * vm1 + 3.0 * v0);
  double q03 = 1.0 / 3.0 * v0 + 5.0 / 6.0 * v1 - 1.0 / 6.0 * v2;
  double q13 = -(1.0 / 6.0 * vm1) + 5.0 / 6.0 * v0 + 1.0 / 3.0 * v1;
  double q23 = 1.0 / 3.0 * vm2 - 7.0 / 6.0 * vm1 + 11.0 / 6.0 * v0;
#if OCFD_FMA_BUILD
  return weno5_fold(C03, C13, C23, q2(ep + S0), q2(ep + S1), q2(ep + S2), q03, q13, q23);
#else
  double a0 = C03 / q2(ep + S0);
  double a1 = C13 / q2(ep + S1);
  double a2 = C23 / q2(ep + S2);
  double am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
#endif
}
// WENO5 flux- from its five values and the second-difference terms (D0 centred on v0, D1 on v1,
// D2 on v2)
__device__ __forceinline__ double weno5M_v(double vm1, double v0, double v1, double v2, double v3, double D0,
                                           double D1, double D2) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double S0 = D0 + 1.0 / 4.0 * q2(3.0 * v1 - 4.0 * v0 + vm1);
  double S1 = D1 + 1.0 / 4.0 * q2(v2 - v0);
  double S2 = D2 + 1.0 / 4.0 * q2(v3 - 4.0 * v2 + 3.0 * v1);
  double q03 = 1.0 / 3.0 * v1 + 5.0 / 6.0 * v0 - 1.0 / 6.0 * vm1;
  double q13 = -(1.0 / 6.0 * v2) + 5.0 / 6.0 * v1 + 1.0 / 3.0 * v0;
  double q23 = 1.0 / 3.0 * v3 - 7.0 / 6.0 * v2 + 11.0 / 6.0 * v1;
#if OCFD_FMA_BUILD
  return weno5_fold(C03, C13, C23, q2(ep + S0), q2(ep + S1), q2(ep + S2), q03, q13, q23);
#else
  double a0 = C03 / q2(ep + S0);
  double a1 = C13 / q2(ep + S1);
  double a2 = C23 / q2(ep + S2);
  double am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
#endif
}
template <int VS>
__device__ __forceinline__ double weno5P(const double* v) {
  const double vm2 = v[-2 * VS], vm1 = v[-VS], v0 = v[0], v1 = v[VS], v2 = v[2 * VS];
  return weno5P_v(vm2, vm1, v0, v1, v2, w5d(v0, v1, v2), w5d(vm1, v0, v1), w5d(vm2, vm1, v0));
}
template <int VS>
__device__ __forceinline__ double weno5M(const double* v) {
  const double vm1 = v[-VS], v0 = v[0], v1 = v[VS], v2 = v[2 * VS], v3 = v[3 * VS];
  return weno5M_v(vm1, v0, v1, v2, v3, w5d(v1, v0, vm1), w5d(v2, v1, v0), w5d(v3, v2, v1));
}
// WENO5 with the out-of-domain sub-stencil removed; del 1 = left, 2 = right (DEL_LIFT / DEL_RIGHT)
template <int VS>
__device__ __forceinline__ double weno5P_bnd(const double* v, int del) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  const double vm2 = v[-2 * VS], vm1 = v[-VS], v0 = v[0], v1 = v[VS], v2 = v[2 * VS];
  double a0 = 0.0, q03 = 0.0, a2 = 0.0, q23 = 0.0;
  if (del != 2) {
    double S0 = 13.0 / 12.0 * q2(v0 - 2.0 * v1 + v2) + 1.0 / 4.0 * q2(3.0 * v0 - 4.0 * v1 + v2);
    a0 = C03 / q2(ep + S0);
    q03 = 1.0 / 3.0 * v0 + 5.0 / 6.0 * v1 - 1.0 / 6.0 * v2;
  }
  double S1 = 13.0 / 12.0 * q2(vm1 - 2.0 * v0 + v1) + 1.0 / 4.0 * q2(vm1 - v1);
  double a1 = C13 / q2(ep + S1);
  double q13 = -(1.0 / 6.0 * vm1) + 5.0 / 6.0 * v0 + 1.0 / 3.0 * v1;
  if (del != 1) {
    double S2 = 13.0 / 12.0 * q2(vm2 - 2.0 * vm1 + v0) + 1.0 / 4.0 * q2(vm2 - 4.0 * vm1 + 3.0 * v0);
    a2 = C23 / q2(ep + S2);
    q23 = 1.0 / 3.0 * vm2 - 7.0 / 6.0 * vm1 + 11.0 / 6.0 * v0;
  }
  double am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}
template <int VS>
__device__ __forceinline__ double weno5M_bnd(const double* v, int del) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  const double vm1 = v[-VS], v0 = v[0], v1 = v[VS], v2 = v[2 * VS], v3 = v[3 * VS];
  double a0 = 0.0, q03 = 0.0, a2 = 0.0, q23 = 0.0;
  if (del != 1) {
    double S0 = 13.0 / 12.0 * q2(v1 - 2.0 * v0 + vm1) + 1.0 / 4.0 * q2(3.0 * v1 - 4.0 * v0 + vm1);
    a0 = C03 / q2(ep + S0);
    q03 = 1.0 / 3.0 * v1 + 5.0 / 6.0 * v0 - 1.0 / 6.0 * vm1;
  }
  double S1 = 13.0 / 12.0 * q2(v2 - 2.0 * v1 + v0) + 1.0 / 4.0 * q2(v2 - v0);
  double a1 = C13 / q2(ep + S1);
  double q13 = -(1.0 / 6.0 * v2) + 5.0 / 6.0 * v1 + 1.0 / 3.0 * v0;
  if (del != 2) {
    double S2 = 13.0 / 12.0 * q2(v3 - 2.0 * v2 + v1) + 1.0 / 4.0 * q2(v3 - 4.0 * v2 + 3.0 * v1);
    a2 = C23 / q2(ep + S2);
    q23 = 1.0 / 3.0 * v3 - 7.0 / 6.0 * v2 + 11.0 / 6.0 * v1;
  }
  double am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}

// WENO7-JS (Balsara-Shu smoothness), OCFD_Schemes.f90:59-197
#define W7C                                                                                                  \
  const double C0 = 1.0 / 35.0, C1 = 12.0 / 35.0, C2 = 18.0 / 35.0, C3 = 4.0 / 35.0;                       \
  const double a11 = -2.0 / 6.0, a12 = 9.0 / 6.0, a13 = -18.0 / 6.0, a14 = 11.0 / 6.0;                      \
  const double a21 = 1.0 / 6.0, a23 = 3.0 / 6.0, a24 = 2.0 / 6.0;                                          \
  const double a31 = -2.0 / 6.0, a32 = -3.0 / 6.0, a34 = -1.0 / 6.0;                                       \
  const double a41 = -11.0 / 6.0, a42 = 18.0 / 6.0, a43 = -9.0 / 6.0, a44 = 2.0 / 6.0;                      \
  const double b12 = 4.0, b13 = -5.0, b14 = 2.0, b22 = -2.0, b41 = 2.0, b42 = -5.0, b43 = 4.0, c12 = 3.0;   \
  const double d12 = 13.0 / 12.0, d13 = 1043.0 / 960.0, d14 = 1.0 / 12.0;                                   \
  const double e11 = -3.0 / 12.0, e12 = 13.0 / 12.0, e13 = -23.0 / 12.0, e14 = 25.0 / 12.0;                 \
  const double e21 = 1.0 / 12.0, e22 = -5.0 / 12.0, e23 = 13.0 / 12.0, e24 = 3.0 / 12.0;                    \
  const double e31 = -1.0 / 12.0, e32 = 7.0 / 12.0, e33 = 7.0 / 12.0, e34 = -1.0 / 12.0;                    \
  const double e41 = 3.0 / 12.0, e42 = 13.0 / 12.0, e43 = -5.0 / 12.0, e44 = 1.0 / 12.0;                    \
  const double ep = 1.0e-8;

// generic WENO7 on seven values w0..w6 ordered upwind -> downwind (P: v(i-3..i+3); M: v(i+4..i-2))
__device__ __forceinline__ double weno7_core(double w0, double w1, double w2, double w3, double w4, double w5,
                                             double w6) {
  W7C
  double S10 = a11 * w0 + a12 * w1 + a13 * w2 + a14 * w3;
  double S11 = a21 * w1 - w2 + a23 * w3 + a24 * w4;
  double S12 = a31 * w2 + a32 * w3 + w4 + a34 * w5;
  double S13 = a41 * w3 + a42 * w4 + a43 * w5 + a44 * w6;
  double S20 = -w0 + b12 * w1 + b13 * w2 + b14 * w3;
  double S21 = w2 + b22 * w3 + w4;
  double S22 = w3 + b22 * w4 + w5;
  double S23 = b41 * w3 + b42 * w4 + b43 * w5 - w6;
  double S30 = -w0 + c12 * (w1 - w2) + w3;
  double S31 = -w1 + c12 * (w2 - w3) + w4;
  double S32 = -w2 + c12 * (w3 - w4) + w5;
  double S33 = -w3 + c12 * (w4 - w5) + w6;
  double S0 = S10 * S10 + d12 * S20 * S20 + d13 * S30 * S30 + d14 * S10 * S30;
  double S1 = S11 * S11 + d12 * S21 * S21 + d13 * S31 * S31 + d14 * S11 * S31;
  double S2 = S12 * S12 + d12 * S22 * S22 + d13 * S32 * S32 + d14 * S12 * S32;
  double S3 = S13 * S13 + d12 * S23 * S23 + d13 * S33 * S33 + d14 * S13 * S33;
  double q0 = e11 * w0 + e12 * w1 + e13 * w2 + e14 * w3;
  double q1 = e21 * w1 + e22 * w2 + e23 * w3 + e24 * w4;
  double q2_ = e31 * w2 + e32 * w3 + e33 * w4 + e34 * w5;
  double q3_ = e41 * w3 + e42 * w4 + e43 * w5 + e44 * w6;
#if OCFD_FMA_BUILD
  // one division: every weight multiplied by the product of the four (ep + S)^2 (in range while
  // the split fluxes are below about 1e20 in magnitude; ep = 1e-8 keeps every factor >= 1e-16)
  const double t0 = q2(ep + S0), t1 = q2(ep + S1), t2 = q2(ep + S2), t3 = q2(ep + S3);
  const double p01 = t0 * t1, p23 = t2 * t3;
  const double b0 = C0 * t1 * p23, b1 = C1 * t0 * p23, b2 = C2 * p01 * t3, b3 = C3 * p01 * t2;
  return (b0 * q0 + b1 * q1 + b2 * q2_ + b3 * q3_) / ((b0 + b1) + (b2 + b3));
#else
  double a0 = C0 / q2(ep + S0);
  double a1 = C1 / q2(ep + S1);
  double a2 = C2 / q2(ep + S2);
  double a3 = C3 / q2(ep + S3);
  double am = a0 + a1 + a2 + a3;
  return (a0 * q0 + a1 * q1 + a2 * q2_ + a3 * q3_) / am;
#endif
}
template <int VS>
__device__ __forceinline__ double weno7P(const double* v) {
  return weno7_core(v[-3 * VS], v[-2 * VS], v[-VS], v[0], v[VS], v[2 * VS], v[3 * VS]);
}
template <int VS>
__device__ __forceinline__ double weno7M(const double* v) {
  return weno7_core(v[4 * VS], v[3 * VS], v[2 * VS], v[VS], v[0], v[-VS], v[-2 * VS]);
}

__device__ __forceinline__ double minmod2(double x1, double x2) {
  return 0.5 * (fsgn(x1) + fsgn(x2)) * fmin(fabs(x1), fabs(x2));
}
__device__ __forceinline__ double minmod4(double x1, double x2, double x3, double x4) {
  double m = 0.5 * (fsgn(x1) + fsgn(x2));
  m = m * fabs(0.5 * (fsgn(x1) + fsgn(x3)));
  m = m * fabs(0.5 * (fsgn(x1) + fsgn(x4)));
  m = m * fmin(fmin(fmin(fabs(x1), fabs(x2)), fabs(x3)), fabs(x4));
  return m;
}
// OMP6 (Leng & Li 2013) on eight values w0..w7 ordered upwind -> downwind:
// P: v(i-3..i+4), M: v(i+4..i-3). The reference's flux- limiter is not the mirror image of the
// flux+ one in one term: its lc uses 0.5*(v(i+1)-v(i)) (OCFD_Schemes.f90:270), i.e. w3-w4,
// where flux+ uses 0.5*(v(i)-v(i-1)) = w3-w2 (OCFD_Schemes.f90:233). PLUS selects which.
template <bool PLUS>
__device__ __forceinline__ double omp6_core(double w0, double w1, double w2, double w3, double w4, double w5,
                                            double w6, double w7) {
  const double m_ = 0.015, n_ = 0.0;
  const double a = 0.5 * (m_ + n_), b = 0.5 * (m_ - n_);
  const double o1 = a, o2 = 1.0 / 60.0 - b - 6.0 * a, o3 = -2.0 / 15.0 + 6.0 * b + 15.0 * a,
               o4 = 37.0 / 60.0 - 15.0 * b - 20.0 * a, o5 = 37.0 / 60.0 + 20.0 * b + 15.0 * a,
               o6 = -2.0 / 15.0 - 6.0 * a - 15.0 * b, o7 = 1.0 / 60.0 + a + 6.0 * b, o8 = -b;
  const double kappa = 4.0, ep = (double)1.0e-10f;
  // reference P: a1*v(i+4)+a2*v(i+3)+...+a8*v(i-3)
  double mid = o1 * w7 + o2 * w6 + o3 * w5 + o4 * w4 + o5 * w3 + o6 * w2 + o7 * w1 + o8 * w0;
  double mp = w3 + minmod2(w4 - w3, kappa * (w3 - w2));
  if ((mid - w3) * (mid - mp) >= ep) {
    double d1 = w1 + w3 - 2.0 * w2;
    double d2 = w2 + w4 - 2.0 * w3;
    double d3 = w3 + w5 - 2.0 * w4;
    double ul = w3 + kappa * (w3 - w2);
    double md = 0.5 * (w3 + w4) - 0.5 * minmod4(4.0 * d2 - d3, 4.0 * d3 - d2, d2, d3);
    double lc = w3 + 0.5 * (PLUS ? (w3 - w2) : (w3 - w4)) + kappa * minmod4(4.0 * d1 - d2, 4.0 * d2 - d1, d2, d1) / 3.0;
    double fmn = fmax(fmin(fmin(w3, w4), md), fmin(fmin(w3, ul), lc));
    double fmx = fmin(fmax(fmax(w3, w4), md), fmax(fmax(w3, ul), lc));
    mid = mid + minmod2(fmx - mid, fmn - mid);
  }
  return mid;
}
template <int VS>
__device__ __forceinline__ double omp6P(const double* v) {
  return omp6_core<true>(v[-3 * VS], v[-2 * VS], v[-VS], v[0], v[VS], v[2 * VS], v[3 * VS], v[4 * VS]);
}
template <int VS>
__device__ __forceinline__ double omp6M(const double* v) {
  return omp6_core<false>(v[4 * VS], v[3 * VS], v[2 * VS], v[VS], v[0], v[-VS], v[-2 * VS], v[-3 * VS]);
}
template <int VS>
__device__ __forceinline__ double ud7lP(const double* v) {
  const double* U = cC.UD7L;
  return U[0] * v[-3 * VS] + U[1] * v[-2 * VS] + U[2] * v[-VS] + U[3] * v[0] + U[4] * v[VS] + U[5] * v[2 * VS] +
         U[6] * v[3 * VS] + U[7] * v[4 * VS];
}
template <int VS>
__device__ __forceinline__ double ud7lM(const double* v) {
  const double* U = cC.UD7L;
  return U[0] * v[4 * VS] + U[1] * v[3 * VS] + U[2] * v[2 * VS] + U[3] * v[VS] + U[4] * v[0] + U[5] * v[-VS] +
         U[6] * v[-2 * VS] + U[7] * v[-3 * VS];
}

__device__ __forceinline__ int hybrid_index(double R0) {
  if (R0 <= cC.theta1) return 1;
  if (R0 <= cC.theta2) return 2;
  return 3;
}

// Numerical flux at interface i (0..n) of a pencil of length n in direction dir, for the
// positive (PLUS) or negative split flux, including the boundary closures of OCFD2d_flux1/2
// (OCFD_inviscous.f90:209-362). v points at v(i).
template <int SCHEME, bool PLUS, int VS>
__device__ __forceinline__ double interface_flux(const double* v, int i, int n, int dir, int scm) {
  const int Ka = PLUS ? cC.Ka1 : cC.Ka2, Kb = PLUS ? cC.Kb1 : cC.Kb2;
  const int b0 = cC.bound[dir][0], b1 = cC.bound[dir][1];
  const int s0 = cC.sb[2 * dir], s1 = cC.sb[2 * dir + 1];
  if (b0 == 1 && i <= -Ka && s0 != -1) {
    if (s0 == 0) {
      if (PLUS) {
        if (i <= 1) {  // (2 f(1) + 5 f(2) - f(3)) / 6 at i = 0 and 1
          const double* f1 = v + (1 - i) * VS;
          return (2.0 * f1[0] + 5.0 * f1[VS] - f1[2 * VS]) / 6.0;
        }
        if (i == 2) return weno5P_bnd<VS>(v, 1);
        return weno5P<VS>(v);
      } else {
        if (i == 0) return (2.0 * v[3 * VS] - 7.0 * v[2 * VS] + 11.0 * v[VS]) / 6.0;
        if (i == 1) return weno5M_bnd<VS>(v, 1);
        return weno5M<VS>(v);
      }
    }
    return PLUS ? weno5P<VS>(v) : weno5M<VS>(v);
  }
  if (b1 == 1 && i >= n - Kb + 1 && s1 != -1) {
    if (s1 == 0) {
      if (PLUS) {
        if (i == n) return (2.0 * v[-2 * VS] - 7.0 * v[-VS] + 11.0 * v[0]) / 6.0;
        if (i == n - 1) return weno5P_bnd<VS>(v, 2);
        return weno5P<VS>(v);
      } else {
        if (i >= n - 1) {  // (2 f(n) + 5 f(n-1) - f(n-2)) / 6 at i = n-1 and n
          const double* fn = v + (n - i) * VS;
          return (2.0 * fn[0] + 5.0 * fn[-VS] - fn[-2 * VS]) / 6.0;
        }
        if (i == n - 2) return weno5M_bnd<VS>(v, 2);
        return weno5M<VS>(v);
      }
    }
    return PLUS ? weno5P<VS>(v) : weno5M<VS>(v);
  }
  if (SCHEME == OCFD_SCHEME_WENO5) return PLUS ? weno5P<VS>(v) : weno5M<VS>(v);
  if (SCHEME == OCFD_SCHEME_WENO7) return PLUS ? weno7P<VS>(v) : weno7M<VS>(v);
  if (SCHEME == OCFD_SCHEME_OMP6) return PLUS ? omp6P<VS>(v) : omp6M<VS>(v);
  if (SCHEME == OCFD_SCHEME_UD7L) return PLUS ? ud7lP<VS>(v) : ud7lM<VS>(v);
  // HYBRID
  if (scm == 1) return PLUS ? ud7lP<VS>(v) : ud7lM<VS>(v);
  if (scm == 2) return PLUS ? weno7P<VS>(v) : weno7M<VS>(v);
  return PLUS ? weno5P<VS>(v) : weno5M<VS>(v);
}

}  // namespace ocfd
