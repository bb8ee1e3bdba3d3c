/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle: upwind reconstructions of OpenCFD-Comb restated in
 * C++ (checker for the CUDA kernels, never shipped).
 *
 * Pencil routines follow code/schemes/OCFD_Schemes.f90 (OCFD_weno5P/M :6-53, OCFD_weno7P/M
 * :59-197, OCFD_OMP6P/M :207-278, minmod2/4 :284-299, OCFD_UD7L_P/M :302-326, OCFD_HybridP/M
 * :329-370). Single-interface routines follow code/schemes/OCFD_Schemes_1.f90 (hh_weno5P/M
 * :9-54, hh_weno7P/M :60-194, hh_weno5P/M_boundary :279-338). Boundary closures follow
 * OCFD2d_flux1/flux2 (code/flow-solver/OCFD_inviscous.f90:209-362).
 *
 * Pointers are offset so that v[i] is the reference's v(i) and hh[i] is hh(i).
 */
#pragma once
#include <cmath>
#include <algorithm>
#include "ocfd_oracle_common.h"

namespace ocfd_oracle {

struct SchemeSet {
  int scheme = 1;    /* OCFD_SCHEME_* */
  int Ka1 = -2, Kb1 = 2, Ka2 = -1, Kb2 = 3;
  double UD7L[8] = {0};
  double theta1 = 1.0, theta2 = 1.0; /* Hybrid_para(2), Hybrid_para(3) */
};

/* ---- single interface, v points at v(0) == v(j) ---- */
inline double hh_weno5P(const double* v) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double S0 = 13.0 / 12.0 * p2(v[0] - 2.0 * v[1] + v[2]) + 1.0 / 4.0 * p2(3.0 * v[0] - 4.0 * v[1] + v[2]);
  double S1 = 13.0 / 12.0 * p2(v[-1] - 2.0 * v[0] + v[1]) + 1.0 / 4.0 * p2(v[-1] - v[1]);
  double S2 = 13.0 / 12.0 * p2(v[-2] - 2.0 * v[-1] + v[0]) + 1.0 / 4.0 * p2(v[-2] - 4.0 * v[-1] + 3.0 * v[0]);
  double a0 = C03 / p2(ep + S0);
  double a1 = C13 / p2(ep + S1);
  double a2 = C23 / p2(ep + S2);
  double am = a0 + a1 + a2;
  double q03 = 1.0 / 3.0 * v[0] + 5.0 / 6.0 * v[1] - 1.0 / 6.0 * v[2];
  double q13 = -(1.0 / 6.0 * v[-1]) + 5.0 / 6.0 * v[0] + 1.0 / 3.0 * v[1];
  double q23 = 1.0 / 3.0 * v[-2] - 7.0 / 6.0 * v[-1] + 11.0 / 6.0 * v[0];
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}
inline double hh_weno5M(const double* v) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double S0 = 13.0 / 12.0 * p2(v[1] - 2.0 * v[0] + v[-1]) + 1.0 / 4.0 * p2(3.0 * v[1] - 4.0 * v[0] + v[-1]);
  double S1 = 13.0 / 12.0 * p2(v[2] - 2.0 * v[1] + v[0]) + 1.0 / 4.0 * p2(v[2] - v[0]);
  double S2 = 13.0 / 12.0 * p2(v[3] - 2.0 * v[2] + v[1]) + 1.0 / 4.0 * p2(v[3] - 4.0 * v[2] + 3.0 * v[1]);
  double a0 = C03 / p2(ep + S0);
  double a1 = C13 / p2(ep + S1);
  double a2 = C23 / p2(ep + S2);
  double am = a0 + a1 + a2;
  double q03 = 1.0 / 3.0 * v[1] + 5.0 / 6.0 * v[0] - 1.0 / 6.0 * v[-1];
  double q13 = -(1.0 / 6.0 * v[2]) + 5.0 / 6.0 * v[1] + 1.0 / 3.0 * v[0];
  double q23 = 1.0 / 3.0 * v[3] - 7.0 / 6.0 * v[2] + 11.0 / 6.0 * v[1];
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}

/* WENO5 with one sub-stencil deleted (hh_weno5P_boundary / hh_weno5M_boundary);
 * del = 1 (DEL_LIFT) or 2 (DEL_RIGHT) */
inline double hh_weno5P_bnd(const double* v, int del) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double a0 = 0.0, q03 = 0.0, a2 = 0.0, q23 = 0.0;
  if (del != 2) {
    double S0 = 13.0 / 12.0 * p2(v[0] - 2.0 * v[1] + v[2]) + 1.0 / 4.0 * p2(3.0 * v[0] - 4.0 * v[1] + v[2]);
    a0 = C03 / p2(ep + S0);
    q03 = 1.0 / 3.0 * v[0] + 5.0 / 6.0 * v[1] - 1.0 / 6.0 * v[2];
  }
  double S1 = 13.0 / 12.0 * p2(v[-1] - 2.0 * v[0] + v[1]) + 1.0 / 4.0 * p2(v[-1] - v[1]);
  double a1 = C13 / p2(ep + S1);
  double q13 = -(1.0 / 6.0 * v[-1]) + 5.0 / 6.0 * v[0] + 1.0 / 3.0 * v[1];
  if (del != 1) {
    double S2 = 13.0 / 12.0 * p2(v[-2] - 2.0 * v[-1] + v[0]) + 1.0 / 4.0 * p2(v[-2] - 4.0 * v[-1] + 3.0 * v[0]);
    a2 = C23 / p2(ep + S2);
    q23 = 1.0 / 3.0 * v[-2] - 7.0 / 6.0 * v[-1] + 11.0 / 6.0 * v[0];
  }
  double am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}
inline double hh_weno5M_bnd(const double* v, int del) {
  const double ep = 1.0e-6, C03 = 3.0 / 10.0, C13 = 3.0 / 5.0, C23 = 1.0 / 10.0;
  double a0 = 0.0, q03 = 0.0, a2 = 0.0, q23 = 0.0;
  if (del != 1) {
    double S0 = 13.0 / 12.0 * p2(v[1] - 2.0 * v[0] + v[-1]) + 1.0 / 4.0 * p2(3.0 * v[1] - 4.0 * v[0] + v[-1]);
    a0 = C03 / p2(ep + S0);
    q03 = 1.0 / 3.0 * v[1] + 5.0 / 6.0 * v[0] - 1.0 / 6.0 * v[-1];
  }
  double S1 = 13.0 / 12.0 * p2(v[2] - 2.0 * v[1] + v[0]) + 1.0 / 4.0 * p2(v[2] - v[0]);
  double a1 = C13 / p2(ep + S1);
  double q13 = -(1.0 / 6.0 * v[2]) + 5.0 / 6.0 * v[1] + 1.0 / 3.0 * v[0];
  if (del != 2) {
    double S2 = 13.0 / 12.0 * p2(v[3] - 2.0 * v[2] + v[1]) + 1.0 / 4.0 * p2(v[3] - 4.0 * v[2] + 3.0 * v[1]);
    a2 = C23 / p2(ep + S2);
    q23 = 1.0 / 3.0 * v[3] - 7.0 / 6.0 * v[2] + 11.0 / 6.0 * v[1];
  }
  double am = a0 + a1 + a2;
  return (a0 * q03 + a1 * q13 + a2 * q23) / am;
}

/* WENO7-JS constants (OCFD_Schemes.f90:66-80) */
struct W7 {
  static constexpr double C0 = 1.0 / 35.0, C1 = 12.0 / 35.0, C2 = 18.0 / 35.0, C3 = 4.0 / 35.0;
  static constexpr double a11 = -2.0 / 6.0, a12 = 9.0 / 6.0, a13 = -18.0 / 6.0, a14 = 11.0 / 6.0;
  static constexpr double a21 = 1.0 / 6.0, a23 = 3.0 / 6.0, a24 = 2.0 / 6.0;
  static constexpr double a31 = -2.0 / 6.0, a32 = -3.0 / 6.0, a34 = -1.0 / 6.0;
  static constexpr double a41 = -11.0 / 6.0, a42 = 18.0 / 6.0, a43 = -9.0 / 6.0, a44 = 2.0 / 6.0;
  static constexpr double b12 = 4.0, b13 = -5.0, b14 = 2.0, b22 = -2.0, b41 = 2.0, b42 = -5.0, b43 = 4.0, c12 = 3.0;
  static constexpr double d12 = 13.0 / 12.0, d13 = 1043.0 / 960.0, d14 = 1.0 / 12.0;
  static constexpr double e11 = -3.0 / 12.0, e12 = 13.0 / 12.0, e13 = -23.0 / 12.0, e14 = 25.0 / 12.0;
  static constexpr double e21 = 1.0 / 12.0, e22 = -5.0 / 12.0, e23 = 13.0 / 12.0, e24 = 3.0 / 12.0;
  static constexpr double e31 = -1.0 / 12.0, e32 = 7.0 / 12.0, e33 = 7.0 / 12.0, e34 = -1.0 / 12.0;
  static constexpr double e41 = 3.0 / 12.0, e42 = 13.0 / 12.0, e43 = -5.0 / 12.0, e44 = 1.0 / 12.0;
  static constexpr double ep = 1.0e-8;
};

/* hh_weno7P: v points at v(j); stencil v(-3..3) */
inline double hh_weno7P(const double* v) {
  using W = W7;
  double S10 = W::a11 * v[-3] + W::a12 * v[-2] + W::a13 * v[-1] + W::a14 * v[0];
  double S11 = W::a21 * v[-2] - v[-1] + W::a23 * v[0] + W::a24 * v[1];
  double S12 = W::a31 * v[-1] + W::a32 * v[0] + v[1] + W::a34 * v[2];
  double S13 = W::a41 * v[0] + W::a42 * v[1] + W::a43 * v[2] + W::a44 * v[3];
  double S20 = -v[-3] + W::b12 * v[-2] + W::b13 * v[-1] + W::b14 * v[0];
  double S21 = v[-1] + W::b22 * v[0] + v[1];
  double S22 = v[0] + W::b22 * v[1] + v[2];
  double S23 = W::b41 * v[0] + W::b42 * v[1] + W::b43 * v[2] - v[3];
  double S30 = -v[-3] + W::c12 * (v[-2] - v[-1]) + v[0];
  double S31 = -v[-2] + W::c12 * (v[-1] - v[0]) + v[1];
  double S32 = -v[-1] + W::c12 * (v[0] - v[1]) + v[2];
  double S33 = -v[0] + W::c12 * (v[1] - v[2]) + v[3];
  double S0 = S10 * S10 + W::d12 * S20 * S20 + W::d13 * S30 * S30 + W::d14 * S10 * S30;
  double S1 = S11 * S11 + W::d12 * S21 * S21 + W::d13 * S31 * S31 + W::d14 * S11 * S31;
  double S2 = S12 * S12 + W::d12 * S22 * S22 + W::d13 * S32 * S32 + W::d14 * S12 * S32;
  double S3 = S13 * S13 + W::d12 * S23 * S23 + W::d13 * S33 * S33 + W::d14 * S13 * S33;
  double a0 = W::C0 / p2(W::ep + S0);
  double a1 = W::C1 / p2(W::ep + S1);
  double a2 = W::C2 / p2(W::ep + S2);
  double a3 = W::C3 / p2(W::ep + S3);
  double am = a0 + a1 + a2 + a3;
  double q0 = W::e11 * v[-3] + W::e12 * v[-2] + W::e13 * v[-1] + W::e14 * v[0];
  double q1 = W::e21 * v[-2] + W::e22 * v[-1] + W::e23 * v[0] + W::e24 * v[1];
  double q2 = W::e31 * v[-1] + W::e32 * v[0] + W::e33 * v[1] + W::e34 * v[2];
  double q3 = W::e41 * v[0] + W::e42 * v[1] + W::e43 * v[2] + W::e44 * v[3];
  return (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / am;
}
/* hh_weno7M: v points at v(j); stencil v(-2..4) */
inline double hh_weno7M(const double* v) {
  using W = W7;
  double S10 = W::a11 * v[4] + W::a12 * v[3] + W::a13 * v[2] + W::a14 * v[1];
  double S11 = W::a21 * v[3] - v[2] + W::a23 * v[1] + W::a24 * v[0];
  double S12 = W::a31 * v[2] + W::a32 * v[1] + v[0] + W::a34 * v[-1];
  double S13 = W::a41 * v[1] + W::a42 * v[0] + W::a43 * v[-1] + W::a44 * v[-2];
  double S20 = -v[4] + W::b12 * v[3] + W::b13 * v[2] + W::b14 * v[1];
  double S21 = v[2] + W::b22 * v[1] + v[0];
  double S22 = v[1] + W::b22 * v[0] + v[-1];
  double S23 = W::b41 * v[1] + W::b42 * v[0] + W::b43 * v[-1] - v[-2];
  double S30 = -v[4] + W::c12 * (v[3] - v[2]) + v[1];
  double S31 = -v[3] + W::c12 * (v[2] - v[1]) + v[0];
  double S32 = -v[2] + W::c12 * (v[1] - v[0]) + v[-1];
  double S33 = -v[1] + W::c12 * (v[0] - v[-1]) + v[-2];
  double S0 = S10 * S10 + W::d12 * S20 * S20 + W::d13 * S30 * S30 + W::d14 * S10 * S30;
  double S1 = S11 * S11 + W::d12 * S21 * S21 + W::d13 * S31 * S31 + W::d14 * S11 * S31;
  double S2 = S12 * S12 + W::d12 * S22 * S22 + W::d13 * S32 * S32 + W::d14 * S12 * S32;
  double S3 = S13 * S13 + W::d12 * S23 * S23 + W::d13 * S33 * S33 + W::d14 * S13 * S33;
  double a0 = W::C0 / p2(W::ep + S0);
  double a1 = W::C1 / p2(W::ep + S1);
  double a2 = W::C2 / p2(W::ep + S2);
  double a3 = W::C3 / p2(W::ep + S3);
  double am = a0 + a1 + a2 + a3;
  double q0 = W::e11 * v[4] + W::e12 * v[3] + W::e13 * v[2] + W::e14 * v[1];
  double q1 = W::e21 * v[3] + W::e22 * v[2] + W::e23 * v[1] + W::e24 * v[0];
  double q2 = W::e31 * v[2] + W::e32 * v[1] + W::e33 * v[0] + W::e34 * v[-1];
  double q3 = W::e41 * v[1] + W::e42 * v[0] + W::e43 * v[-1] + W::e44 * v[-2];
  return (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / am;
}

inline double minmod2(double x1, double x2) {
  return 0.5 * (fsign1(x1) + fsign1(x2)) * std::min(std::fabs(x1), std::fabs(x2));
}
inline double minmod4(double x1, double x2, double x3, double x4) {
  double m = 0.5 * (fsign1(x1) + fsign1(x2));
  m = m * std::fabs(0.5 * (fsign1(x1) + fsign1(x3)));
  m = m * std::fabs(0.5 * (fsign1(x1) + fsign1(x4)));
  m = m * std::min(std::min(std::min(std::fabs(x1), std::fabs(x2)), std::fabs(x3)), std::fabs(x4));
  return m;
}

/* OMP6 coefficients (OCFD_Schemes.f90:215-221); ep is the single-precision literal 1.e-10 */
struct OMP {
  double a1, a2, a3, a4, a5, a6, a7, a8, kappa, ep;
  OMP() {
    const double m = 0.015, n = 0.0;
    double a = 0.5 * (m + n), b = 0.5 * (m - n);
    a1 = a;
    a2 = 1.0 / 60.0 - b - 6.0 * a;
    a3 = -2.0 / 15.0 + 6.0 * b + 15.0 * a;
    a4 = 37.0 / 60.0 - 15.0 * b - 20.0 * a;
    a5 = 37.0 / 60.0 + 20.0 * b + 15.0 * a;
    a6 = -2.0 / 15.0 - 6.0 * a - 15.0 * b;
    a7 = 1.0 / 60.0 + a + 6.0 * b;
    a8 = -b;
    kappa = 4.0;
    ep = (double)1.0e-10f;
  }
};

/* OMP6 flux+ at interface i (v points at v(i)) */
inline double omp6P(const OMP& c, const double* v) {
  double mid = c.a1 * v[4] + c.a2 * v[3] + c.a3 * v[2] + c.a4 * v[1] + c.a5 * v[0] + c.a6 * v[-1] + c.a7 * v[-2] +
               c.a8 * v[-3];
  double mp = v[0] + minmod2(v[1] - v[0], c.kappa * (v[0] - v[-1]));
  if ((mid - v[0]) * (mid - mp) >= c.ep) {
    double d1 = v[-2] + v[0] - 2.0 * v[-1];
    double d2 = v[-1] + v[1] - 2.0 * v[0];
    double d3 = v[0] + v[2] - 2.0 * v[1];
    double ul = v[0] + c.kappa * (v[0] - v[-1]);
    double md = 0.5 * (v[0] + v[1]) - 0.5 * minmod4(4.0 * d2 - d3, 4.0 * d3 - d2, d2, d3);
    double lc = v[0] + 0.5 * (v[0] - v[-1]) + c.kappa * minmod4(4.0 * d1 - d2, 4.0 * d2 - d1, d2, d1) / 3.0;
    double fmin = std::max(std::min(std::min(v[0], v[1]), md), std::min(std::min(v[0], ul), lc));
    double fmax = std::min(std::max(std::max(v[0], v[1]), md), std::max(std::max(v[0], ul), lc));
    mid = mid + minmod2(fmax - mid, fmin - mid);
  }
  return mid;
}
/* OMP6 flux- at interface i (v points at v(i)) */
inline double omp6M(const OMP& c, const double* v) {
  double mid = c.a1 * v[-3] + c.a2 * v[-2] + c.a3 * v[-1] + c.a4 * v[0] + c.a5 * v[1] + c.a6 * v[2] + c.a7 * v[3] +
               c.a8 * v[4];
  double mp = v[1] + minmod2(v[0] - v[1], c.kappa * (v[1] - v[2]));
  if ((mid - v[1]) * (mid - mp) >= c.ep) {
    double d1 = v[3] + v[1] - 2.0 * v[2];
    double d2 = v[2] + v[0] - 2.0 * v[1];
    double d3 = v[1] + v[-1] - 2.0 * v[0];
    double ul = v[1] + c.kappa * (v[1] - v[2]);
    double md = 0.5 * (v[1] + v[0]) - 0.5 * minmod4(4.0 * d2 - d3, 4.0 * d3 - d2, d2, d3);
    double lc = v[1] + 0.5 * (v[1] - v[0]) + c.kappa * minmod4(4.0 * d1 - d2, 4.0 * d2 - d1, d2, d1) / 3.0;
    double fmin = std::max(std::min(std::min(v[1], v[0]), md), std::min(std::min(v[1], ul), lc));
    double fmax = std::min(std::max(std::max(v[1], v[0]), md), std::max(std::max(v[1], ul), lc));
    mid = mid + minmod2(fmax - mid, fmin - mid);
  }
  return mid;
}
inline double ud7lP(const double* U, const double* v) {
  return U[0] * v[-3] + U[1] * v[-2] + U[2] * v[-1] + U[3] * v[0] + U[4] * v[1] + U[5] * v[2] + U[6] * v[3] +
         U[7] * v[4];
}
inline double ud7lM(const double* U, const double* v) {
  return U[0] * v[4] + U[1] * v[3] + U[2] * v[2] + U[3] * v[1] + U[4] * v[0] + U[5] * v[-1] + U[6] * v[-2] +
         U[7] * v[-3];
}

/* OCFD2d_flux1 / OCFD2d_flux2 for one pencil: f1d(1-LAP:n+LAP) -> hh(0:n).
 * bnd[2] = Bound_index(1:2) of this direction, sb[2] = Scheme_boundary of its two ends.
 * scm = per-interface hybrid index Scm_Hy(0:n) (used only by HYBRID). */
inline void flux_pencil(bool plus, const SchemeSet& S, const double* v, double* hh, int n, const int bnd[2],
                        const int sb[2], const int* scm) {
  static const OMP omp;
  const int Ka = plus ? S.Ka1 : S.Ka2, Kb = plus ? S.Kb1 : S.Kb2;
  int ib = (bnd[0] == 0 || sb[0] == -1) ? 0 : -Ka + 1;
  int ie = (bnd[1] == 0 || sb[1] == -1) ? n : n - Kb;
  if (plus) {
    for (int i = ib; i <= ie; i++) {
      double h;
      switch (S.scheme) {
        case 3: h = omp6P(omp, v + i); break;
        case 2: h = hh_weno7P(v + i); break;
        case 1: h = hh_weno5P(v + i); break;
        case 4: h = ud7lP(S.UD7L, v + i); break;
        default: /* HYBRID */
          if (scm[i] == 1) h = ud7lP(S.UD7L, v + i);
          else if (scm[i] == 2) h = hh_weno7P(v + i);
          else h = hh_weno5P(v + i);
      }
      hh[i] = h;
    }
  } else {
    for (int i = ib; i <= ie; i++) {
      double h;
      switch (S.scheme) {
        case 3: h = omp6M(omp, v + i); break;
        case 2: h = hh_weno7M(v + i); break;
        case 1: h = hh_weno5M(v + i); break;
        case 4: h = ud7lM(S.UD7L, v + i); break;
        default:
          if (scm[i] == 1) h = ud7lM(S.UD7L, v + i);
          else if (scm[i] == 2) h = hh_weno7M(v + i);
          else h = hh_weno5M(v + i);
      }
      hh[i] = h;
    }
  }
  /* boundary closures */
  if (plus) {
    if (bnd[0] == 1) {
      for (int i = 0; i <= -Ka; i++) {
        if (sb[0] == 0) {
          if (i == 0 || i == 1) hh[i] = (2.0 * v[1] + 5.0 * v[2] - v[3]) / 6.0;
          else if (i == 2) hh[i] = hh_weno5P_bnd(v + i, 1);
          else hh[i] = hh_weno5P(v + i);
        } else if (sb[0] == 1) {
          hh[i] = hh_weno5P(v + i);
        }
      }
    }
    if (bnd[1] == 1) {
      for (int i = n - Kb + 1; i <= n; i++) {
        if (sb[1] == 0) {
          if (i == n) hh[i] = (2.0 * v[n - 2] - 7.0 * v[n - 1] + 11.0 * v[n]) / 6.0;
          else if (i == n - 1) hh[i] = hh_weno5P_bnd(v + i, 2);
          else hh[i] = hh_weno5P(v + i);
        } else if (sb[1] == 1) {
          hh[i] = hh_weno5P(v + i);
        }
      }
    }
  } else {
    if (bnd[0] == 1) {
      for (int i = 0; i <= -Ka; i++) {
        if (sb[0] == 0) {
          if (i == 0) hh[i] = (2.0 * v[3] - 7.0 * v[2] + 11.0 * v[1]) / 6.0;
          else if (i == 1) hh[i] = hh_weno5M_bnd(v + i, 1);
          else hh[i] = hh_weno5M(v + i);
        } else if (sb[0] == 1) {
          hh[i] = hh_weno5M(v + i);
        }
      }
    }
    if (bnd[1] == 1) {
      for (int i = n - Kb + 1; i <= n; i++) {
        if (sb[1] == 0) {
          if (i == n || i == n - 1) hh[i] = (2.0 * v[n] + 5.0 * v[n - 1] - v[n - 2]) / 6.0;
          else if (i == n - 2) hh[i] = hh_weno5M_bnd(v + i, 2);
          else hh[i] = hh_weno5M(v + i);
        } else if (sb[1] == 1) {
          hh[i] = hh_weno5M(v + i);
        }
      }
    }
  }
}

/* One interface i of a pencil of n cells for the characteristic-space flux, following flux_x1
 * (sign +) and flux_x2 (sign -) of OCFD_inviscous_character.f90:321-425: f points at the
 * stencil value of interface i (f[mm] = value at i + mm). Interior points take the scheme (HYBRID
 * by its per-interface index), points near a closed face the WENO5-type boundary schemes. */
inline double iface_flux(bool plus, const SchemeSet& S, const double* f, int i, int n, const int bnd[2],
                         const int sb[2], int scm) {
  static const OMP omp;
  const int Ka = plus ? S.Ka1 : S.Ka2, Kb = plus ? S.Kb1 : S.Kb2;
  const bool inner = (bnd[0] == 0 || i > -Ka || sb[0] == -1) && (bnd[1] == 0 || i <= n - Kb || sb[1] == -1);
  if (inner) {
    int sc = S.scheme;
    if (sc == OCFD_SCHEME_HYBRID) sc = scm == 1 ? 4 : (scm == 2 ? 2 : 1);
    switch (sc) {
      case 3: return plus ? omp6P(omp, f) : omp6M(omp, f);
      case 2: return plus ? hh_weno7P(f) : hh_weno7M(f);
      case 4: return plus ? ud7lP(S.UD7L, f) : ud7lM(S.UD7L, f);
      default: return plus ? hh_weno5P(f) : hh_weno5M(f);
    }
  }
  if (i <= -Ka && bnd[0] == 1 && sb[0] != -1) { /* left face */
    if (sb[0] == 0) {
      if (plus) {
        if (i == 1) return (2.0 * f[0] + 5.0 * f[1] - f[2]) / 6.0;
        if (i == 2) return hh_weno5P_bnd(f, 1);
        return hh_weno5P(f);
      }
      if (i == 1) return hh_weno5M_bnd(f, 1);
      return hh_weno5M(f);
    }
    return plus ? hh_weno5P(f) : hh_weno5M(f); /* Scheme_boundary = 1 */
  }
  /* right face (i > n - Kb, bnd[1] == 1, sb[1] != -1) */
  if (sb[1] == 0) {
    if (plus) {
      if (i == n - 1) return hh_weno5P_bnd(f, 2);
      return hh_weno5P(f);
    }
    if (i == n - 1) return (2.0 * f[1] + 5.0 * f[0] - f[-1]) / 6.0;
    if (i == n - 2) return hh_weno5M_bnd(f, 2);
    return hh_weno5M(f);
  }
  return plus ? hh_weno5P(f) : hh_weno5M(f);
}

}  // namespace ocfd_oracle
