/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle: thermodynamics, transport and finite-rate
 * chemistry of OpenCFD-Comb restated in C++ (checker for the CUDA kernels, never shipped).
 *
 * Follows, routine by routine and in the reference's evaluation order:
 *   code/Chemical/CHEM_thermdyn.f90      (comput_E/Cp/T/hi/P/d, perfect and real gas, Gibbs)
 *   code/Chemical/TRANSPORT_modules.f90  (Sutherland / Wilke viscosity, Pr / Wilke
 *                                         conductivity, Sc / mixture diffusion)
 *   code/Chemical/CHEM_reactions.f90     (Arrhenius, Troe, three-body, Gibbs Kc, Park,
 *                                         Euler / RK2 / RK3 / linearised implicit Euler, Gauss)
 */
#pragma once
#include <cmath>
#include <cstring>
#include "../include/ocfd_gpu.h"
#include "ocfd_oracle_common.h"

namespace ocfd_oracle {

constexpr double R0 = 8.314;     /* CHEM_modules.f90:20 */
constexpr double ATM = 1.013e5;  /* CHEM_modules.f90:22 */

struct Chem {
  int ns = 1, nreac = 0, rereac = 0, n_tct = 1, if_realgas = 0, timeadv = 1;
  double tct[OCFD_NTCT_MAX] = {0}, tct_max = 0;
  double Mi[OCFD_MAX_SPEC] = {0}, Ri[OCFD_MAX_SPEC] = {0};
  int specflag[OCFD_MAX_SPEC] = {0};
  double A[OCFD_MAX_SPEC][OCFD_NTCT_MAX], B[OCFD_MAX_SPEC][OCFD_NTCT_MAX], C[OCFD_MAX_SPEC][OCFD_NTCT_MAX],
      D[OCFD_MAX_SPEC][OCFD_NTCT_MAX], E[OCFD_MAX_SPEC][OCFD_NTCT_MAX], F[OCFD_MAX_SPEC][OCFD_NTCT_MAX],
      G[OCFD_MAX_SPEC][OCFD_NTCT_MAX], Ect[OCFD_MAX_SPEC][OCFD_NTCT_MAX];
  ocfd_kinetics kin;
  ocfd_transport tr;
  bool have_kin = false;

  /* read_Spec, CHEM_thermdyn.f90:39-47 */
  void set_thermo(const ocfd_thermo* th, int realgas) {
    ns = th->n_spec;
    n_tct = th->n_tct;
    if_realgas = realgas;
    for (int j = 0; j < OCFD_NTCT_MAX; j++) tct[j] = th->tct[j];
    tct_max = th->tct_max;
    for (int k = 0; k < ns; k++) {
      Mi[k] = th->mi[k];
      specflag[k] = th->spec_flag[k];
      Ri[k] = R0 / Mi[k];
      for (int j = 0; j < n_tct; j++) {
        A[k][j] = th->coef[k][j][0];
        B[k][j] = th->coef[k][j][1];
        C[k][j] = th->coef[k][j][2];
        D[k][j] = th->coef[k][j][3];
        E[k][j] = th->coef[k][j][4];
        F[k][j] = th->coef[k][j][5];
        G[k][j] = th->coef[k][j][6];
      }
      Ect[k][0] = 0.0;
      for (int j = 0; j < n_tct - 1; j++) {
        double t = tct[j];
        double s = (A[k][j + 1] - A[k][j]) * t + (B[k][j + 1] - B[k][j]) * p2(t) / 2.0 +
                   (C[k][j + 1] - C[k][j]) * p3(t) / 3.0 + (D[k][j + 1] - D[k][j]) * p4(t) / 4.0 +
                   (E[k][j + 1] - E[k][j]) * p5(t) / 5.0;
        Ect[k][j + 1] = -s + Ect[k][j];
      }
    }
  }

  int range(double T) const {
    int jc = 0;
    for (int j = 0; j < n_tct - 1; j++)
      if (T > tct[j]) jc = j + 1;
    return jc;
  }

  /* comput_E (CHEM_thermdyn.f90:58-68, 114-123, 203-231) */
  double E_of_T(const double* di, double T) const {
    if (if_realgas == 0) {
      double e = 0.0;
      for (int k = 0; k < ns; k++) e = e + 2.5 * Ri[k] * di[k] * T;
      return e;
    }
    double A1 = 0, B1 = 0, C1 = 0, D1 = 0, E1 = 0, Ec = 0;
    int jc = range(T);
    for (int k = 0; k < ns; k++) {
      double R1 = Ri[k];
      A1 = A1 + (A[k][jc] - 1.0) * R1 * di[k];
      B1 = B1 + B[k][jc] * R1 * di[k];
      C1 = C1 + C[k][jc] * R1 * di[k];
      D1 = D1 + D[k][jc] * R1 * di[k];
      E1 = E1 + E[k][jc] * R1 * di[k];
      Ec = Ec + Ect[k][jc] * R1 * di[k];
    }
    if (T <= tct_max) {
      return A1 * T + B1 * p2(T) / 2.0 + C1 * p3(T) / 3.0 + D1 * p4(T) / 4.0 + E1 * p5(T) / 5.0 + Ec;
    }
    double tm = tct_max;
    double Cv2 = A1 + B1 * tm + C1 * p2(tm) + D1 * p3(tm) + E1 * p4(tm);
    return A1 * tm + B1 * p2(tm) / 2.0 + C1 * p3(tm) / 3.0 + D1 * p4(tm) / 4.0 + E1 * p5(tm) / 5.0 + Ec +
           Cv2 * (T - tm);
  }

  /* comput_Cp (CHEM_thermdyn.f90:72-82, 126-136, 234-266) */
  double Cp(double d, const double* di, double T) const {
    if (if_realgas == 0) {
      double cp = 0.0;
      for (int k = 0; k < ns; k++) cp = cp + 3.5 * Ri[k] * di[k];
      return cp / d;
    }
    double A1 = 0, B1 = 0, C1 = 0, D1 = 0, E1 = 0;
    int jc = range(T);
    for (int k = 0; k < ns; k++) {
      double R1 = Ri[k];
      A1 = A1 + A[k][jc] * R1 * di[k];
      B1 = B1 + B[k][jc] * R1 * di[k];
      C1 = C1 + C[k][jc] * R1 * di[k];
      D1 = D1 + D[k][jc] * R1 * di[k];
      E1 = E1 + E[k][jc] * R1 * di[k];
    }
    if (T <= tct_max) return (A1 + B1 * T + C1 * p2(T) + D1 * p3(T) + E1 * p4(T)) / d;
    double tm = tct_max;
    return (A1 + B1 * tm + C1 * p2(tm) + D1 * p3(tm) + E1 * p4(tm)) / d;
  }

  /* comput_T (CHEM_thermdyn.f90:85-95, 158-168, 327-382); returns Newton iterations used */
  double T_of_E(const double* di, double Ein, int* iters = nullptr) const {
    if (if_realgas == 0) {
      double rCv = 0.0;
      for (int k = 0; k < ns; k++) rCv = rCv + 2.5 * Ri[k] * di[k];
      if (iters) *iters = 0;
      return Ein / rCv;
    }
    double A1[OCFD_NTCT_MAX], B1[OCFD_NTCT_MAX], C1[OCFD_NTCT_MAX], D1[OCFD_NTCT_MAX], E1[OCFD_NTCT_MAX],
        Ec[OCFD_NTCT_MAX];
    for (int j = 0; j < n_tct; j++) {
      A1[j] = B1[j] = C1[j] = D1[j] = E1[j] = Ec[j] = 0.0;
      for (int k = 0; k < ns; k++) {
        double R1 = Ri[k];
        A1[j] = A1[j] + (A[k][j] - 1.0) * R1 * di[k];
        B1[j] = B1[j] + B[k][j] * R1 * di[k];
        C1[j] = C1[j] + C[k][j] * R1 * di[k];
        D1[j] = D1[j] + D[k][j] * R1 * di[k];
        E1[j] = E1[j] + E[k][j] * R1 * di[k];
        Ec[j] = Ec[j] + Ect[k][j] * R1 * di[k];
      }
    }
    double T1 = Ein / A1[0], T2 = T1;
    int ks = 0;
    while (ks <= 30) {
      int jc = range(T1);
      double Et1, Ex;
      if (T1 <= tct_max) {
        Et1 = A1[jc] * T1 + B1[jc] * p2(T1) / 2.0 + C1[jc] * p3(T1) / 3.0 + D1[jc] * p4(T1) / 4.0 +
              E1[jc] * p5(T1) / 5.0 + Ec[jc];
        Ex = A1[jc] + B1[jc] * T1 + C1[jc] * p2(T1) + D1[jc] * p3(T1) + E1[jc] * p4(T1);
      } else {
        double tm = tct_max;
        Ex = A1[jc] + B1[jc] * tm + C1[jc] * p2(tm) + D1[jc] * p3(tm) + E1[jc] * p4(tm);
        Et1 = A1[jc] * tm + B1[jc] * p2(tm) / 2.0 + C1[jc] * p3(tm) / 3.0 + D1[jc] * p4(tm) / 4.0 +
              E1[jc] * p5(tm) / 5.0 + Ec[jc] + Ex * (T1 - tm);
      }
      T2 = T1 - (Et1 - Ein) / Ex;
      ks = ks + 1;
      double err = std::fabs(T2 - T1);
      T1 = T2;
      if (err < 1.0e-3) break;
    }
    if (iters) *iters = ks;
    return T2;
  }

  /* comput_P (CHEM_thermdyn.f90:385-395) */
  double P(const double* di, double T) const {
    double p = 0.0;
    for (int k = 0; k < ns; k++) p = p + Ri[k] * di[k] * T;
    return p;
  }
  /* comput_d (CHEM_thermdyn.f90:399-409) */
  double Dens(const double* ai, double T, double p) const {
    double R1 = 0.0;
    for (int k = 0; k < ns; k++) R1 = R1 + Ri[k] * ai[k];
    return p / (T * R1);
  }
  /* comput_hi (CHEM_thermdyn.f90:98-108, 172-178, 271-293) */
  double hi(int k, double T) const {
    if (if_realgas == 0) return 3.5 * Ri[k] * T;
    int jc = range(T);
    if (T <= tct_max)
      return (A[k][jc] * T + B[k][jc] * p2(T) / 2.0 + C[k][jc] * p3(T) / 3.0 + D[k][jc] * p4(T) / 4.0 +
              E[k][jc] * p5(T) / 5.0 + Ect[k][jc]) *
             Ri[k];
    double tm = tct_max;
    double cpm = A[k][jc] + B[k][jc] * tm + C[k][jc] * p2(tm) + D[k][jc] * p3(tm) + E[k][jc] * p4(tm);
    return (A[k][jc] * tm + B[k][jc] * p2(tm) / 2.0 + C[k][jc] * p3(tm) / 3.0 + D[k][jc] * p4(tm) / 4.0 +
            E[k][jc] * p5(tm) / 5.0 + Ect[k][jc] + cpm * (T - tm)) *
           Ri[k];
  }
  /* comput_gibbs (CHEM_thermdyn.f90:296-319), gi = G/Ri */
  double gibbs(int k, double T) const {
    int jc = range(T);
    if (T <= tct_max) {
      return A[k][jc] * (1.0 - std::log(T)) * T - B[k][jc] * p2(T) / 2.0 - C[k][jc] * p3(T) / 6.0 -
             D[k][jc] * p4(T) / 12.0 - E[k][jc] * p5(T) / 20.0 + F[k][jc] - G[k][jc] * T;
    }
    double tm = tct_max;
    double cpm = A[k][jc] + B[k][jc] * tm + C[k][jc] * p2(tm) + D[k][jc] * p3(tm) + E[k][jc] * p4(tm);
    double hm = A[k][jc] * tm + B[k][jc] * p2(tm) / 2.0 + C[k][jc] * p3(tm) / 3.0 + D[k][jc] * p4(tm) / 4.0 +
                E[k][jc] * p5(tm) / 5.0 + F[k][jc];
    double sm = A[k][jc] * std::log(tm) + B[k][jc] * tm + C[k][jc] * p2(tm) / 2.0 + D[k][jc] * p3(tm) / 3.0 +
                E[k][jc] * p4(tm) / 4.0 + G[k][jc];
    return hm + cpm * (T - tm) - T * (sm + cpm * std::log(T / tm));
  }
  /* update_Et (CHEM_thermdyn.f90:184-196) */
  double update_Et(const double* di, const double* dinew, double E0) const {
    double e = E0;
    for (int i = 0; i < ns; i++) e = e - (dinew[i] - di[i]) * Ri[i] * F[i][0];
    return e;
  }

  /* Constant-pressure reactor (an extension: the reference's reactor is constant-volume,
   * OCFD_Time_Adv.f90:174-193). The reactor keeps its initial pressure p0 and specific total
   * enthalpy h0 = (E + sum d_k R_k F_k + p) / rho, E the sensible energy of comput_E and F_k the
   * formation term that update_Et (CHEM_thermdyn.f90:184-196) books. After every constant-volume
   * sub-step the mixture (mass fractions Y fixed) is brought back to p0 at h0: Newton on T for
   * e(T, Y) + R T + sum Y_k R_k F_k = h0 (e from comput_E with Y as densities, derivative the
   * mass-specific Cp), stopped when |dT| <= 1e-10 T (at most 50 iterations), then
   * rho = p0 / (R T), d = Y rho, E = comput_E(d, T). The GPU applies the identical operations. */
  void cp_reference(const double* di, double Et, double& h0, double& p0) const {
    double T = T_of_E(di, Et);
    p0 = P(di, T);
    double rho = 0.0, cf = 0.0;
    for (int k = 0; k < ns; k++) {
      rho = rho + di[k];
      cf = cf + di[k] * Ri[k] * F[k][0];
    }
    h0 = (Et + cf + p0) / rho;
  }
  void cp_restore(double* di, double& Et, double h0, double p0) const {
    double rho = 0.0;
    for (int k = 0; k < ns; k++) rho = rho + di[k];
    double Y[OCFD_MAX_SPEC];
    double R1 = 0.0, cf = 0.0;
    for (int k = 0; k < ns; k++) {
      Y[k] = di[k] / rho;
      R1 = R1 + Ri[k] * Y[k];
      cf = cf + Y[k] * Ri[k] * F[k][0];
    }
    double T = T_of_E(di, Et);
    for (int it = 0; it < 50; it++) {
      double g = E_of_T(Y, T) + R1 * T + cf - h0;
      double dT = g / Cp(1.0, Y, T);
      T = T - dT;
      if (std::fabs(dT) <= 1.0e-10 * T) break;
    }
    double r1 = p0 / (R1 * T);
    for (int k = 0; k < ns; k++) di[k] = Y[k] * r1;
    Et = E_of_T(di, T);
  }

  /* ---------------- transport (TRANSPORT_modules.f90) ---------------- */
  double viscosity(double T, const double* Xi) const {
    if (tr.flag_vis == 0) {
      const double TA = 288.15, TC = 110.4;
      return tr.amu0 * std::sqrt(p3(T / TA)) * (TA + TC) / (TC + T);
    }
    double mui[OCFD_MAX_SPEC];
    double L = std::log(T);
    for (int m = 0; m < ns; m++)
      mui[m] = std::exp(tr.mu_an[m][0] + tr.mu_an[m][1] * L + tr.mu_an[m][2] * p2(L) + tr.mu_an[m][3] * p3(L)) * 0.1;
    double mu = 0.0;
    for (int k = 0; k < ns; k++) {
      double pk0 = 0.0;
      for (int j = 0; j < ns; j++) {
        double s = 1.0 + std::sqrt(mui[k] / mui[j] * std::sqrt(Mi[j] / Mi[k]));
        double pkj = p2(s) / std::sqrt(8.0 * (1.0 + Mi[k] / Mi[j]));
        pk0 = pk0 + Xi[j] * pkj;
      }
      mu = mu + Xi[k] * mui[k] / pk0;
    }
    return mu;
  }
  double conductivity(double Amu, double cp, double T, const double* Xi) const {
    if (tr.flag_cond == 0) return Amu * cp / tr.pr;
    double ki[OCFD_MAX_SPEC];
    double L = std::log(T);
    for (int m = 0; m < ns; m++)
      ki[m] = std::exp(tr.k_an[m][0] + tr.k_an[m][1] * L + tr.k_an[m][2] * p2(L) + tr.k_an[m][3] * p3(L)) * 1.0e-5;
    double a1 = 0.0, a2 = 0.0;
    for (int m = 0; m < ns; m++) {
      a1 = a1 + Xi[m] * ki[m];
      a2 = a2 + Xi[m] / ki[m];
    }
    return 0.5 * (a1 + 1.0 / a2);
  }
  void diffusion(double* AmDi, double Amu, double T, double d, double p, const double* Xi) const {
    if (tr.flag_diff == 0) {
      double d0 = 0.0;
      for (int m = 0; m < ns; m++) d0 = d0 + Xi[m] * Mi[m];
      for (int m = 0; m < ns; m++) AmDi[m] = Amu * (1.0 - Xi[m] * Mi[m] / d0) / ((1.0 - Xi[m]) * tr.sc * d + 1.0e-20);
      return;
    }
    double D2[OCFD_MAX_SPEC][OCFD_MAX_SPEC];
    double L = std::log(T);
    for (int j = 0; j < ns; j++)
      for (int k = 0; k <= j; k++)
        D2[k][j] = std::exp(tr.d_an[k][j][0] + tr.d_an[k][j][1] * L + tr.d_an[k][j][2] * p2(L) +
                            tr.d_an[k][j][3] * p3(L)) *
                   1.0e-4;
    for (int j = 0; j < ns; j++)
      for (int k = j + 1; k < ns; k++) D2[k][j] = D2[j][k];
    for (int k = 0; k < ns; k++) {
      double ds = 0.0;
      for (int j = 0; j < ns; j++)
        if (j != k) ds = ds + Xi[j] / D2[k][j];
      AmDi[k] = (1.0 - Xi[k]) / (ds + 1.0e-20) * ATM / p;
    }
  }

  /* ---------------- kinetics (CHEM_reactions.f90) ---------------- */
  static double arrhenius(double A_, double b, double E_, double T) { return A_ * std::pow(T, b) * std::exp(-E_ / T); }

  void rate_coef(const double* ci, double* wf, double* wr, double T) const {
    double Kjx[OCFD_MAX_REAC];
    if (kin.rereac == 0) {
      const double Rs = R0 / ATM * 1.0e6;
      double gi[OCFD_MAX_SPEC];
      for (int i = 0; i < ns; i++) gi[i] = gibbs(i, T);
      for (int j = 0; j < nreac; j++) {
        double dgi = 0.0;
        int sgm = 0;
        for (int i = 0; i < ns; i++) {
          dgi = dgi + gi[i] * (double)(kin.vr[j][i] - kin.vf[j][i]);
          sgm = sgm + kin.vr[j][i] - kin.vf[j][i];
        }
        Kjx[j] = std::exp(-dgi / T) * powi_rt(Rs * T, -sgm);
      }
    }
    for (int j = 0; j < nreac; j++) {
      double Ctrb = 0.0;
      if (kin.tr_reac[j] == 1) {
        for (int i = 0; i < ns; i++) Ctrb = Ctrb + ci[i] * kin.treff[j][i];
      }
      double wf1 = arrhenius(kin.af[j][0], kin.bf[j][0], kin.ef[j][0], T);
      if (kin.af_type[j] == 0) {
        wf[j] = wf1;
      } else if (kin.af_type[j] == 2) {
        double wf2 = arrhenius(kin.af[j][1], kin.bf[j][1], kin.ef[j][1], T);
        wf[j] = wf1 + wf2;
      } else if (kin.af_type[j] == 1) {
        double wf2 = arrhenius(kin.af[j][1], kin.bf[j][1], kin.ef[j][1], T);
        double Prs = wf1 / wf2 * Ctrb;
        double Fc = kin.fc_troe[j];
        double lfc = std::log10(Fc);
        double ac = -0.4 - (double)0.67f * lfc;
        double an = 0.75 - (double)1.27f * lfc;
        double lpr = std::log10(Prs);
        double q = (lpr + ac) / (an - 0.14 * (lpr + ac));
        double Fx = std::pow(10.0, lfc / (1.0 + p2(q)));
        wf[j] = wf2 * Prs / (1.0 + Prs) * Fx;
      }
      if (kin.rereac == 0) {
        wr[j] = wf[j] / Kjx[j];
      } else if (kin.rereac == 1) {
        wr[j] = arrhenius(kin.ar[j], kin.br[j], kin.er[j], T);
      } else {
        double z = 10000.0 / T;
        double kj = std::exp(kin.park[j][0] + kin.park[j][1] * z + kin.park[j][2] * p2(z) + kin.park[j][3] * p3(z) +
                             kin.park[j][4] * p4(z));
        if (kj < 1.0e-30) kj = 1.0e-30;
        wr[j] = wf[j] / kj;
      }
      if (kin.tr_reac[j] == 1 && kin.af_type[j] != 1) {
        wf[j] = wf[j] * Ctrb;
        wr[j] = wr[j] * Ctrb;
      }
    }
  }

  /* Reaction_rate (CHEM_reactions.f90:203-225) */
  void rate(const double* ci, double* ri, double T) const {
    double wf[OCFD_MAX_REAC], wr[OCFD_MAX_REAC];
    rate_coef(ci, wf, wr, T);
    for (int i = 0; i < ns; i++) ri[i] = 0.0;
    for (int j = 0; j < nreac; j++) {
      double wf1 = wf[j], wr1 = wr[j];
      for (int i = 0; i < ns; i++) {
        if (kin.vf[j][i] != 0) wf1 = wf1 * powi_rt(ci[i], kin.vf[j][i]);
        if (kin.vr[j][i] != 0) wr1 = wr1 * powi_rt(ci[i], kin.vr[j][i]);
      }
      for (int i = 0; i < ns; i++) ri[i] = ri[i] + (wf1 - wr1) * (double)(kin.vr[j][i] - kin.vf[j][i]);
    }
  }

  /* Reaction_rate_and_Matrix (CHEM_reactions.f90:230-272); Ar is [i][j] */
  void rate_and_matrix(const double* ci, double* ri, double Ar[OCFD_MAX_SPEC][OCFD_MAX_SPEC], double T) const {
    double wf[OCFD_MAX_REAC], wr[OCFD_MAX_REAC];
    rate_coef(ci, wf, wr, T);
    for (int i = 0; i < ns; i++) {
      ri[i] = 0.0;
      for (int j = 0; j < ns; j++) Ar[i][j] = 0.0;
    }
    for (int k = 0; k < nreac; k++) {
      double wf1 = wf[k], wr1 = wr[k];
      for (int i = 0; i < ns; i++) {
        if (kin.vf[k][i] != 0) wf1 = wf1 * powi_rt(ci[i], kin.vf[k][i]);
        if (kin.vr[k][i] != 0) wr1 = wr1 * powi_rt(ci[i], kin.vr[k][i]);
      }
      for (int i = 0; i < ns; i++) ri[i] = ri[i] + (wf1 - wr1) * (double)(kin.vr[k][i] - kin.vf[k][i]);
      for (int j = 0; j < ns; j++) {
        double Awf = (double)kin.vf[k][j] * wf1 / (ci[j] + 1.0e-20);
        double Awr = (double)kin.vr[k][j] * wr1 / (ci[j] + 1.0e-20);
        for (int i = 0; i < ns; i++) Ar[i][j] = Ar[i][j] + (Awf - Awr) * (double)(kin.vr[k][i] - kin.vf[k][i]);
      }
    }
  }

  /* Gauss elimination with partial pivoting (CHEM_reactions.f90:523-567). Columns left of the
   * pivot column are never read again, so skipping their update does not change any result. */
  void gauss(int n, double a[OCFD_MAX_SPEC][OCFD_MAX_SPEC], double* b, double* x) const {
    for (int k = 0; k < n - 1; k++) {
      double fmax = std::fabs(a[k][k]);
      int kk = k;
      for (int i = k + 1; i < n; i++)
        if (std::fabs(a[i][k]) > fmax) {
          fmax = std::fabs(a[i][k]);
          kk = i;
        }
      for (int j = k; j < n; j++) {
        double t = a[k][j];
        a[k][j] = a[kk][j];
        a[kk][j] = t;
      }
      double t = b[k];
      b[k] = b[kk];
      b[kk] = t;
      for (int i = k + 1; i < n; i++) {
        double f = -a[i][k] / a[k][k];
        for (int j = k; j < n; j++) a[i][j] = a[i][j] + f * a[k][j];
        b[i] = b[i] + f * b[k];
      }
    }
    x[n - 1] = b[n - 1] / a[n - 1][n - 1];
    for (int i = n - 2; i >= 0; i--) {
      x[i] = b[i];
      for (int j = i + 1; j < n; j++) x[i] = x[i] - a[i][j] * x[j];
      x[i] = x[i] / a[i][i];
    }
  }

  /* chemical_timeAdv (CHEM_reactions.f90:374-602): di and E updated in place */
  void time_adv(double* di, double& Et, double dt) const {
    double ci[OCFD_MAX_SPEC], ri[OCFD_MAX_SPEC], dinew[OCFD_MAX_SPEC];
    if (timeadv == 1) {
      double T = T_of_E(di, Et);
      for (int i = 0; i < ns; i++) ci[i] = di[i] / Mi[i] * 1.0e-6;
      rate(ci, ri, T);
      for (int i = 0; i < ns; i++) dinew[i] = di[i] + ri[i] * Mi[i] * 1.0e6 * dt;
      Et = update_Et(di, dinew, Et);
      for (int i = 0; i < ns; i++) di[i] = dinew[i];
    } else if (timeadv == 2) {
      double di1[OCFD_MAX_SPEC];
      double T = T_of_E(di, Et);
      for (int i = 0; i < ns; i++) ci[i] = di[i] / Mi[i] * 1.0e-6;
      rate(ci, ri, T);
      for (int i = 0; i < ns; i++) di1[i] = di[i] + ri[i] * Mi[i] * 1.0e6 * dt;
      Et = update_Et(di, di1, Et);
      T = T_of_E(di, Et); /* the reference evaluates T from the old di here (CHEM_reactions.f90:452) */
      for (int i = 0; i < ns; i++) ci[i] = di1[i] / Mi[i] * 1.0e-6;
      rate(ci, ri, T);
      for (int i = 0; i < ns; i++) dinew[i] = 0.5 * di[i] + 0.5 * di1[i] + 0.5 * ri[i] * Mi[i] * 1.0e6 * dt;
      Et = update_Et(di1, dinew, Et);
      for (int i = 0; i < ns; i++) di[i] = dinew[i];
    } else if (timeadv == 3) {
      const double ra[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0}, rb[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
      double din[OCFD_MAX_SPEC];
      for (int i = 0; i < ns; i++) din[i] = di[i];
      for (int krk = 0; krk < 3; krk++) {
        double T = T_of_E(di, Et);
        for (int i = 0; i < ns; i++) ci[i] = di[i] / Mi[i] * 1.0e-6;
        rate(ci, ri, T);
        for (int i = 0; i < ns; i++) dinew[i] = ra[krk] * din[i] + rb[krk] * (di[i] + ri[i] * Mi[i] * 1.0e6 * dt);
        Et = update_Et(di, dinew, Et);
        for (int i = 0; i < ns; i++) di[i] = dinew[i];
      }
    } else { /* -1: linearised implicit Euler */
      double Ar[OCFD_MAX_SPEC][OCFD_MAX_SPEC], A1[OCFD_MAX_SPEC][OCFD_MAX_SPEC], di1[OCFD_MAX_SPEC], dd[OCFD_MAX_SPEC];
      double T = T_of_E(di, Et);
      for (int i = 0; i < ns; i++) ci[i] = di[i] / Mi[i] * 1.0e-6;
      rate_and_matrix(ci, ri, Ar, T);
      for (int j = 0; j < ns; j++)
        for (int i = 0; i < ns; i++) {
          double a = (i == j) ? 1.0 : 0.0;
          A1[i][j] = a - Ar[i][j] * Mi[i] / Mi[j] * dt;
        }
      for (int i = 0; i < ns; i++) di1[i] = ri[i] * Mi[i] * 1.0e6 * dt;
      gauss(ns, A1, di1, dd);
      for (int i = 0; i < ns; i++) dinew[i] = di[i] + dd[i];
      Et = update_Et(di, dinew, Et);
      for (int i = 0; i < ns; i++) di[i] = dinew[i];
    }
  }
};

}  // namespace ocfd_oracle
