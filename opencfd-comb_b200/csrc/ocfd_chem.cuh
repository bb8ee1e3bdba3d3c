// Finite-rate chemistry on sm_100a (code/Chemical/CHEM_reactions.f90).
//
// One thread integrates one reactor (cell): rate coefficients (Arrhenius, dual Arrhenius, Troe
// fall-off, three-body), reverse rates from Gibbs equilibrium constants / Arrhenius / Park fits,
// and the four integrators of chemical_timeAdv (explicit Euler, RK2, RK3, linearised implicit
// Euler with a partially pivoted Gauss elimination). The mechanism lives in constant memory, so
// the reaction loops are warp-uniform broadcasts.
//
// k_chem_cells : Chemical_time_advance x nsub + comput_T_P on the flow grid (OCFD_Time_Adv.f90:169-196)
// k_chem_batch : independent 0-D reactors as a persistent work queue. Reactors are visited in
//                descending order of their sub-step count (counting sort on the device), so the
//                32 reactors of a warp carry near-equal work and long reactors start first.
#pragma once
#include "ocfd_device.cuh"

// resident 128-thread blocks per SM given to the register allocator of the chemistry kernels:
// 3 (at most 170 registers) measured 16-18 % faster than the unconstrained 255 registers on the
// 2^20-reactor batch and the jet's cells, 4 (128 registers) spills too much
#ifndef OCFD_CHEM_MINB
#define OCFD_CHEM_MINB 3
#endif

namespace ocfd {

template <int NS>
__device__ __forceinline__ void rate_coef(const double* ci, double* wf, double* wr, double T) {
  double gi[NS];
  double Rs = 8.314 / 1.013e5 * 1.0e6;
  if (cC.rereac == 0) {
    double lt = log(T);
#pragma unroll
    for (int i = 0; i < NS; i++) gi[i] = dev_gibbs(i, T, lt);
  }
  for (int j = 0; j < cC.nreac; j++) {
    double Ctrb = 0.0;
    if (cC.tr_reac[j] == 1) {
#pragma unroll
      for (int i = 0; i < NS; i++) Ctrb = Ctrb + ci[i] * cC.treff[j][i];
    }
    double wf1 = cC.af[j][0] * pow(T, cC.bf[j][0]) * exp(-cC.ef[j][0] / T);
    double w;
    const int at = cC.af_type[j];
    if (at == 0) {
      w = wf1;
    } else {
      double wf2 = cC.af[j][1] * pow(T, cC.bf[j][1]) * exp(-cC.ef[j][1] / T);
      if (at == 2) {
        w = wf1 + wf2;
      } else {  // Troe fall-off; 0.67 and 1.27 are single-precision literals in the reference
        double Prs = wf1 / wf2 * Ctrb;
        double lfc = log10(cC.fc_troe[j]);
        double ac = -0.4 - (double)0.67f * lfc;
        double an = 0.75 - (double)1.27f * lfc;
        double lpr = log10(Prs);
        double qq = (lpr + ac) / (an - 0.14 * (lpr + ac));
        double Fx = pow(10.0, lfc / (1.0 + q2(qq)));
        w = wf2 * Prs / (1.0 + Prs) * Fx;
      }
    }
    double r;
    if (cC.rereac == 0) {
      double dgi = 0.0;
#pragma unroll
      for (int i = 0; i < NS; i++) dgi = dgi + gi[i] * (double)(cC.vr[j][i] - cC.vf[j][i]);
      double kjx = exp(-dgi / T) * powi_rt(Rs * T, -cC.sgm[j]);
      r = w / kjx;
    } else if (cC.rereac == 1) {
      r = cC.ar[j] * pow(T, cC.br[j]) * exp(-cC.er[j] / T);
    } else {
      double z = 10000.0 / T;
      double kj = exp(cC.park[j][0] + cC.park[j][1] * z + cC.park[j][2] * q2(z) + cC.park[j][3] * q3(z) +
                      cC.park[j][4] * q4(z));
      if (kj < 1.0e-30) kj = 1.0e-30;
      r = w / kj;
    }
    if (cC.tr_reac[j] == 1 && at != 1) {
      w = w * Ctrb;
      r = r * Ctrb;
    }
    wf[j] = w;
    wr[j] = r;
  }
}

template <int NS>
__device__ __forceinline__ void progress(const double* ci, double wf, double wr, int k, double& wf1, double& wr1) {
  wf1 = wf;
  wr1 = wr;
#pragma unroll
  for (int i = 0; i < NS; i++) {
    int a = cC.vf[k][i], b = cC.vr[k][i];
    if (a != 0) wf1 = wf1 * powi_rt(ci[i], a);
    if (b != 0) wr1 = wr1 * powi_rt(ci[i], b);
  }
}

// Reaction_rate (CHEM_reactions.f90:203-225)
template <int NS>
__device__ void reaction_rate(const double* ci, double* ri, double T) {
  double wf[OCFD_MAX_REAC], wr[OCFD_MAX_REAC];
  rate_coef<NS>(ci, wf, wr, T);
#pragma unroll
  for (int i = 0; i < NS; i++) ri[i] = 0.0;
  for (int k = 0; k < cC.nreac; k++) {
    double wf1, wr1;
    progress<NS>(ci, wf[k], wr[k], k, wf1, wr1);
#pragma unroll
    for (int i = 0; i < NS; i++) ri[i] = ri[i] + (wf1 - wr1) * (double)(cC.vr[k][i] - cC.vf[k][i]);
  }
}

// Reaction_rate_and_Matrix (CHEM_reactions.f90:230-272); Ar[i*NS+j] = d r_i / d c_j
template <int NS>
__device__ void reaction_rate_matrix(const double* ci, double* ri, double* Ar, double T) {
  double wf[OCFD_MAX_REAC], wr[OCFD_MAX_REAC];
  rate_coef<NS>(ci, wf, wr, T);
  for (int i = 0; i < NS; i++) {
    ri[i] = 0.0;
    for (int j = 0; j < NS; j++) Ar[i * NS + j] = 0.0;
  }
  for (int k = 0; k < cC.nreac; k++) {
    double wf1, wr1;
    progress<NS>(ci, wf[k], wr[k], k, wf1, wr1);
#pragma unroll
    for (int i = 0; i < NS; i++) ri[i] = ri[i] + (wf1 - wr1) * (double)(cC.vr[k][i] - cC.vf[k][i]);
    for (int j = 0; j < NS; j++) {
      int a = cC.vf[k][j], b = cC.vr[k][j];
      if (a == 0 && b == 0) continue;  // both derivatives are exactly +0: adding them changes nothing
      double Awf = (double)a * wf1 / (ci[j] + 1.0e-20);
      double Awr = (double)b * wr1 / (ci[j] + 1.0e-20);
      double dA = Awf - Awr;
#pragma unroll
      for (int i = 0; i < NS; i++) Ar[i * NS + j] = Ar[i * NS + j] + dA * (double)(cC.vr[k][i] - cC.vf[k][i]);
    }
  }
}

// Gauss elimination with partial pivoting (CHEM_reactions.f90:523-567); a is row-major NSxNS.
// Columns left of the pivot are never read again, so only columns >= k are updated.
template <int NS>
__device__ void gauss(double* a, double* b, double* x) {
  for (int k = 0; k < NS - 1; k++) {
    double fmax = fabs(a[k * NS + k]);
    int kk = k;
    for (int i = k + 1; i < NS; i++)
      if (fabs(a[i * NS + k]) > fmax) {
        fmax = fabs(a[i * NS + k]);
        kk = i;
      }
    if (kk != k) {
      for (int j = k; j < NS; j++) {
        double t = a[k * NS + j];
        a[k * NS + j] = a[kk * NS + j];
        a[kk * NS + j] = t;
      }
      double t = b[k];
      b[k] = b[kk];
      b[kk] = t;
    }
    for (int i = k + 1; i < NS; i++) {
      double f = -a[i * NS + k] / a[k * NS + k];
      for (int j = k; j < NS; j++) a[i * NS + j] = a[i * NS + j] + f * a[k * NS + j];
      b[i] = b[i] + f * b[k];
    }
  }
  x[NS - 1] = b[NS - 1] / a[(NS - 1) * NS + NS - 1];
  for (int i = NS - 2; i >= 0; i--) {
    double s = b[i];
    for (int j = i + 1; j < NS; j++) s = s - a[i * NS + j] * x[j];
    x[i] = s / a[i * NS + i];
  }
}

template <int NS>
__device__ __forceinline__ double update_et(const double* di, const double* dn, double E) {
#pragma unroll
  for (int i = 0; i < NS; i++) E = E - (dn[i] - di[i]) * cC.Ri[i] * cC.cf[i][0][5];
  return E;
}

// chemical_timeAdv (CHEM_reactions.f90:374-390) for one reactor
template <int NS>
__device__ void chem_step(double* di, double& E, double dt, int* nfail) {
  double ci[NS], ri[NS], dn[NS];
  const int mode = cC.timeadv;
  if (mode == 1) {
    double T = dev_T<NS>(di, E, nfail);
#pragma unroll
    for (int i = 0; i < NS; i++) ci[i] = di[i] / cC.Mi[i] * 1.0e-6;
    reaction_rate<NS>(ci, ri, T);
#pragma unroll
    for (int i = 0; i < NS; i++) dn[i] = di[i] + ri[i] * cC.Mi[i] * 1.0e6 * dt;
    E = update_et<NS>(di, dn, E);
#pragma unroll
    for (int i = 0; i < NS; i++) di[i] = dn[i];
  } else if (mode == 2) {
    double d1[NS];
    double T = dev_T<NS>(di, E, nfail);
#pragma unroll
    for (int i = 0; i < NS; i++) ci[i] = di[i] / cC.Mi[i] * 1.0e-6;
    reaction_rate<NS>(ci, ri, T);
#pragma unroll
    for (int i = 0; i < NS; i++) d1[i] = di[i] + ri[i] * cC.Mi[i] * 1.0e6 * dt;
    E = update_et<NS>(di, d1, E);
    T = dev_T<NS>(di, E, nfail);  // the reference takes T from the old densities here
#pragma unroll
    for (int i = 0; i < NS; i++) ci[i] = d1[i] / cC.Mi[i] * 1.0e-6;
    reaction_rate<NS>(ci, ri, T);
#pragma unroll
    for (int i = 0; i < NS; i++) dn[i] = 0.5 * di[i] + 0.5 * d1[i] + 0.5 * ri[i] * cC.Mi[i] * 1.0e6 * dt;
    E = update_et<NS>(d1, dn, E);
#pragma unroll
    for (int i = 0; i < NS; i++) di[i] = dn[i];
  } else if (mode == 3) {
    const double ra[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0}, rb[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
    double d0[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) d0[i] = di[i];
    for (int krk = 0; krk < 3; krk++) {
      double T = dev_T<NS>(di, E, nfail);
#pragma unroll
      for (int i = 0; i < NS; i++) ci[i] = di[i] / cC.Mi[i] * 1.0e-6;
      reaction_rate<NS>(ci, ri, T);
#pragma unroll
      for (int i = 0; i < NS; i++) dn[i] = ra[krk] * d0[i] + rb[krk] * (di[i] + ri[i] * cC.Mi[i] * 1.0e6 * dt);
      E = update_et<NS>(di, dn, E);
#pragma unroll
      for (int i = 0; i < NS; i++) di[i] = dn[i];
    }
  } else {  // -1: linearised backward Euler
    double Ar[NS * NS], rhs[NS], dd[NS];
    double T = dev_T<NS>(di, E, nfail);
#pragma unroll
    for (int i = 0; i < NS; i++) ci[i] = di[i] / cC.Mi[i] * 1.0e-6;
    reaction_rate_matrix<NS>(ci, ri, Ar, T);
    for (int j = 0; j < NS; j++)
      for (int i = 0; i < NS; i++) {
        double a = (i == j) ? 1.0 : 0.0;
        Ar[i * NS + j] = a - Ar[i * NS + j] * cC.Mi[i] / cC.Mi[j] * dt;
      }
#pragma unroll
    for (int i = 0; i < NS; i++) rhs[i] = ri[i] * cC.Mi[i] * 1.0e6 * dt;
    gauss<NS>(Ar, rhs, dd);
#pragma unroll
    for (int i = 0; i < NS; i++) dn[i] = di[i] + dd[i];
    E = update_et<NS>(di, dn, E);
#pragma unroll
    for (int i = 0; i < NS; i++) di[i] = dn[i];
  }
}

template <int NS>
__global__ void __launch_bounds__(128, OCFD_CHEM_MINB) k_chem_cells(double* f, double* Et, double* T, double* p, double* di,
                                                    double dt2, int nsub, int* nfail) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cC.N) return;
  int i = t % cC.nx + 1, j = (t / cC.nx) % cC.ny + 1, k = t / cC.nx / cC.ny + 1;
  const int q = hidx(i, j, k);
  double d1[NS];
#pragma unroll
  for (int m = 0; m < NS; m++) d1[m] = di[(size_t)m * cC.H + q];
  double e = Et[q];
  double f5 = f[4 * cC.N + t];
  for (int s = 0; s < nsub; s++) {
    double e0 = e;
    chem_step<NS>(d1, e, dt2, nfail);
    f5 = f5 + (e - e0);
  }
#pragma unroll
  for (int m = 0; m < NS; m++) di[(size_t)m * cC.H + q] = d1[m];
  Et[q] = e;
  f[4 * cC.N + t] = f5;
  double TT = dev_T<NS>(d1, e, nfail);
  T[q] = TT;
  p[q] = dev_P<NS>(d1, TT);
}

// ---- batched reactors ----
static __global__ void k_nsub_hist(int n, const int* nsub, int* hist, int nbins) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int s = nsub ? nsub[t] : 1;
  int b = min(max(s, 0), nbins - 1);
  atomicAdd(&hist[nbins - 1 - b], 1);  // descending sub-step count
}
static __global__ void k_nsub_scan(int* hist, int nbins) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int acc = 0;
  for (int b = 0; b < nbins; b++) {
    int c = hist[b];
    hist[b] = acc;
    acc += c;
  }
}
static __global__ void k_nsub_scatter(int n, const int* nsub, int* cursor, int nbins, int* perm) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int s = nsub ? nsub[t] : 1;
  int b = min(max(s, 0), nbins - 1);
  int pos = atomicAdd(&cursor[nbins - 1 - b], 1);
  perm[pos] = t;
}

template <int NS>
__global__ void __launch_bounds__(128, OCFD_CHEM_MINB) k_chem_batch(int n, double* di, double* e, const double* dt, const int* nsub,
                                                    const int* perm, int* counter, int* nfail) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(counter, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    int idx = base + lane;
    if (idx < n) {
      int r = perm[idx];
      int ks = nsub ? nsub[r] : 1;
      double dt2 = dt[r] / ks;
      double d1[NS];
#pragma unroll
      for (int m = 0; m < NS; m++) d1[m] = di[(size_t)r * NS + m];
      double ee = e[r];
      for (int s = 0; s < ks; s++) chem_step<NS>(d1, ee, dt2, nfail);
#pragma unroll
      for (int m = 0; m < NS; m++) di[(size_t)r * NS + m] = d1[m];
      e[r] = ee;
    }
  }
}

}  // namespace ocfd
