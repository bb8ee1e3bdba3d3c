// Finite-rate chemistry on sm_100a (code/Chemical/CHEM_reactions.f90).
//
// One thread integrates one reactor (cell): rate coefficients (Arrhenius, dual Arrhenius, Troe
// fall-off, three-body), reverse rates from Gibbs equilibrium constants / Arrhenius / Park fits,
// and the four integrators of chemical_timeAdv (explicit Euler, RK2, RK3, linearised implicit
// Euler with a partially pivoted Gauss elimination). The mechanism lives in constant memory, so
// the reaction loops are warp-uniform broadcasts.
//
// Nothing of a reactor is indexed at run time in thread-local memory: the reference's per-reaction
// coefficient arrays (wf, wr) are consumed inside one reaction loop, the species loops are unrolled
// (registers), and the NS x NS implicit-Euler matrix lives in the block's shared memory, one
// column-strided slab per thread (element m of thread t at sA[m * TPB + t]: a warp's accesses
// are consecutive words). The Gauss elimination is unrolled over the pivot column; only the pivot
// row index is a run-time value (a shared-memory address; the right-hand side in registers is
// swapped by predicated selects). Empty asm statements with a memory clobber between the matrix
// columns / rows keep the compiler from hoisting every shared-memory load of the unrolled loops
// to the top (which made it spill).
//
// k_chem_cells : Chemical_time_advance x nsub + comput_T_P on the flow grid (OCFD_Time_Adv.f90:169-196)
// k_chem_batch : independent 0-D reactors as a persistent work queue. Reactors are visited in
//                descending order of their sub-step count (counting sort on the device), so the
//                32 reactors of a warp carry near-equal work and long reactors start first.
//                Constant-volume (the reference's reactor) or, on request, constant-pressure.
//
// Error words (nfail points at two ints): nfail[0] counts Newton T(E) iterations that did not
// converge (comput_T_rgas, CHEM_thermdyn.f90:327-382), nfail[1] reactors whose Gauss elimination
// met a zero pivot or whose result is not finite. The arithmetic goes on as the reference's
// does (a zero pivot divides by zero); the host turns nfail[1] > 0 into an error code.
#pragma once
#include "ocfd_device.cuh"

// threads per block of the chemistry kernels and the resident-block target given to the register
// allocator: 64-thread blocks hold their 64 implicit-Euler matrices in 41.5 KB of shared memory
// (9 species); four of them per SM (two warps per scheduler) leave 255 registers per thread, which
// the 9-species cell kernel fills without spilling (five blocks cap it at 168 and spill 400 bytes)
#ifndef OCFD_CHEM_TPB
#define OCFD_CHEM_TPB 64
#endif
#ifndef OCFD_CHEM_MINB
#define OCFD_CHEM_MINB 4
#endif

namespace ocfd {

// one thread's NS x NS matrix in a column-strided shared-memory slab
template <int STRIDE>
struct Slab {
  double* b;
  __device__ __forceinline__ double& operator[](int m) const { return b[m * STRIDE]; }
};

// Forward and reverse rate coefficients of reaction j (Reaction_rate_coef,
// CHEM_reactions.f90:130-197), three-body factor included. Arrhenius A T^b exp(-E/T) is evaluated
// as A exp(b ln T - E (1/T)) with ln T and 1/T formed once per reactor: the same quantity, one
// exponential instead of a power and an exponential. 0.67 and 1.27 of the Troe form are
// single-precision literals in the reference. The reaction's structure (third-body flag tb, rate
// form at, reverse-rate form rereac, stoichiometric sum sgm) comes in as arguments: values read
// from the constant block in the generic kernels, literals in a compiled mechanism. dgi() returns
// sum_i g_i (vr_i - vf_i) (called when rereac = 0, where the reference forms it).
template <int NS, class DG>
__device__ __forceinline__ void rate_coef_core(int j, int tb, int at, int rereac, int sgm, const double* ci, DG dgi,
                                               double T, double lt, double rT, double& w, double& r) {
  double Ctrb = 0.0;
  if (tb == 1) {
#pragma unroll
    for (int i = 0; i < NS; i++) Ctrb = Ctrb + ci[i] * cC.treff[j][i];
  }
  const double wf1 = cC.af[j][0] * exp(cC.bf[j][0] * lt - cC.ef[j][0] * rT);
  if (at == 0) {
    w = wf1;
  } else {
    const double wf2 = cC.af[j][1] * exp(cC.bf[j][1] * lt - cC.ef[j][1] * rT);
    if (at == 2) {
      w = wf1 + wf2;
    } else {  // Troe fall-off
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
  if (rereac == 0) {
    const double Rs = 8.314 / 1.013e5 * 1.0e6;
    double kjx = exp(-dgi() * rT) * powi_rt(Rs * T, -sgm);
    r = w / kjx;
  } else if (rereac == 1) {
    r = cC.ar[j] * exp(cC.br[j] * lt - cC.er[j] * rT);
  } else {
    double z = 10000.0 * rT;
    double kj = exp(cC.park[j][0] + cC.park[j][1] * z + cC.park[j][2] * q2(z) + cC.park[j][3] * q3(z) +
                    cC.park[j][4] * q4(z));
    if (kj < 1.0e-30) kj = 1.0e-30;
    r = w / kj;
  }
  if (tb == 1 && at != 1) {
    w = w * Ctrb;
    r = r * Ctrb;
  }
}
template <int NS>
__device__ __forceinline__ void rate_coef_j(int j, const double* ci, const double* gi, double T, double lt, double rT,
                                            double& w, double& r) {
  auto dgi = [&]() {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < NS; i++) s = s + gi[i] * (double)(cC.vr[j][i] - cC.vf[j][i]);
    return s;
  };
  rate_coef_core<NS>(j, cC.tr_reac[j], cC.af_type[j], cC.rereac, cC.sgm[j], ci, dgi, T, lt, rT, w, r);
}

// rate-of-progress factors: w prod c^vf, r prod c^vr (CHEM_reactions.f90:213-218, 245-250)
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

// Gibbs energies of every species (comput_gibbs) when the reverse rates use Kc
template <int NS>
__device__ __forceinline__ void gibbs_all(double T, double lt, double* gi) {
  if (cC.rereac == 0) {
    const int jc = trange(T);
#pragma unroll
    for (int i = 0; i < NS; i++) gi[i] = dev_gibbs_jc(i, jc, T, lt);
  }
}

}  // namespace ocfd
#include "ocfd_mech_h2air9.cuh"
namespace ocfd {

// Mechanism forms of the kernels: MECH_GENERIC reads the mechanism's structure from the constant
// block; MECH_H2AIR9 runs the compiled 9-species H2-air code (ocfd_mech_h2air9.cuh), which the
// host selects only when the loaded mechanism has exactly that structure.
constexpr int MECH_GENERIC = 0, MECH_H2AIR9 = 1;

// Reaction_rate (CHEM_reactions.f90:203-225)
template <int NS, int MECH = MECH_GENERIC>
__device__ void reaction_rate(const double* ci, double* ri, double T) {
  const double lt = log(T), rT = 1.0 / T;
  double gi[NS];
  gibbs_all<NS>(T, lt, gi);
  if constexpr (MECH == MECH_H2AIR9 && NS == mech_h2air9::NS) {
    mech_h2air9::rates(ci, ri, gi, T, lt, rT);
    return;
  }
#pragma unroll
  for (int i = 0; i < NS; i++) ri[i] = 0.0;
  for (int k = 0; k < cC.nreac; k++) {
    double w, r, wf1, wr1;
    rate_coef_j<NS>(k, ci, gi, T, lt, rT, w, r);
    progress<NS>(ci, w, r, k, wf1, wr1);
#pragma unroll
    for (int i = 0; i < NS; i++) ri[i] = ri[i] + (wf1 - wr1) * (double)(cC.vr[k][i] - cC.vf[k][i]);
  }
}

// Reaction_rate_and_Matrix (CHEM_reactions.f90:230-272): ri and Ar(i, j) = d r_i / d c_j into the
// thread's slab (Ar[i * NS + j]). The division by c_j + 1e-20 is a multiplication by its
// reciprocal, formed once per species (the same quantity up to the last place).
template <int NS, int STRIDE, int MECH = MECH_GENERIC>
__device__ void reaction_rate_matrix(const double* ci, double* ri, Slab<STRIDE> Ar, double T) {
  const double lt = log(T), rT = 1.0 / T;
  double gi[NS], rc[NS];
  gibbs_all<NS>(T, lt, gi);
#pragma unroll
  for (int i = 0; i < NS; i++) {
    ri[i] = 0.0;
    rc[i] = 1.0 / (ci[i] + 1.0e-20);
  }
#pragma unroll
  for (int m = 0; m < NS * NS; m++) Ar[m] = 0.0;
  if constexpr (MECH == MECH_H2AIR9 && NS == mech_h2air9::NS) {
    mech_h2air9::rates_matrix<STRIDE>(ci, rc, ri, Ar, gi, T, lt, rT);
    return;
  }
  for (int k = 0; k < cC.nreac; k++) {
    double w, r, wf1, wr1;
    rate_coef_j<NS>(k, ci, gi, T, lt, rT, w, r);
    progress<NS>(ci, w, r, k, wf1, wr1);
    double s[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) {
      s[i] = (double)(cC.vr[k][i] - cC.vf[k][i]);
      ri[i] = ri[i] + (wf1 - wr1) * s[i];
    }
#pragma unroll
    for (int j = 0; j < NS; j++) {
      const int a = cC.vf[k][j], b = cC.vr[k][j];
      if (a == 0 && b == 0) continue;  // both derivatives are exactly +0: adding them changes nothing
      const double dA = (double)a * wf1 * rc[j] - (double)b * wr1 * rc[j];
#pragma unroll
      for (int i = 0; i < NS; i++) Ar[i * NS + j] = Ar[i * NS + j] + dA * s[i];
      asm volatile("" ::: "memory");  // one column's loads at a time (keeps the register pressure low)
    }
  }
}

// Gauss elimination with partial pivoting (CHEM_reactions.f90:523-567) on the thread's slab
// (row-major NS x NS), right-hand side b in registers, solution into x. Columns left of the pivot
// are never read again, so only columns >= k are updated. Returns true when a pivot was zero
// (the reference then divides by zero; so does this, so the values stay the reference's).
template <int NS, int STRIDE>
__device__ __forceinline__ bool gauss(Slab<STRIDE> a, double* b, double* x) {
  bool zero = false;
#pragma unroll
  for (int k = 0; k < NS - 1; k++) {
    double fmax = fabs(a[k * NS + k]);
    int kk = k;
#pragma unroll
    for (int i = k + 1; i < NS; i++) {
      const double v = fabs(a[i * NS + k]);
      if (v > fmax) {
        fmax = v;
        kk = i;
      }
    }
    zero = zero || fmax == 0.0;
    if (kk != k) {
#pragma unroll
      for (int j = k; j < NS; j++) {
        double t = a[k * NS + j];
        a[k * NS + j] = a[kk * NS + j];
        a[kk * NS + j] = t;
      }
#pragma unroll
      for (int i = k + 1; i < NS; i++)
        if (i == kk) {
          double t = b[k];
          b[k] = b[i];
          b[i] = t;
        }
    }
    double piv[NS];
#pragma unroll
    for (int j = k; j < NS; j++) piv[j] = a[k * NS + j];
#pragma unroll
    for (int i = k + 1; i < NS; i++) {
      double f = -a[i * NS + k] / piv[k];
#pragma unroll
      for (int j = k; j < NS; j++) a[i * NS + j] = a[i * NS + j] + f * piv[j];
      b[i] = b[i] + f * b[k];
      asm volatile("" ::: "memory");  // one row's loads at a time
    }
  }
  const double last = a[(NS - 1) * NS + NS - 1];
  zero = zero || last == 0.0;
  x[NS - 1] = b[NS - 1] / last;
#pragma unroll
  for (int i = NS - 2; i >= 0; i--) {
    double s = b[i];
#pragma unroll
    for (int j = i + 1; j < NS; j++) s = s - a[i * NS + j] * x[j];
    x[i] = s / a[i * NS + i];
  }
  return zero;
}

template <int NS>
__device__ __forceinline__ double update_et(const double* di, const double* dn, double E) {
#pragma unroll
  for (int i = 0; i < NS; i++) E = E - (dn[i] - di[i]) * cC.Ri[i] * cC.cf[i][0][5];
  return E;
}

// chemical_timeAdv (CHEM_reactions.f90:374-390) for one reactor; returns true when the implicit
// step met a zero pivot. A compiled mechanism (MECH != MECH_GENERIC) carries only the linearised
// implicit Euler (the host runs it for CHEM_TimeAdv = -1 alone): its straight-line reaction code
// appears once in the kernel.
template <int NS, int STRIDE, int MECH = MECH_GENERIC>
__device__ __forceinline__ bool chem_step(double* di, double& E, double dt, int* nfail, Slab<STRIDE> sA) {
  double ci[NS], ri[NS], dn[NS];
  const int mode = MECH == MECH_GENERIC ? cC.timeadv : -1;
  bool zero = false;
  if (mode == 1) {
    double T = dev_T<NS>(di, E, nfail);
#pragma unroll
    for (int i = 0; i < NS; i++) ci[i] = di[i] / cC.Mi[i] * 1.0e-6;
    reaction_rate<NS, MECH>(ci, ri, T);
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
    reaction_rate<NS, MECH>(ci, ri, T);
#pragma unroll
    for (int i = 0; i < NS; i++) d1[i] = di[i] + ri[i] * cC.Mi[i] * 1.0e6 * dt;
    E = update_et<NS>(di, d1, E);
    T = dev_T<NS>(di, E, nfail);  // the reference takes T from the old densities here
#pragma unroll
    for (int i = 0; i < NS; i++) ci[i] = d1[i] / cC.Mi[i] * 1.0e-6;
    reaction_rate<NS, MECH>(ci, ri, T);
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
#pragma unroll
    for (int krk = 0; krk < 3; krk++) {
      double T = dev_T<NS>(di, E, nfail);
#pragma unroll
      for (int i = 0; i < NS; i++) ci[i] = di[i] / cC.Mi[i] * 1.0e-6;
      reaction_rate<NS, MECH>(ci, ri, T);
#pragma unroll
      for (int i = 0; i < NS; i++) dn[i] = ra[krk] * d0[i] + rb[krk] * (di[i] + ri[i] * cC.Mi[i] * 1.0e6 * dt);
      E = update_et<NS>(di, dn, E);
#pragma unroll
      for (int i = 0; i < NS; i++) di[i] = dn[i];
    }
  } else {  // -1: linearised backward Euler, (I - J (M_i / M_j) dt) dd = r M 1e6 dt
    double rhs[NS], dd[NS];
    double T = dev_T<NS>(di, E, nfail);
#pragma unroll
    for (int i = 0; i < NS; i++) ci[i] = di[i] / cC.Mi[i] * 1.0e-6;
    reaction_rate_matrix<NS, STRIDE, MECH>(ci, ri, sA, T);
#pragma unroll
    for (int i = 0; i < NS; i++) {
#pragma unroll
      for (int j = 0; j < NS; j++) {
        const double a = (i == j) ? 1.0 : 0.0;
        sA[i * NS + j] = a - sA[i * NS + j] * cC.mratio[i][j] * dt;
      }
      asm volatile("" ::: "memory");
    }
#pragma unroll
    for (int i = 0; i < NS; i++) rhs[i] = ri[i] * cC.Mi[i] * 1.0e6 * dt;
    zero = gauss<NS, STRIDE>(sA, rhs, dd);
#pragma unroll
    for (int i = 0; i < NS; i++) dn[i] = di[i] + dd[i];
    E = update_et<NS>(di, dn, E);
#pragma unroll
    for (int i = 0; i < NS; i++) di[i] = dn[i];
  }
  return zero;
}

// Constant-pressure reactors (an extension for batched 0-D reactors; the reference's reactor and the
// flow solver's cells are constant-volume, OCFD_Time_Adv.f90:174-193). A reactor keeps its initial
// pressure p0 and specific total enthalpy h0 = (E + sum d_k R_k F_k + p) / rho (F_k the formation
// term that update_Et books). After each constant-volume sub-step the mixture is brought back to
// p0 at h0 with the mass fractions fixed: Newton on T for e(T, Y) + R T + sum Y_k R_k F_k = h0 (e
// from comput_E with Y as densities, derivative the mass-specific Cp), stopped when |dT| <= 1e-10 T
// (at most 50 iterations), then rho = p0 / (R T), d = Y rho, E = comput_E(d, T). The oracle applies
// the identical operations.
template <int NS>
__device__ __forceinline__ void cp_reference(const double* di, double Et, double& h0, double& p0, int* nfail) {
  const double T = dev_T<NS>(di, Et, nfail);
  p0 = dev_P<NS>(di, T);
  double rho = 0.0, cf = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    rho = rho + di[k];
    cf = cf + di[k] * cC.Ri[k] * cC.cf[k][0][5];
  }
  h0 = (Et + cf + p0) / rho;
}
template <int NS>
__device__ __forceinline__ void cp_restore(double* di, double& Et, double h0, double p0, int* nfail) {
  double rho = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) rho = rho + di[k];
  double Y[NS];
  double R1 = 0.0, cf = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    Y[k] = di[k] / rho;
    R1 = R1 + cC.Ri[k] * Y[k];
    cf = cf + Y[k] * cC.Ri[k] * cC.cf[k][0][5];
  }
  double T = dev_T<NS>(di, Et, nfail);
  for (int it = 0; it < 50; it++) {
    const double g = dev_E<NS>(Y, T) + R1 * T + cf - h0;
    const double dT = g / dev_Cp<NS>(1.0, Y, T);
    T = T - dT;
    if (fabs(dT) <= 1.0e-10 * T) break;
  }
  const double r1 = p0 / (R1 * T);
#pragma unroll
  for (int k = 0; k < NS; k++) di[k] = Y[k] * r1;
  Et = dev_E<NS>(di, T);
}

// a reactor's result is an error when a pivot was zero or a density or the energy is not finite
template <int NS>
__device__ __forceinline__ void chem_check(const double* di, double E, bool zero, int* nfail) {
  bool bad = zero || !isfinite(E);
#pragma unroll
  for (int m = 0; m < NS; m++) bad = bad || !isfinite(di[m]);
  if (bad && nfail) atomicAdd(nfail + 1, 1);
}

template <int NS, int MECH = MECH_GENERIC>
__global__ void __launch_bounds__(OCFD_CHEM_TPB, OCFD_CHEM_MINB) k_chem_cells(double* f, double* Et, double* T,
                                                                             double* p, double* di, double dt2,
                                                                             int nsub, int* nfail) {
  __shared__ double sA[NS * NS * OCFD_CHEM_TPB];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cC.N) return;
  int i = t % cC.nx + 1, j = (t / cC.nx) % cC.ny + 1, k = t / cC.nx / cC.ny + 1;
  const int q = hidx(i, j, k);
  double d1[NS];
#pragma unroll
  for (int m = 0; m < NS; m++) d1[m] = di[(size_t)m * cC.H + q];
  double e = Et[q];
  double f5 = f[4 * cC.N + t];
  bool zero = false;
  const Slab<OCFD_CHEM_TPB> slab{sA + threadIdx.x};
  for (int s = 0; s < nsub; s++) {
    double e0 = e;
    zero = chem_step<NS, OCFD_CHEM_TPB, MECH>(d1, e, dt2, nfail, slab) || zero;
    f5 = f5 + (e - e0);
  }
  chem_check<NS>(d1, e, zero, nfail);
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

// CP: constant-pressure reactors (a template parameter, so the reference's constant-volume form
// carries none of the pressure-restoring code in its registers)
template <int NS, bool CP, int MECH = MECH_GENERIC>
__global__ void __launch_bounds__(OCFD_CHEM_TPB, OCFD_CHEM_MINB) k_chem_batch(int n, double* di, double* e,
                                                                             const double* dt, const int* nsub,
                                                                             const int* perm, int* counter,
                                                                             int* nfail) {
  __shared__ double sA[NS * NS * OCFD_CHEM_TPB];
  const int lane = threadIdx.x & 31;
  const Slab<OCFD_CHEM_TPB> slab{sA + threadIdx.x};
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
      bool zero = false;
      if (CP) {
        double h0, p0;
        cp_reference<NS>(d1, ee, h0, p0, nfail);
        for (int s = 0; s < ks; s++) {
          zero = chem_step<NS, OCFD_CHEM_TPB, MECH>(d1, ee, dt2, nfail, slab) || zero;
          cp_restore<NS>(d1, ee, h0, p0, nfail);
        }
      } else {
        for (int s = 0; s < ks; s++) zero = chem_step<NS, OCFD_CHEM_TPB, MECH>(d1, ee, dt2, nfail, slab) || zero;
      }
      chem_check<NS>(d1, ee, zero, nfail);
#pragma unroll
      for (int m = 0; m < NS; m++) di[(size_t)r * NS + m] = d1[m];
      e[r] = ee;
    }
  }
}

// ---- warp-cooperative implicit Euler (batched reactors) ----
// The same linearised backward-Euler step, one reactor per group of NS lanes (lane s of a group
// owns species s: its density, row s of the matrix and of the right-hand side); 32 / NS reactors per
// warp. The reactions are spread over the group's lanes (lane s evaluates reactions s, s + NS, ...)
// and their rates of progress exchanged through shared memory; each lane then accumulates its own
// row of the Jacobian in registers, over the reactions in order, with the serial kernel's
// expressions; the pivot search, the row swap and the pivot row of the Gauss elimination go through
// shared memory, and the back substitution keeps the serial order. Every value is formed by the same
// operations in the same order as in chem_step, so both kernels give the same numbers bit for bit.
// Per reactor it has a fraction of the serial kernel's latency per sub-step, which decides the time
// of a batch too small to fill the GPU (a few stiff reactors with many sub-steps, such as the
// reactors the surrogate's gate rejects: the gated pass of 2^20 reactor states 9.45 -> 4.65 ms);
// its throughput on batches that fill the GPU is a fifth of the serial kernel's, which therefore
// keeps those (launch_chem_batch picks by the batch size).
// The group's lanes run warp-synchronously: every lane of the warp executes every sub-step (a warp
// loops to the largest sub-step count of its reactors; reactors with fewer sub-steps, and the idle
// lanes above 32 / NS groups, compute without keeping the result).
template <int NS>
struct CoopArea {
  double d[NS], rc[NS], gi[NS], col[NS], x[NS], dn[NS];
  double rowA[NS + 1], rowB[NS + 1], piv[NS + 1];
  double wf[OCFD_MAX_REAC], wr[OCFD_MAX_REAC];
};
constexpr int COOP_THREADS = 64;  // two warps: the areas of 32 / NS reactors per warp stay small

template <int NS>
__device__ __forceinline__ void coop_implicit_step(CoopArea<NS>& A, int s, double& d_own, double& E, double dt,
                                                   bool live, bool& zero, int* nfail) {
  // every lane of the group gathers the reactor's densities
  A.d[s] = d_own;
  __syncwarp();
  double d[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) d[k] = A.d[k];
  const double T = dev_T<NS>(d, E, (live && s == 0) ? nfail : nullptr);
  double ci[NS];
#pragma unroll
  for (int i = 0; i < NS; i++) ci[i] = d[i] / cC.Mi[i] * 1.0e-6;
  const double lt = log(T), rT = 1.0 / T;
  A.rc[s] = 1.0 / (ci[s] + 1.0e-20);
  if (cC.rereac == 0) A.gi[s] = dev_gibbs_jc(s, trange(T), T, lt);
  __syncwarp();
  double gi[NS];
#pragma unroll
  for (int i = 0; i < NS; i++) gi[i] = A.gi[i];
  // the group's reactions, spread over its lanes
  for (int k = s; k < cC.nreac; k += NS) {
    double w, r, wf1, wr1;
    rate_coef_j<NS>(k, ci, gi, T, lt, rT, w, r);
    progress<NS>(ci, w, r, k, wf1, wr1);
    A.wf[k] = wf1;
    A.wr[k] = wr1;
  }
  __syncwarp();
  double rc[NS];
#pragma unroll
  for (int j = 0; j < NS; j++) rc[j] = A.rc[j];
  // row s of Reaction_rate_and_Matrix, reactions in order
  double ri = 0.0, row[NS];
#pragma unroll
  for (int j = 0; j < NS; j++) row[j] = 0.0;
  for (int k = 0; k < cC.nreac; k++) {
    const double wf1 = A.wf[k], wr1 = A.wr[k];
    const double si = (double)(cC.vr[k][s] - cC.vf[k][s]);
    ri = ri + (wf1 - wr1) * si;
#pragma unroll
    for (int j = 0; j < NS; j++) {
      const int a = cC.vf[k][j], b = cC.vr[k][j];
      if (a == 0 && b == 0) continue;
      const double dA = (double)a * wf1 * rc[j] - (double)b * wr1 * rc[j];
      row[j] = row[j] + dA * si;
    }
  }
#pragma unroll
  for (int j = 0; j < NS; j++) {
    const double a = (s == j) ? 1.0 : 0.0;
    row[j] = a - row[j] * cC.mratio[s][j] * dt;
  }
  double rhs = ri * cC.Mi[s] * 1.0e6 * dt;
  // Gauss elimination with partial pivoting across the group's rows
#pragma unroll
  for (int k = 0; k < NS - 1; k++) {
    A.col[s] = fabs(row[k]);
    __syncwarp();
    double fmax = A.col[k];
    int kk = k;
#pragma unroll
    for (int i = k + 1; i < NS; i++) {
      const double v = A.col[i];
      if (v > fmax) {
        fmax = v;
        kk = i;
      }
    }
    zero = zero || fmax == 0.0;
    if (kk != k) {  // rows k and kk trade places (columns >= k and the right-hand side)
      if (s == k) {
#pragma unroll
        for (int j = k; j < NS; j++) A.rowA[j] = row[j];
        A.rowA[NS] = rhs;
      }
      if (s == kk) {
#pragma unroll
        for (int j = k; j < NS; j++) A.rowB[j] = row[j];
        A.rowB[NS] = rhs;
      }
    }
    __syncwarp();
    if (kk != k) {
      if (s == k) {
#pragma unroll
        for (int j = k; j < NS; j++) row[j] = A.rowB[j];
        rhs = A.rowB[NS];
      }
      if (s == kk) {
#pragma unroll
        for (int j = k; j < NS; j++) row[j] = A.rowA[j];
        rhs = A.rowA[NS];
      }
    }
    if (s == k) {
#pragma unroll
      for (int j = k; j < NS; j++) A.piv[j] = row[j];
      A.piv[NS] = rhs;
    }
    __syncwarp();
    if (s > k) {
      const double f = -row[k] / A.piv[k];
#pragma unroll
      for (int j = k; j < NS; j++) row[j] = row[j] + f * A.piv[j];
      rhs = rhs + f * A.piv[NS];
    }
    __syncwarp();
  }
  // back substitution in the serial order: x(NS-1), then x(i) = (b(i) - sum_j>i a(i,j) x(j)) / a(i,i)
  if (s == NS - 1) A.x[NS - 1] = rhs / row[NS - 1];
  __syncwarp();
#pragma unroll
  for (int i = NS - 2; i >= 0; i--) {
    if (s == i) {
      double sacc = rhs;
#pragma unroll
      for (int j = i + 1; j < NS; j++) sacc = sacc - row[j] * A.x[j];
      A.x[i] = sacc / row[i];
    }
    __syncwarp();
  }
  {
    // the last pivot's test (made by lane NS-1 above) for the whole group
    A.col[s] = (s == NS - 1 && row[NS - 1] == 0.0) ? 1.0 : 0.0;
    __syncwarp();
    zero = zero || A.col[NS - 1] != 0.0;
  }
  const double dn = d_own + A.x[s];
  A.dn[s] = dn;
  __syncwarp();
  double En = E;
#pragma unroll
  for (int i = 0; i < NS; i++) En = En - (A.dn[i] - d[i]) * cC.Ri[i] * cC.cf[i][0][5];
  __syncwarp();  // the area is rewritten by the next sub-step
  if (live) {
    d_own = dn;
    E = En;
  }
}

template <int NS, bool CP>
__global__ void __launch_bounds__(COOP_THREADS) k_chem_batch_coop(int n, double* di, double* e, const double* dt,
                                                                  const int* nsub, const int* perm, int* counter,
                                                                  int* nfail) {
  constexpr int G = 32 / NS;  // reactors per warp
  __shared__ CoopArea<NS> area[COOP_THREADS / 32][G + 1];  // the last area is the idle lanes' sink
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int g = lane / NS, s = lane - g * NS;
  const bool lane_ok = g < G;
  CoopArea<NS>& A = area[wq][lane_ok ? g : G];
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(counter, G);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const int idx = base + g;
    const bool act = lane_ok && idx < n;
    const int r = act ? perm[idx] : 0;
    const int ks = act ? (nsub ? nsub[r] : 1) : 0;
    int kmax = ks;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    const double dt2 = act ? dt[r] / ks : 0.0;
    double d_own = act ? di[(size_t)r * NS + s] : 1.0;
    double E = act ? e[r] : 1.0;
    double h0 = 0.0, p0 = 0.0;
    int* nf0 = (act && s == 0) ? nfail : nullptr;  // one lane per reactor counts Newton failures
    if (CP) {
      A.d[s] = d_own;
      __syncwarp();
      double d[NS];
#pragma unroll
      for (int k = 0; k < NS; k++) d[k] = A.d[k];
      __syncwarp();
      cp_reference<NS>(d, E, h0, p0, nf0);
    }
    bool zero = false;
    for (int st = 0; st < kmax; st++) {
      const bool live = act && st < ks;
      coop_implicit_step<NS>(A, s, d_own, E, dt2, live, zero, nfail);
      if (CP) {
        A.d[s] = d_own;
        __syncwarp();
        double d[NS];
#pragma unroll
        for (int k = 0; k < NS; k++) d[k] = A.d[k];
        __syncwarp();
        double Ec = E;
        cp_restore<NS>(d, Ec, h0, p0, live ? nf0 : nullptr);
        if (live) {
          d_own = d[s];
          E = Ec;
        }
      }
    }
    // error check of the reactor: zero pivot or a non-finite density / energy in the group
    A.col[s] = (isfinite(d_own) && isfinite(E)) ? 0.0 : 1.0;
    __syncwarp();
    bool bad = zero;
#pragma unroll
    for (int k = 0; k < NS; k++) bad = bad || A.col[k] != 0.0;
    __syncwarp();
    if (act) {
      di[(size_t)r * NS + s] = d_own;
      if (s == 0) {
        e[r] = E;
        if (bad && nfail) atomicAdd(nfail + 1, 1);
      }
    }
  }
}

}  // namespace ocfd
