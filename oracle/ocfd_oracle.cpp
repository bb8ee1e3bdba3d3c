/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle of the OpenCFD-Comb per-step hot path.
 *
 * This file restates the reference's Fortran in C++, loop by loop and in its expression
 * order, so that it can judge the CUDA implementation in opencfd-comb_b200/. It is loaded
 * only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline; the product never
 * includes or links it. Parity with the Fortran binary itself is unpinned: the reference
 * cannot be compiled here (no Fortran compiler, no MPI) and its own tests hold no golden
 * outputs, so this restatement is the reference behaviour the tests pin.
 *
 * Reference files restated (paths inside the OpenCFD-Comb tree):
 *   code/flow-solver/OCFD_Time_Adv.f90      flow_time_advance :7-92, RK3 :98-166,
 *                                           Chemical_time_advance :169-196, show_flow_msg :210-223
 *   code/flow-solver/OCFD_inviscous.f90     du_inviscous :47-202, OCFD2d_flux1/2 :209-362
 *   code/flow-solver/OCFD_flux_split.f90    split_Stager_Warming :6-73, split_Local_LaxFriedrichs :76-103
 *   code/flow-solver/OCFD_viscous.f90       du_viscous :27-131
 *   code/flow-solver/OCFD_scaler_inviscous.f90, OCFD_scaler_viscous.f90 (species transport)
 *   code/flow-solver/Comput_flow_variables.f90 (prims, T/p, cc, transport coefficients, Rescaling_di)
 *   code/others/OCFD_handle_NegativeT.f90
 *   code/schemes/OCFD_dxyz_viscous.f90      OCFD_dx0/dy0/dz0 (CD6/CD8 + closures)
 *   code/schemes/OCFD_SetHybrid.f90         set_hybrid_scheme :2-15, comput_Rhybrid :17-143
 *   code/boundary-condition/OCFD_BC.f90     OCFD_bc :2-188 (face re-derivation)
 *   code/boundary-condition/OCFD_BC_Boundarylayers.f90 ocfd_bc_BoundaryLayer :20-243, init_bc_nonRef :448-487
 *   code/boundary-condition/OCFD_GhostCell.f90 Flow_Ghost_Extent_2nd :166-364
 *   code/flow-solver/OCFD_mesh.f90          init_mesh :1-57, comput_Jacobian3d :60-107, updata_Axyz_periodic :109-185
 *   code/mpi-io/OCFD_mpi.f90                exchange_boundary_x/y/z :201-236 (single rank: periodic copy)
 *   code/mpi-io/OCFD_readpara.f90           set_parameters :347-409, set_scheme_para :424-431
 *   code/others/OCFD_filtering.f90          filtering :4-72, Fo9p filters :78-189, shock filters :194-360
 *   code/others/OCFD_ANA.f90                ana_time_average :39-140, ana_getQ :143-190, ana_box :197-303
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/ocfd_gpu.h"
#include "ocfd_oracle_chem.h"
#include "ocfd_oracle_schemes.h"

using namespace ocfd_oracle;

namespace {

enum { M_AKX = 0, M_AKY, M_AKZ, M_AIX, M_AIY, M_AIZ, M_ASX, M_ASY, M_ASZ, M_AJAC, M_AKX1, M_AKY1, M_AKZ1, M_AIX1,
       M_AIY1, M_AIZ1, M_ASX1, M_ASY1, M_ASZ1, M_NUM };

struct Oracle {
  ocfd_params P;
  Chem ch;
  SchemeSet S;
  int nx, ny, nz, L, NS;
  long HX, HY, HZ, H, N;
  double hx, hy, hz;
  int bound[3][2];
  int bcdata_inlet = 0, bcdata_upper = 0;
  std::vector<double> inlet, upper, wall_pertb, tm, fait;
  std::vector<int> nonref;

  std::vector<double> f, fn, du, d, u, v, w, T, p, Et, cc, di, din, Amu, Amk, AmD, X, Y, Z, Rh, Ev1, Ev2, Ev3,
      dk[12], Qpx, Qpy, Qpz;
  std::vector<double> M[M_NUM];
  long neg_et = 0;
  std::string err;

  long ih(int i, int j, int k) const { return (long)(i + L - 1) + HX * ((long)(j + L - 1) + HY * (long)(k + L - 1)); }
  long in(int i, int j, int k) const { return (long)(i - 1) + (long)nx * ((long)(j - 1) + (long)ny * (long)(k - 1)); }

  /* ---------------- halo exchange (single rank) ---------------- */
  void exch_x(double* a) {
    if (!P.iperiodic[0]) return;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int l = 0; l < L; l++) {
          a[ih(nx + 1 + l, j, k)] = a[ih(1 + l, j, k)];
          a[ih(1 - L + l, j, k)] = a[ih(nx + 1 - L + l, j, k)];
        }
  }
  void exch_y(double* a) {
    if (!P.iperiodic[1]) return;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int l = 0; l < L; l++)
        for (int i = 1; i <= nx; i++) {
          a[ih(i, ny + 1 + l, k)] = a[ih(i, 1 + l, k)];
          a[ih(i, 1 - L + l, k)] = a[ih(i, ny + 1 - L + l, k)];
        }
  }
  void exch_z(double* a) {
    if (!P.iperiodic[2]) return;
#pragma omp parallel for collapse(2)
    for (int l = 0; l < L; l++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          a[ih(i, j, nz + 1 + l)] = a[ih(i, j, 1 + l)];
          a[ih(i, j, 1 - L + l)] = a[ih(i, j, nz + 1 - L + l)];
        }
  }
  void exch(double* a) {
    exch_x(a);
    exch_y(a);
    exch_z(a);
  }

  /* ---------------- OCFD_dx0 / dy0 / dz0 ---------------- */
  void dxyz(int dir, const double* fa, double* fx) {
    int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
    double h = dir == 0 ? hx : (dir == 1 ? hy : hz);
    long s = dir == 0 ? 1 : (dir == 1 ? HX : HX * HY);
    double a1 = 1.0 / (60.0 * h), a2 = -3.0 / (20.0 * h), a3 = 3.0 / (4.0 * h);
    double c1 = 0.8 / h, c2 = -0.2 / h, c3 = 3.80952380952380952e-2 / h, c4 = -3.571428571428571428e-3 / h;
    bool cd8 = P.scheme_vis == OCFD_SCHEME_CD8;
    bool nonper = P.iperiodic[dir] == 0;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          const double* q = fa + ih(i, j, k);
          int ii = dir == 0 ? i : (dir == 1 ? j : k);
          double r;
          if (!cd8)
            r = a1 * (q[3 * s] - q[-3 * s]) + a2 * (q[2 * s] - q[-2 * s]) + a3 * (q[s] - q[-s]);
          else
            r = c1 * (q[s] - q[-s]) + c2 * (q[2 * s] - q[-2 * s]) + c3 * (q[3 * s] - q[-3 * s]) +
                c4 * (q[4 * s] - q[-4 * s]);
          if (nonper) {
            /* q[m*s] is f at offset m from this point; closures use interior points only */
            if (ii == 1) r = (-3.0 * q[0] + 4.0 * q[s] - q[2 * s]) / (2.0 * h);
            else if (ii == 2) r = (q[s] - q[-s]) / (2.0 * h);
            else if (ii == 3) r = (8.0 * (q[s] - q[-s]) - (q[2 * s] - q[-2 * s])) / (12.0 * h);
            else if (cd8 && ii == 4) r = a1 * (q[3 * s] - q[-3 * s]) + a2 * (q[2 * s] - q[-2 * s]) + a3 * (q[s] - q[-s]);
            if (ii == n) r = (q[-2 * s] - 4.0 * q[-s] + 3.0 * q[0]) / (2.0 * h);
            else if (ii == n - 1) r = (q[s] - q[-s]) / (2.0 * h);
            else if (ii == n - 2) r = (8.0 * (q[s] - q[-s]) - (q[2 * s] - q[-2 * s])) / (12.0 * h);
            else if (cd8 && ii == n - 3) r = a1 * (q[3 * s] - q[-3 * s]) + a2 * (q[2 * s] - q[-2 * s]) + a3 * (q[s] - q[-s]);
          }
          fx[in(i, j, k)] = r;
        }
  }

  /* ---------------- init ---------------- */
  int init(const ocfd_params* pp, const ocfd_thermo* th, const ocfd_kinetics* kin, const ocfd_transport* tr,
           const ocfd_bcdata* bc, const double* coords, const double* metrics) {
    P = *pp;
    nx = P.nx; ny = P.ny; nz = P.nz; L = P.lap; NS = P.n_spec;
    if (L != 4 || NS < 1 || NS > OCFD_MAX_SPEC || nx < 8 || ny < 8 || nz < 8) { err = "bad sizes"; return OCFD_ERR_PARAM; }
    for (int m = 0; m < 6; m++)
      if (P.ghost_cell[m] < 0 || P.ghost_cell[m] > 2) { err = "Ghost_Cell must be 0, 1 or 2"; return OCFD_ERR_UNSUPPORTED; }
    HX = nx + 2 * L; HY = ny + 2 * L; HZ = nz + 2 * L; H = HX * HY * HZ; N = (long)nx * ny * nz;
    hx = 1.0 / (nx - 1.0); hy = 1.0 / (ny - 1.0); hz = 1.0 / (nz - 1.0);
    for (int dd = 0; dd < 3; dd++) bound[dd][0] = bound[dd][1] = P.iperiodic[dd] == 0 ? 1 : 0;
    S.scheme = P.scheme_invis;
    switch (S.scheme) {
      case 1: S.Ka1 = -2; S.Kb1 = 2; S.Ka2 = -1; S.Kb2 = 3; break;
      case 2: S.Ka1 = -3; S.Kb1 = 3; S.Ka2 = -2; S.Kb2 = 4; break;
      case 3: case 4: case 10: S.Ka1 = -3; S.Kb1 = 4; S.Ka2 = -3; S.Kb2 = 4; break;
      default: err = "scheme"; return OCFD_ERR_PARAM;
    }
    {
      const double UD7[8] = {-3.0, 25.0, -101.0, 319.0, 214.0, -38.0, 4.0, 0.0};
      const double CD8[8] = {-3.0, 29.0, -139.0, 533.0, 533.0, -139.0, 29.0, -3.0};
      for (int k = 0; k < 8; k++) S.UD7L[k] = P.ud7l_diss * UD7[k] / 420.0 + (1.0 - P.ud7l_diss) * CD8[k] / 840.0;
    }
    S.theta1 = P.hybrid_para[1];
    S.theta2 = P.hybrid_para[2];
    ch.set_thermo(th, P.if_realgas);
    ch.tr = *tr;
    ch.timeadv = P.chem_timeadv;
    if (kin) { ch.kin = *kin; ch.nreac = kin->n_reac; ch.have_kin = true; }

    auto alloc = [&](std::vector<double>& a, long n, double val) { a.assign(n, val); };
    alloc(f, 5 * N, 0); alloc(fn, 5 * N, 0); alloc(du, 5 * N, 0);
    /* allocate_flow_data (OCFD_allocate_data.f90:53-56) initial values */
    alloc(d, H, 1.0); alloc(u, H, 1.0); alloc(v, H, 1.0); alloc(w, H, 1.0); alloc(T, H, 300.0);
    alloc(p, H, 1.0); alloc(cc, H, 1.0); alloc(Et, H, 1.0);
    alloc(di, H * NS, 1.0); alloc(din, N * NS, 1.0);
    alloc(Amu, N, 0); alloc(Amk, N, 0); alloc(AmD, N * NS, 0);
    alloc(Rh, H, 0.0);
    alloc(Ev1, 4 * H, 0); alloc(Ev2, 4 * H, 0); alloc(Ev3, 4 * H, 0);
    for (int m = 0; m < 12; m++) alloc(dk[m], N, 0);
    alloc(Qpx, N, 0); alloc(Qpy, N, 0); alloc(Qpz, N, 0);
    alloc(X, H, 1.0); alloc(Y, H, 1.0); alloc(Z, H, 1.0);
    for (int m = 0; m < M_NUM; m++) alloc(M[m], H, 1.0);

    /* init_mesh */
    std::memcpy(X.data(), coords, sizeof(double) * H);
    std::memcpy(Y.data(), coords + H, sizeof(double) * H);
    std::memcpy(Z.data(), coords + 2 * H, sizeof(double) * H);
    exch(X.data()); exch(Y.data()); exch(Z.data());
    periodic_shift();
    if (metrics) {
      for (int m = 0; m < 10; m++) std::memcpy(M[m].data(), metrics + m * H, sizeof(double) * H);
    } else {
      jacobian();
    }
    for (int m = 0; m < 10; m++) exch(M[m].data());
    jac_ghost();
    for (long q = 0; q < H; q++) {
      double jac = M[M_AJAC][q];
      for (int m = 0; m < 9; m++) M[M_AKX1 + m][q] = M[M_AKX + m][q] / jac;
    }

    /* jet inflow data: a 2-D inlet table (ocfd_bc_jet forces BcData_inlet = 2, no upper data) */
    if (P.ibc == OCFD_BC_JET) {
      if (!bc) { err = "bcdata"; return OCFD_ERR_PARAM; }
      bcdata_inlet = 2;
      bcdata_upper = -1;
      inlet.assign(bc->inlet, bc->inlet + (long)(5 + NS) * ny * nz);
    }
    /* boundary-layer data */
    if (P.ibc == OCFD_BC_BOUNDARYLAYER) {
      if (!bc) { err = "bcdata"; return OCFD_ERR_PARAM; }
      bcdata_inlet = (int)std::lround(P.bc_para[0]);
      bcdata_upper = (int)std::lround(P.bc_para[1]);
      int nv = 5 + NS;
      long ni = bcdata_inlet == 0 ? nv : (bcdata_inlet == 1 ? (long)nv * ny : (long)nv * ny * nz);
      long nu = bcdata_upper == 0 ? nv : (bcdata_upper == 1 ? (long)nv * nx : (long)nv * nx * nz);
      inlet.assign(bc->inlet, bc->inlet + ni);
      if (bcdata_upper >= 0) upper.assign(bc->upper, bc->upper + nu);
      wall_pertb.assign((long)nx * nz, 0.0);
      if (bc->wall_pertb) wall_pertb.assign(bc->wall_pertb, bc->wall_pertb + (long)nx * nz);
      tm.assign(bc->tm, bc->tm + bc->n_tm);
      fait.assign(bc->fait, bc->fait + bc->n_tm);
      /* init_bc_nonRef (OCFD_BC_Boundarylayers.f90:448-487) */
      nonref.assign((long)nx * nz, 0);
      int mode = (int)std::lround(P.bc_para[2]);
      double sy0 = std::tan(P.aoa);
      for (int k = 1; k <= nz; k++)
        for (int i = 1; i <= nx; i++) {
          int val = 0;
          if (mode == 1) val = 1;
          else if (mode == 0) {
            double sy;
            if (i == 1) sy = (Y[ih(i + 1, ny, k)] - Y[ih(i, ny, k)]) / (X[ih(i + 1, ny, k)] - X[ih(i, ny, k)]);
            else sy = (Y[ih(i, ny, k)] - Y[ih(i - 1, ny, k)]) / (X[ih(i, ny, k)] - X[ih(i - 1, ny, k)]);
            val = (sy >= sy0 + 1.0e-6) ? 0 : 1;
          }
          nonref[(i - 1) + (long)nx * (k - 1)] = val;
        }
    }
    return 0;
  }

  /* Jac_Ghost_boundary (OCFD_GhostCell.f90:1-6): on every face with Ghost_Cell = 1 the ghost
   * slab (LAP planes outside the face, tangential interior range) copies the face plane's metrics
   * and extrapolates the coordinates linearly (Jac_Ghost_Extent_1st, :18-160); with Ghost_Cell = 2
   * the coordinates are mirrored (x_g = 2 x_b - x_mirror) and the metrics recomputed in the slab
   * by comput_Jacobian3d_Ghost (:366-580), whose derivatives are one-sided at the ends of each
   * range, 2nd-order central next to them and 4th-order central elsewhere. */
  void jac_ghost() {
    for (int pass = 1; pass <= 2; pass++)
      for (int face = 0; face < 6; face++) {
        if (P.ghost_cell[face] != pass) continue;
        const int dir = face / 2, side = face % 2;
        const int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
        const int ta = dir == 0 ? ny : nx, tb = dir == 2 ? ny : nz; /* tangential sizes */
        auto at = [&](int s, int a, int b) {
          return dir == 0 ? ih(s, a, b) : (dir == 1 ? ih(a, s, b) : ih(a, b, s));
        };
        const int g0 = side == 0 ? 1 - L : n + 1, g1 = side == 0 ? 0 : n + L;
        const int ib = side == 0 ? 1 : n;
        for (int b = 1; b <= tb; b++)
          for (int a = 1; a <= ta; a++)
            for (int g = g0; g <= g1; g++) {
              long qg = at(g, a, b), qb = at(ib, a, b);
              if (pass == 1) {
                for (int m = 0; m < 10; m++) M[m][qg] = M[m][qb];
                long q2 = at(side == 0 ? 2 : n - 1, a, b);
                double f = side == 0 ? (1.0 - g) : (double)(g - n);
                X[qg] = X[qb] + f * (X[qb] - X[q2]);
                Y[qg] = Y[qb] + f * (Y[qb] - Y[q2]);
                Z[qg] = Z[qb] + f * (Z[qb] - Z[q2]);
              } else {
                long qm = at(side == 0 ? 2 - g : 2 * n - g, a, b);
                X[qg] = 2.0 * X[qb] - X[qm];
                Y[qg] = 2.0 * Y[qb] - Y[qm];
                Z[qg] = 2.0 * Z[qb] - Z[qm];
              }
            }
        if (pass == 2) {
          /* derivative ranges: [lo, hi] along each direction */
          int lo[3] = {1, 1, 1}, hi[3] = {nx, ny, nz};
          lo[dir] = side == 0 ? 1 - L : n;
          hi[dir] = side == 0 ? 1 : n + L;
          const double hh[3] = {hx, hy, hz};
          const long st[3] = {1, HX, HX * HY};
          auto der = [&](const std::vector<double>& A, long q, int dd, int pos) {
            const double* f = A.data() + q;
            const long s = st[dd];
            const double h = hh[dd];
            if (pos == lo[dd]) return (-3.0 * f[0] + 4.0 * f[s] - f[2 * s]) / (2.0 * h);
            if (pos == hi[dd]) return (f[-2 * s] - 4.0 * f[-s] + 3.0 * f[0]) / (2.0 * h);
            if (pos == lo[dd] + 1 || pos == hi[dd] - 1) return (f[s] - f[-s]) / (2.0 * h);
            return (8.0 * (f[s] - f[-s]) - (f[2 * s] - f[-2 * s])) / (12.0 * h);
          };
          for (int b = 1; b <= tb; b++)
            for (int a = 1; a <= ta; a++)
              for (int g = g0; g <= g1; g++) {
                int i = dir == 0 ? g : a, j = dir == 0 ? a : (dir == 1 ? g : b), k = dir == 2 ? g : b;
                if (dir == 2) { i = a; j = b; }
                long q = ih(i, j, k);
                int pos[3] = {i, j, k};
                double xi1 = der(X, q, 0, pos[0]), yi1 = der(Y, q, 0, pos[0]), zi1 = der(Z, q, 0, pos[0]);
                double xj1 = der(X, q, 1, pos[1]), yj1 = der(Y, q, 1, pos[1]), zj1 = der(Z, q, 1, pos[1]);
                double xk1 = der(X, q, 2, pos[2]), yk1 = der(Y, q, 2, pos[2]), zk1 = der(Z, q, 2, pos[2]);
                double jac = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1 - zi1 * yj1 * xk1 -
                                    yi1 * xj1 * zk1 - xi1 * zj1 * yk1);
                M[M_AJAC][q] = jac;
                M[M_AKX][q] = jac * (yj1 * zk1 - zj1 * yk1);
                M[M_AKY][q] = jac * (zj1 * xk1 - xj1 * zk1);
                M[M_AKZ][q] = jac * (xj1 * yk1 - yj1 * xk1);
                M[M_AIX][q] = jac * (yk1 * zi1 - zk1 * yi1);
                M[M_AIY][q] = jac * (zk1 * xi1 - xk1 * zi1);
                M[M_AIZ][q] = jac * (xk1 * yi1 - yk1 * xi1);
                M[M_ASX][q] = jac * (yi1 * zj1 - zi1 * yj1);
                M[M_ASY][q] = jac * (zi1 * xj1 - xi1 * zj1);
                M[M_ASZ][q] = jac * (xi1 * yj1 - yi1 * xj1);
              }
        }
      }
  }

  void periodic_shift() {
    for (int dd = 0; dd < 3; dd++) {
      if (!P.iperiodic[dd]) continue;
      const double* sp = P.periodic_span[dd];
      for (int k = 1 - L; k <= nz + L; k++)
        for (int j = 1 - L; j <= ny + L; j++)
          for (int i = 1 - L; i <= nx + L; i++) {
            int ii = dd == 0 ? i : (dd == 1 ? j : k);
            bool inside_other = (dd == 0) ? (j >= 1 && j <= ny && k >= 1 && k <= nz)
                                : (dd == 1) ? (i >= 1 && i <= nx && k >= 1 && k <= nz)
                                            : (i >= 1 && i <= nx && j >= 1 && j <= ny);
            if (!inside_other) continue;
            int n = dd == 0 ? nx : (dd == 1 ? ny : nz);
            long q = ih(i, j, k);
            if (ii <= 0) { X[q] = X[q] - sp[0]; Y[q] = Y[q] - sp[1]; Z[q] = Z[q] - sp[2]; }
            else if (ii > n) { X[q] = X[q] + sp[0]; Y[q] = Y[q] + sp[1]; Z[q] = Z[q] + sp[2]; }
          }
    }
  }

  void jacobian() {
    std::vector<double> xi(N), xj(N), xk(N), yi(N), yj(N), yk(N), zi(N), zj(N), zk(N);
    dxyz(0, X.data(), xi.data()); dxyz(0, Y.data(), yi.data()); dxyz(0, Z.data(), zi.data());
    dxyz(1, X.data(), xj.data()); dxyz(1, Y.data(), yj.data()); dxyz(1, Z.data(), zj.data());
    dxyz(2, X.data(), xk.data()); dxyz(2, Y.data(), yk.data()); dxyz(2, Z.data(), zk.data());
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long a = in(i, j, k), q = ih(i, j, k);
          double xi1 = xi[a], xj1 = xj[a], xk1 = xk[a], yi1 = yi[a], yj1 = yj[a], yk1 = yk[a], zi1 = zi[a], zj1 = zj[a],
                 zk1 = zk[a];
          double jac = 1.0 / (xi1 * yj1 * zk1 + yi1 * zj1 * xk1 + zi1 * xj1 * yk1 - zi1 * yj1 * xk1 - yi1 * xj1 * zk1 -
                              xi1 * zj1 * yk1);
          M[M_AJAC][q] = jac;
          M[M_AKX][q] = jac * (yj1 * zk1 - zj1 * yk1);
          M[M_AKY][q] = jac * (zj1 * xk1 - xj1 * zk1);
          M[M_AKZ][q] = jac * (xj1 * yk1 - yj1 * xk1);
          M[M_AIX][q] = jac * (yk1 * zi1 - zk1 * yi1);
          M[M_AIY][q] = jac * (zk1 * xi1 - xk1 * zi1);
          M[M_AIZ][q] = jac * (xk1 * yi1 - yk1 * xi1);
          M[M_ASX][q] = jac * (yi1 * zj1 - zi1 * yj1);
          M[M_ASY][q] = jac * (zi1 * xj1 - xi1 * zj1);
          M[M_ASZ][q] = jac * (xi1 * yj1 - yi1 * xj1);
        }
  }

  /* ---------------- per-cell thermo wrappers ---------------- */
  void cell_di(long q, double* out) const {
    for (int m = 0; m < NS; m++) out[m] = di[(long)m * H + q];
  }

  /* comput_Amu_Amk_AMD (Comput_flow_variables.f90:69-98) */
  void transport_coeffs() {
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long q = ih(i, j, k), a = in(i, j, k);
          double d0[OCFD_MAX_SPEC], Xi[OCFD_MAX_SPEC], AmDi[OCFD_MAX_SPEC];
          double X0 = 0.0;
          for (int m = 0; m < NS; m++) {
            d0[m] = di[(long)m * H + q];
            Xi[m] = d0[m] / ch.Mi[m];
            X0 = X0 + Xi[m];
          }
          for (int m = 0; m < NS; m++) Xi[m] = Xi[m] / X0;
          double mu = ch.viscosity(T[q], Xi);
          double cp = ch.Cp(d[q], d0, T[q]);
          Amu[a] = mu;
          Amk[a] = ch.conductivity(mu, cp, T[q], Xi);
          ch.diffusion(AmDi, mu, T[q], d[q], p[q], Xi);
          for (int m = 0; m < NS; m++) AmD[(long)m * N + a] = AmDi[m];
        }
  }

  /* comput_Rhybrid (OCFD_SetHybrid.f90:17-104) */
  void comput_rhybrid() {
    int sensor = (int)std::lround(P.hybrid_para[0]);
    if (sensor == 1) {
#pragma omp parallel for collapse(2)
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) {
            long q = ih(i, j, k);
            const long sy = HX, sz = HX * HY;
            Rh[q] = std::fabs((p[q - 1] - 2.0 * p[q] + p[q + 1]) / (p[q - 1] + 2.0 * p[q] + p[q + 1])) +
                    std::fabs((p[q - sy] - 2.0 * p[q] + p[q + sy]) / (p[q - sy] + 2.0 * p[q] + p[q + sy])) +
                    std::fabs((p[q - sz] - 2.0 * p[q] + p[q + sz]) / (p[q - sz] + 2.0 * p[q] + p[q + sz]));
          }
    } else {
      std::vector<double> pk(N), pi(N), ps(N);
      dxyz(0, p.data(), pk.data()); dxyz(1, p.data(), pi.data()); dxyz(2, p.data(), ps.data());
      double dp0 = 0.0;
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) {
            long q = ih(i, j, k), a = in(i, j, k);
            double px = pk[a] * M[M_AKX][q] + pi[a] * M[M_AIX][q] + ps[a] * M[M_ASX][q];
            double py = pk[a] * M[M_AKY][q] + pi[a] * M[M_AIY][q] + ps[a] * M[M_ASY][q];
            double pz = pk[a] * M[M_AKZ][q] + pi[a] * M[M_AIZ][q] + ps[a] * M[M_ASZ][q];
            Rh[q] = std::sqrt(px * px + py * py + pz * pz);
            dp0 = dp0 + Rh[q];
          }
      double dp_av = dp0 / (1.0 * nx * ny * nz);
      double dp_av1 = 1.0 / (dp_av + 1.0e-30);
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) Rh[ih(i, j, k)] = Rh[ih(i, j, k)] * dp_av1;
    }
    /* patches forced to the most robust scheme; the reference reads the patch j-end into ie
     * (OCFD_SetHybrid.f90:85), this restatement uses the evident je */
    int mpatch = (int)std::lround(P.hybrid_para[3]);
    for (int m = 0; m < mpatch; m++) {
      int ib = std::max((int)std::lround(P.hybrid_para[4 + m * 6]), 1);
      int ie = std::min((int)std::lround(P.hybrid_para[5 + m * 6]), nx);
      int jb = std::max((int)std::lround(P.hybrid_para[6 + m * 6]), 1);
      int je = std::min((int)std::lround(P.hybrid_para[7 + m * 6]), ny);
      int kb = std::max((int)std::lround(P.hybrid_para[8 + m * 6]), 1);
      int ke = std::min((int)std::lround(P.hybrid_para[9 + m * 6]), nz);
      for (int k = kb; k <= ke; k++)
        for (int j = jb; j <= je; j++)
          for (int i = ib; i <= ie; i++) Rh[ih(i, j, k)] = Rh[ih(i, j, k)] + 100.0;
    }
    exch(Rh.data());
  }

  int set_hybrid(double R0) const {
    if (R0 <= S.theta1) return 1;
    if (R0 <= S.theta2) return 2;
    return 3;
  }

  /* split_Stager_Warming / split_Local_LaxFriedrichs at one point */
  void split(double Et1, double p1, double c1, double d1, double u1, double v1, double w1, double A1, double A2,
             double A3, double* fp, double* fm) const {
    if (P.flux_splitting == OCFD_SPLIT_SW) {
      double gamma = p1 / Et1 + 1.0;
      double tmp1 = 2.0 * (gamma - 1.0);
      double tmp3 = (3.0 - gamma) / (2.0 * (gamma - 1.0));
      double ss = std::sqrt(A1 * A1 + A2 * A2 + A3 * A3);
      double ss1 = 1.0 / ss;
      double ak1 = A1 * ss1, ak2 = A2 * ss1, ak3 = A3 * ss1;
      double vs = A1 * u1 + A2 * v1 + A3 * w1;
      double E1 = vs, E2 = vs - c1 * ss, E3 = vs + c1 * ss;
      double E1P = (E1 + std::fabs(E1)) * 0.5, E2P = (E2 + std::fabs(E2)) * 0.5, E3P = (E3 + std::fabs(E3)) * 0.5;
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
      double ss = std::sqrt(A1 * A1 + A2 * A2 + A3 * A3);
      double un = A1 * u1 + A2 * v1 + A3 * w1;
      double lam = std::fabs(un) + ss * c1;
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

  /* One direction of du_inviscous (and, with scalar != nullptr, of du_scaler_invis).
   * mode 0: out = x-part; 1: out += y-part; 2: out = -(out + z-part)*Ajac */
  void inviscid_dir(int dir, const double* scalar, double* out, int ncomp) {
    int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
    long s = dir == 0 ? 1 : (dir == 1 ? HX : HX * HY);
    double h1 = 1.0 / (dir == 0 ? hx : (dir == 1 ? hy : hz));
    const double* A1a = M[M_AKX1 + 3 * dir].data();
    const double* A2a = M[M_AKX1 + 3 * dir + 1].data();
    const double* A3a = M[M_AKX1 + 3 * dir + 2].data();
    int sb[2] = {P.scheme_boundary[2 * dir], P.scheme_boundary[2 * dir + 1]};
    int n1 = dir == 0 ? ny : nx, n2 = dir == 2 ? ny : nz;
#pragma omp parallel
    {
      std::vector<double> fpb(5 * (n + 2 * L)), fmb(5 * (n + 2 * L)), hh1(n + 1), hh2(n + 1);
      std::vector<int> scm(n + 1, 0);
#pragma omp for collapse(2)
      for (int b = 1; b <= n2; b++)
        for (int a = 1; a <= n1; a++) {
          int i0 = dir == 0 ? 0 : a, j0 = dir == 0 ? a : (dir == 1 ? 0 : b), k0 = dir == 2 ? 0 : b;
          if (dir == 1) { i0 = a; k0 = b; }
          if (dir == 2) { i0 = a; j0 = b; }
          long base = ih(dir == 0 ? 0 : i0, dir == 1 ? 0 : j0, dir == 2 ? 0 : k0); /* point index 0 */
          if (S.scheme == OCFD_SCHEME_HYBRID)
            for (int i = 0; i <= n; i++) scm[i] = set_hybrid(std::max(Rh[base + i * s], Rh[base + (i + 1) * s]));
          for (int i = 1 - L; i <= n + L; i++) {
            long q = base + i * s;
            double fp[5], fm[5];
            if (scalar) {
              double vs = A1a[q] * u[q] + A2a[q] * v[q] + A3a[q] * w[q];
              fp[0] = 0.5 * (vs + std::fabs(vs)) * scalar[q];
              fm[0] = 0.5 * (vs - std::fabs(vs)) * scalar[q];
            } else {
              split(Et[q], p[q], cc[q], d[q], u[q], v[q], w[q], A1a[q], A2a[q], A3a[q], fp, fm);
            }
            for (int m = 0; m < ncomp; m++) {
              fpb[m * (n + 2 * L) + (i + L - 1)] = fp[m];
              fmb[m * (n + 2 * L) + (i + L - 1)] = fm[m];
            }
          }
          for (int m = 0; m < ncomp; m++) {
            const double* vp = fpb.data() + m * (n + 2 * L) + (L - 1); /* vp[i] = f(i) */
            const double* vm = fmb.data() + m * (n + 2 * L) + (L - 1);
            flux_pencil(true, S, vp, hh1.data(), n, bound[dir], sb, scm.data());
            flux_pencil(false, S, vm, hh2.data(), n, bound[dir], sb, scm.data());
            for (int i = 1; i <= n; i++) {
              int ii = dir == 0 ? i : i0, jj = dir == 1 ? i : j0, kk = dir == 2 ? i : k0;
              long a2 = in(ii, jj, kk) + (long)m * N;
              double val = (hh1[i] - hh1[i - 1] + hh2[i] - hh2[i - 1]) * h1;
              if (dir == 0) out[a2] = val;
              else if (dir == 1) out[a2] = out[a2] + val;
              else out[a2] = -(out[a2] + val) * M[M_AJAC][ih(ii, jj, kk)];
            }
          }
        }
    }
  }

  /* One direction of du_inviscous_Character (OCFD_inviscous_character.f90:3-160) with
   * flux_charteric (:162-319): at every interface the split fluxes of the stencil are projected
   * on the left eigenvectors of the interface-averaged state, reconstructed component by
   * component, summed (h0 = h+ + h-) and projected back with the right eigenvectors; HYBRID
   * interfaces that take the linear scheme skip the projection. A closed face with the default
   * closure takes the non-reflecting physical-space flux at interfaces 0 and n. */
  void inviscid_dir_char(int dir, double* out) {
    int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
    long s = dir == 0 ? 1 : (dir == 1 ? HX : HX * HY);
    double h1 = 1.0 / (dir == 0 ? hx : (dir == 1 ? hy : hz));
    const double* A1a = M[M_AKX1 + 3 * dir].data();
    const double* A2a = M[M_AKX1 + 3 * dir + 1].data();
    const double* A3a = M[M_AKX1 + 3 * dir + 2].data();
    int sb[2] = {P.scheme_boundary[2 * dir], P.scheme_boundary[2 * dir + 1]};
    const int* bnd = bound[dir];
    int n1 = dir == 0 ? ny : nx, n2 = dir == 2 ? ny : nz;
    const int ia = (bnd[0] == 0 || sb[0] != 0) ? 0 : 1;
    const int ib = (bnd[1] == 0 || sb[1] != 0) ? n : n - 1;
    const int W = n + 2 * L;
#pragma omp parallel
    {
      std::vector<double> fpb(5 * W), fmb(5 * W), hh(5 * (n + 1));
      std::vector<int> scm(n + 1, 0);
#pragma omp for collapse(2)
      for (int b = 1; b <= n2; b++)
        for (int a = 1; a <= n1; a++) {
          int i0 = a, j0 = a, k0 = b;
          if (dir == 0) { j0 = a; k0 = b; }
          if (dir == 1) { i0 = a; k0 = b; }
          if (dir == 2) { i0 = a; j0 = b; }
          long base = ih(dir == 0 ? 0 : i0, dir == 1 ? 0 : j0, dir == 2 ? 0 : k0); /* point index 0 */
          if (S.scheme == OCFD_SCHEME_HYBRID)
            for (int i = 0; i <= n; i++) scm[i] = set_hybrid(std::max(Rh[base + i * s], Rh[base + (i + 1) * s]));
          for (int i = 1 - L; i <= n + L; i++) {
            long q = base + i * s;
            double fp[5], fm[5];
            split(Et[q], p[q], cc[q], d[q], u[q], v[q], w[q], A1a[q], A2a[q], A3a[q], fp, fm);
            for (int m = 0; m < 5; m++) {
              fpb[m * W + (i + L - 1)] = fp[m];
              fmb[m * W + (i + L - 1)] = fm[m];
            }
          }
          auto FP = [&](int i, int m) { return fpb[m * W + (i + L - 1)]; };
          auto FM = [&](int i, int m) { return fmb[m * W + (i + L - 1)]; };
          for (int i = ia; i <= ib; i++) {
            double fpc[8][5], fmc[8][5]; /* stencil offsets -3..4 at [mm + 3] */
            double S1[5][5];
            const bool lin = scm[i] == 1;
            if (lin) {
              for (int mm = -3; mm <= 4; mm++)
                for (int m = 0; m < 5; m++) { fpc[mm + 3][m] = FP(i + mm, m); fmc[mm + 3][m] = FM(i + mm, m); }
            } else {
              long q0 = base + i * s, q1 = base + (i + 1) * s;
              double u1 = (u[q0] + u[q1]) * 0.5, v1 = (v[q0] + v[q1]) * 0.5, w1 = (w[q0] + w[q1]) * 0.5;
              double c1 = (cc[q0] + cc[q1]) * 0.5, p1 = (p[q0] + p[q1]) * 0.5, Et1 = (Et[q0] + Et[q1]) * 0.5;
              double a1 = (A1a[q0] + A1a[q1]) * 0.5, a2 = (A2a[q0] + A2a[q1]) * 0.5, a3 = (A3a[q0] + A3a[q1]) * 0.5;
              double Sm[5][5];
              char_matrices(u1, v1, w1, c1, p1, Et1, a1, a2, a3, Sm, S1);
              for (int mm = -3; mm <= 4; mm++) {
                double xp[5], xm[5];
                for (int m = 0; m < 5; m++) { xp[m] = FP(i + mm, m); xm[m] = FM(i + mm, m); }
                for (int r = 0; r < 5; r++) {
                  fpc[mm + 3][r] = Sm[r][0] * xp[0] + Sm[r][1] * xp[1] + Sm[r][2] * xp[2] + Sm[r][3] * xp[3] + Sm[r][4] * xp[4];
                  fmc[mm + 3][r] = Sm[r][0] * xm[0] + Sm[r][1] * xm[1] + Sm[r][2] * xm[2] + Sm[r][3] * xm[3] + Sm[r][4] * xm[4];
                }
              }
            }
            double h0[5];
            for (int m = 0; m < 5; m++) {
              double gp[8], gm[8];
              for (int mm = 0; mm < 8; mm++) { gp[mm] = fpc[mm][m]; gm[mm] = fmc[mm][m]; }
              double ha = iface_flux(true, S, gp + 3, i, n, bnd, sb, scm[i]);
              double hb = iface_flux(false, S, gm + 3, i, n, bnd, sb, scm[i]);
              h0[m] = ha + hb;
            }
            for (int m = 0; m < 5; m++)
              hh[m * (n + 1) + i] = lin ? h0[m]
                                        : S1[m][0] * h0[0] + S1[m][1] * h0[1] + S1[m][2] * h0[2] + S1[m][3] * h0[3] +
                                              S1[m][4] * h0[4];
          }
          if (bnd[0] == 1 && sb[0] == 0)
            for (int m = 0; m < 5; m++)
              hh[m * (n + 1)] = (2.0 * FP(1, m) + 5.0 * FP(2, m) - FP(3, m) + 2.0 * FM(3, m) - 7.0 * FM(2, m) +
                                 11.0 * FM(1, m)) / 6.0;
          if (bnd[1] == 1 && sb[1] == 0)
            for (int m = 0; m < 5; m++)
              hh[m * (n + 1) + n] = (2.0 * FP(n - 2, m) - 7.0 * FP(n - 1, m) + 11.0 * FP(n, m) + 2.0 * FM(n, m) +
                                     5.0 * FM(n - 1, m) - FM(n - 2, m)) / 6.0;
          for (int m = 0; m < 5; m++)
            for (int i = 1; i <= n; i++) {
              int ii = dir == 0 ? i : i0, jj = dir == 1 ? i : j0, kk = dir == 2 ? i : k0;
              long a2 = in(ii, jj, kk) + (long)m * N;
              double val = (hh[m * (n + 1) + i] - hh[m * (n + 1) + i - 1]) * h1;
              if (dir == 0) out[a2] = val;
              else if (dir == 1) out[a2] = out[a2] + val;
              else out[a2] = -(out[a2] + val) * M[M_AJAC][ih(ii, jj, kk)];
            }
        }
    }
  }

  /* left (S) and right (S1) eigenvector matrices of the flux Jacobian along the metric vector
   * a at the interface-averaged state (OCFD_inviscous_character.f90:213-270) */
  static void char_matrices(double u1, double v1, double w1, double c1, double p1, double Et1, double a1, double a2,
                            double a3, double Sm[5][5], double S1[5][5]) {
    double ss = std::sqrt(a1 * a1 + a2 * a2 + a3 * a3);
    double n1 = a1 / ss, n2 = a2 / ss, n3 = a3 / ss;
    double l1, l2, l3;
    if (std::fabs(n3) <= std::fabs(n2)) {
      ss = std::sqrt(n1 * n1 + n2 * n2);
      l1 = -n2 / ss; l2 = n1 / ss; l3 = 0.0;
    } else {
      ss = std::sqrt(n1 * n1 + n3 * n3);
      l1 = -n3 / ss; l2 = 0.0; l3 = n1 / ss;
    }
    double m1 = n2 * l3 - n3 * l2, m2 = n3 * l1 - n1 * l3, m3 = n1 * l2 - n2 * l1;
    double un = u1 * n1 + v1 * n2 + w1 * n3, ul = u1 * l1 + v1 * l2 + w1 * l3, um = u1 * m1 + v1 * m2 + w1 * m3;
    double V2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5;
    double gamma = p1 / Et1 + 1.0;
    double KK = (gamma - 1.0) / (c1 * c1);
    double KK1 = KK * 0.5, X1 = 1.0 / (2.0 * c1), Hh = V2 + 1.0 / KK;
    double A[5][5] = {{1.0 - KK * V2, KK * u1, KK * v1, KK * w1, -KK},
                      {-ul, l1, l2, l3, 0.0},
                      {-um, m1, m2, m3, 0.0},
                      {KK1 * V2 + X1 * un, -X1 * n1 - KK1 * u1, -X1 * n2 - KK1 * v1, -X1 * n3 - KK1 * w1, KK1},
                      {KK1 * V2 - X1 * un, X1 * n1 - KK1 * u1, X1 * n2 - KK1 * v1, X1 * n3 - KK1 * w1, KK1}};
    double B[5][5] = {{1.0, 0.0, 0.0, 1.0, 1.0},
                      {u1, l1, m1, u1 - c1 * n1, u1 + c1 * n1},
                      {v1, l2, m2, v1 - c1 * n2, v1 + c1 * n2},
                      {w1, l3, m3, w1 - c1 * n3, w1 + c1 * n3},
                      {V2, ul, um, Hh - c1 * un, Hh + c1 * un}};
    for (int r = 0; r < 5; r++)
      for (int c = 0; c < 5; c++) { Sm[r][c] = A[r][c]; S1[r][c] = B[r][c]; }
  }

  /* comput_cc (Comput_flow_variables.f90:50-63) over the full halo range */
  void comput_cc() {
#pragma omp parallel for
    for (long q = 0; q < H; q++) {
      double gamma = p[q] / Et[q] + 1.0;
      cc[q] = std::sqrt(gamma * p[q] / d[q]);
    }
  }

  void du_inviscous() {
    comput_cc();
    if (P.if_scheme_character == 1) { /* OCFD_Time_Adv.f90:76-80 */
      inviscid_dir_char(0, du.data());
      inviscid_dir_char(1, du.data());
      inviscid_dir_char(2, du.data());
    } else {
      inviscid_dir(0, nullptr, du.data(), 5);
      inviscid_dir(1, nullptr, du.data(), 5);
      inviscid_dir(2, nullptr, du.data(), 5);
    }
    if (P.if_mass_force == 1) {
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) {
            long a = in(i, j, k), q = ih(i, j, k);
            du[N + a] = du[N + a] + d[q] * P.mass_force[0];
            du[2 * N + a] = du[2 * N + a] + d[q] * P.mass_force[1];
            du[3 * N + a] = du[3 * N + a] + d[q] * P.mass_force[2];
            du[4 * N + a] =
                du[4 * N + a] + d[q] * (u[q] * P.mass_force[0] + v[q] * P.mass_force[1] + w[q] * P.mass_force[2]);
          }
    }
  }

  /* du_viscous (OCFD_viscous.f90:27-131) */
  void du_viscous() {
    double* uk = dk[0].data(); double* vk = dk[1].data(); double* wk = dk[2].data(); double* Tk = dk[3].data();
    double* ui = dk[4].data(); double* vi = dk[5].data(); double* wi = dk[6].data(); double* Ti = dk[7].data();
    double* us = dk[8].data(); double* vs = dk[9].data(); double* ws = dk[10].data(); double* Ts = dk[11].data();
    dxyz(0, u.data(), uk); dxyz(0, v.data(), vk); dxyz(0, w.data(), wk); dxyz(0, T.data(), Tk);
    dxyz(1, u.data(), ui); dxyz(1, v.data(), vi); dxyz(1, w.data(), wi); dxyz(1, T.data(), Ti);
    dxyz(2, u.data(), us); dxyz(2, v.data(), vs); dxyz(2, w.data(), ws); dxyz(2, T.data(), Ts);
    const double tmp2_3 = 2.0 / 3.0;
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long a = in(i, j, k), q = ih(i, j, k);
          const double Akx = M[M_AKX][q], Aky = M[M_AKY][q], Akz = M[M_AKZ][q], Aix = M[M_AIX][q], Aiy = M[M_AIY][q],
                       Aiz = M[M_AIZ][q], Asx = M[M_ASX][q], Asy = M[M_ASY][q], Asz = M[M_ASZ][q];
          double ux = uk[a] * Akx + ui[a] * Aix + us[a] * Asx;
          double vx = vk[a] * Akx + vi[a] * Aix + vs[a] * Asx;
          double wx = wk[a] * Akx + wi[a] * Aix + ws[a] * Asx;
          double Tx = Tk[a] * Akx + Ti[a] * Aix + Ts[a] * Asx;
          double uy = uk[a] * Aky + ui[a] * Aiy + us[a] * Asy;
          double vy = vk[a] * Aky + vi[a] * Aiy + vs[a] * Asy;
          double wy = wk[a] * Aky + wi[a] * Aiy + ws[a] * Asy;
          double Ty = Tk[a] * Aky + Ti[a] * Aiy + Ts[a] * Asy;
          double uz = uk[a] * Akz + ui[a] * Aiz + us[a] * Asz;
          double vz = vk[a] * Akz + vi[a] * Aiz + vs[a] * Asz;
          double wz = wk[a] * Akz + wi[a] * Aiz + ws[a] * Asz;
          double Tz = Tk[a] * Akz + Ti[a] * Aiz + Ts[a] * Asz;
          double div = ux + vy + wz;
          double Amu1 = Amu[a], Amuk = Amk[a];
          double s11 = (2.0 * ux - tmp2_3 * div) * Amu1;
          double s22 = (2.0 * vy - tmp2_3 * div) * Amu1;
          double s33 = (2.0 * wz - tmp2_3 * div) * Amu1;
          double s12 = (uy + vx) * Amu1, s13 = (uz + wx) * Amu1, s23 = (vz + wy) * Amu1;
          double E1 = u[q] * s11 + v[q] * s12 + w[q] * s13 + Amuk * Tx + Qpx[a];
          double E2 = u[q] * s12 + v[q] * s22 + w[q] * s23 + Amuk * Ty + Qpy[a];
          double E3 = u[q] * s13 + v[q] * s23 + w[q] * s33 + Amuk * Tz + Qpz[a];
          for (int dd = 0; dd < 3; dd++) {
            double* Ev = dd == 0 ? Ev1.data() : (dd == 1 ? Ev2.data() : Ev3.data());
            double B1 = M[M_AKX1 + 3 * dd][q], B2 = M[M_AKX1 + 3 * dd + 1][q], B3 = M[M_AKX1 + 3 * dd + 2][q];
            Ev[q] = B1 * s11 + B2 * s12 + B3 * s13;
            Ev[H + q] = B1 * s12 + B2 * s22 + B3 * s23;
            Ev[2 * H + q] = B1 * s13 + B2 * s23 + B3 * s33;
            Ev[3 * H + q] = B1 * E1 + B2 * E2 + B3 * E3;
          }
        }
    for (int m = 0; m < 4; m++) {
      exch_x(Ev1.data() + m * H);
      exch_y(Ev2.data() + m * H);
      exch_z(Ev3.data() + m * H);
      dxyz(0, Ev1.data() + m * H, uk);
      dxyz(1, Ev2.data() + m * H, ui);
      dxyz(2, Ev3.data() + m * H, us);
#pragma omp parallel for collapse(2)
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) {
            long a = in(i, j, k);
            du[(m + 1) * N + a] = du[(m + 1) * N + a] + (uk[a] + ui[a] + us[a]) * M[M_AJAC][ih(i, j, k)];
          }
    }
  }

  /* du_scaler_viscous (OCFD_scaler_viscous.f90:4-79) for species ks (0-based) */
  void du_scaler_viscous(int ks, const double* fs, double* Dus) {
    double* uk = dk[0].data(); double* ui = dk[4].data(); double* us = dk[8].data();
    if (ks == 0) {
      std::fill(Qpx.begin(), Qpx.end(), 0.0);
      std::fill(Qpy.begin(), Qpy.end(), 0.0);
      std::fill(Qpz.begin(), Qpz.end(), 0.0);
    }
    for (long q = 0; q < H; q++) Ev1[q] = fs[q] / d[q];
    dxyz(0, Ev1.data(), uk); dxyz(1, Ev1.data(), ui); dxyz(2, Ev1.data(), us);
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long a = in(i, j, k), q = ih(i, j, k);
          double hi = ch.hi(ks, T[q]);
          double cix = uk[a] * M[M_AKX][q] + ui[a] * M[M_AIX][q] + us[a] * M[M_ASX][q];
          double ciy = uk[a] * M[M_AKY][q] + ui[a] * M[M_AIY][q] + us[a] * M[M_ASY][q];
          double ciz = uk[a] * M[M_AKZ][q] + ui[a] * M[M_AIZ][q] + us[a] * M[M_ASZ][q];
          double dD = d[q] * AmD[(long)ks * N + a];
          double E1 = dD * cix, E2 = dD * ciy, E3 = dD * ciz;
          Qpx[a] = Qpx[a] + E1 * hi;
          Qpy[a] = Qpy[a] + E2 * hi;
          Qpz[a] = Qpz[a] + E3 * hi;
          Ev1[q] = E1 * M[M_AKX1][q] + E2 * M[M_AKY1][q] + E3 * M[M_AKZ1][q];
          Ev1[H + q] = E1 * M[M_AIX1][q] + E2 * M[M_AIY1][q] + E3 * M[M_AIZ1][q];
          Ev1[2 * H + q] = E1 * M[M_ASX1][q] + E2 * M[M_ASY1][q] + E3 * M[M_ASZ1][q];
        }
    exch_x(Ev1.data());
    exch_y(Ev1.data() + H);
    exch_z(Ev1.data() + 2 * H);
    dxyz(0, Ev1.data(), uk); dxyz(1, Ev1.data() + H, ui); dxyz(2, Ev1.data() + 2 * H, us);
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long a = in(i, j, k);
          Dus[a] = Dus[a] + (uk[a] + ui[a] + us[a]) * M[M_AJAC][ih(i, j, k)];
        }
  }

  /* OCFD_time_adv_RK3 / Scalar_time_adv_RK3 */
  void rk3(int krk, double dt) {
    const double ra[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0}, rb[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
#pragma omp parallel for
    for (long a = 0; a < 5 * N; a++) {
      if (krk == 1) f[a] = fn[a] + dt * du[a];
      else f[a] = ra[krk - 1] * fn[a] + rb[krk - 1] * (f[a] + dt * du[a]);
    }
  }
  void scalar_rk3(int krk, int m, const double* dus, double dt) {
    const double ra[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0}, rb[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long a = in(i, j, k), q = (long)m * H + ih(i, j, k);
          if (krk == 1) di[q] = din[(long)m * N + a] + dt * dus[a];
          else di[q] = ra[krk - 1] * din[(long)m * N + a] + rb[krk - 1] * (di[q] + dt * dus[a]);
        }
  }

  /* comput_flow_variables + handle_NegativeEt + Rescaling_di + comput_T_P */
  /* The reference loop is serial because a repaired cell averages its six neighbours, of
   * which the ones earlier in (i,j,k) loop order already hold this pass's values and the
   * later ones (and all halo points) still hold the previous ones. The restatement computes
   * the new Et in parallel into a scratch array and then replays the repairs serially with
   * exactly that neighbour rule. */
  int comput_flow_variables() {
    std::vector<double> etn(N);
    std::vector<char> neg(N, 0);
    long nneg = 0;
#pragma omp parallel for collapse(2) reduction(+ : nneg)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long a = in(i, j, k), q = ih(i, j, k);
          d[q] = f[a];
          u[q] = f[N + a] / f[a];
          v[q] = f[2 * N + a] / f[a];
          w[q] = f[3 * N + a] / f[a];
          etn[a] = f[4 * N + a] - (f[N + a] * u[q] + f[2 * N + a] * v[q] + f[3 * N + a] * w[q]) * 0.5;
          if (etn[a] <= 0) { neg[a] = 1; nneg++; }
        }
    if (nneg) {
      int num_neg = 0;
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) {
            long a = in(i, j, k);
            if (!neg[a]) continue;
            auto nb = [&](int ii, int jj, int kk) {
              bool inside = ii >= 1 && ii <= nx && jj >= 1 && jj <= ny && kk >= 1 && kk <= nz;
              if (inside && in(ii, jj, kk) < a) return etn[in(ii, jj, kk)];
              return Et[ih(ii, jj, kk)];
            };
            double e0 = etn[a];
            etn[a] = (nb(i + 1, j, k) + nb(i - 1, j, k) + nb(i, j + 1, k) + nb(i, j - 1, k) + nb(i, j, k + 1) +
                      nb(i, j, k - 1)) /
                     6.0;
            f[4 * N + a] = f[4 * N + a] + (etn[a] - e0);
            num_neg++;
            neg_et++;
            if (num_neg > 10) { err = "Number of Negative Temperature Points > Limit"; return OCFD_ERR_NEGATIVE_ET; }
          }
    }
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) Et[ih(i, j, k)] = etn[in(i, j, k)];
    rescale_di();
    comput_T_P();
    return 0;
  }
  void rescale_di() {
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long q = ih(i, j, k);
          double d0 = 0.0;
          for (int m = 0; m < NS; m++) {
            if (di[(long)m * H + q] < 0.0) di[(long)m * H + q] = 0.0;
            d0 = d0 + di[(long)m * H + q];
          }
          double tmp = d[q] / d0;
          for (int m = 0; m < NS; m++) di[(long)m * H + q] = di[(long)m * H + q] * tmp;
        }
  }
  void comput_T_P() {
#pragma omp parallel for collapse(2)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long q = ih(i, j, k);
          double d0[OCFD_MAX_SPEC];
          cell_di(q, d0);
          T[q] = ch.T_of_E(d0, Et[q]);
          p[q] = ch.P(d0, T[q]);
        }
  }

  /* face re-derivation of one cell (OCFD_BC.f90:33-184 body) */
  void face_cell(int i, int j, int k) {
    long q = ih(i, j, k), a = in(i, j, k);
    double di1[OCFD_MAX_SPEC];
    double d0 = 0.0;
    for (int m = 0; m < NS; m++) { di1[m] = di[(long)m * H + q]; d0 = d0 + di1[m]; }
    double dtmp = d[q] / d0;
    for (int m = 0; m < NS; m++) { di1[m] = di1[m] * dtmp; di[(long)m * H + q] = di1[m]; }
    Et[q] = ch.E_of_T(di1, T[q]);
    p[q] = ch.P(di1, T[q]);
    f[a] = d[q];
    f[N + a] = d[q] * u[q];
    f[2 * N + a] = d[q] * v[q];
    f[3 * N + a] = d[q] * w[q];
    f[4 * N + a] = Et[q] + d[q] * (u[q] * u[q] + v[q] * v[q] + w[q] * w[q]) * 0.5;
  }

  void bc_boundary_layer(double tt) {
    int nv = 5 + NS;
    /* inlet i=1 */
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) {
        long q = ih(1, j, k);
        double vals[5 + OCFD_MAX_SPEC];
        for (int c = 0; c < nv; c++) {
          if (bcdata_inlet == 0) vals[c] = inlet[c];
          else if (bcdata_inlet == 1) vals[c] = inlet[(long)c * ny + (j - 1)];
          else vals[c] = inlet[((long)c * nz + (k - 1)) * ny + (j - 1)];
        }
        d[q] = vals[0]; u[q] = vals[1]; v[q] = vals[2]; w[q] = vals[3]; T[q] = vals[4];
        for (int m = 0; m < NS; m++) di[(long)m * H + q] = vals[5 + m];
      }
    /* upper j=ny */
    if (bcdata_upper >= 0) {
      for (int k = 1; k <= nz; k++)
        for (int i = 1; i <= nx; i++) {
          if (nonref[(i - 1) + (long)nx * (k - 1)] != 0) continue;
          long q = ih(i, ny, k);
          double vals[5 + OCFD_MAX_SPEC];
          for (int c = 0; c < nv; c++) {
            if (bcdata_upper == 0) vals[c] = upper[c];
            else if (bcdata_upper == 1) vals[c] = upper[(long)c * nx + (i - 1)];
            else vals[c] = upper[((long)c * nz + (k - 1)) * nx + (i - 1)];
          }
          d[q] = vals[0]; u[q] = vals[1]; v[q] = vals[2]; w[q] = vals[3]; T[q] = vals[4];
          for (int m = 0; m < NS; m++) di[(long)m * H + q] = vals[5 + m];
        }
    }
    /* wall j=1 (get_ht_multifrequancy, OCFD_BC_Boundarylayers.f90:579-618) */
    const double PI = 3.14159265358979;
    double ht = 0.0;
    double beta = P.bc_para[13];
    if (beta > 0.0) {
      for (size_t m = 0; m < tm.size(); m++) ht = ht + tm[m] * std::sin((m + 1) * beta * tt * 2.0 * PI + 2.0 * PI * fait[m]);
    } else {
      ht = 1.0;
    }
    double Tw = P.bc_para[4], Xinit = P.bc_para[5], disA = P.bc_para[7];
    for (int k = 1; k <= nz; k++)
      for (int i = 1; i <= nx; i++) {
        long q1 = ih(i, 1, k), q2 = ih(i, 2, k), q3 = ih(i, 3, k);
        if (X[q1] < Xinit) {
          d[q1] = d[q2]; u[q1] = u[q2]; v[q1] = v[q2]; w[q1] = w[q2]; T[q1] = T[q2];
          for (int m = 0; m < NS; m++) di[(long)m * H + q1] = di[(long)m * H + q2];
        } else {
          double Aix = M[M_AIX][q1], Aiy = M[M_AIY][q1], Aiz = M[M_AIZ][q1];
          double tmp = 1.0 / std::sqrt(Aix * Aix + Aiy * Aiy + Aiz * Aiz);
          double A0 = disA * ht * wall_pertb[(i - 1) + (long)nx * (k - 1)];
          u[q1] = A0 * Aix * tmp;
          v[q1] = A0 * Aiy * tmp;
          w[q1] = A0 * Aiz * tmp;
          if (Tw > 0) T[q1] = Tw;
          else T[q1] = (4.0 * T[q2] - T[q3]) / 3.0;
          double di2[OCFD_MAX_SPEC], di3[OCFD_MAX_SPEC], di1[OCFD_MAX_SPEC];
          cell_di(q2, di2);
          cell_di(q3, di3);
          double pp2 = ch.P(di2, T[q2]);
          double pp3 = ch.P(di3, T[q3]);
          double pp1 = (4.0 * pp2 - pp3) / 3.0;
          for (int m = 0; m < NS; m++) di1[m] = di2[m] / d[q2];
          double d1 = ch.Dens(di1, T[q1], pp1);
          d[q1] = d1;
          for (int m = 0; m < NS; m++) di[(long)m * H + q1] = di1[m] * d1;
        }
      }
    /* outlet i=nx */
    int outlet = (int)std::lround(P.bc_para[3]);
    if (outlet == 1 || outlet == 2) {
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++) {
          long q = ih(nx, j, k), q1 = ih(nx - 1, j, k), q2 = ih(nx - 2, j, k);
          if (outlet == 1) {
            d[q] = d[q1]; u[q] = u[q1]; v[q] = v[q1]; w[q] = w[q1]; T[q] = T[q1];
            for (int m = 0; m < NS; m++) di[(long)m * H + q] = di[(long)m * H + q1];
          } else {
            d[q] = 2.0 * d[q1] - d[q2]; u[q] = 2.0 * u[q1] - u[q2]; v[q] = 2.0 * v[q1] - v[q2];
            w[q] = 2.0 * w[q1] - w[q2]; T[q] = 2.0 * T[q1] - T[q2];
            for (int m = 0; m < NS; m++) di[(long)m * H + q] = 2.0 * di[(long)m * H + q1] - di[(long)m * H + q2];
          }
        }
    }
  }

  /* ocfd_bc_jet (OCFD_BC_jet.f90:2-96): 2-D inlet table, Dirichlet (Iflag_inlet = 0) or
   * subsonic / supersonic switch on the inlet Mach number (1); zeroth-order outlet */
  void bc_jet() {
    int iflag = (int)std::lround(P.bc_para[0]);
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) {
        long q = ih(1, j, k);
        double vals[5 + OCFD_MAX_SPEC];
        for (int c = 0; c < 5 + NS; c++) vals[c] = inlet[((long)c * nz + (k - 1)) * ny + (j - 1)];
        if (iflag == 0) {
          d[q] = vals[0]; u[q] = vals[1]; v[q] = vals[2]; w[q] = vals[3]; T[q] = vals[4];
          for (int m = 0; m < NS; m++) di[(long)m * H + q] = vals[5 + m];
        } else {
          u[q] = vals[1]; v[q] = vals[2]; w[q] = vals[3]; T[q] = vals[4];
          double d1 = vals[0], di1[OCFD_MAX_SPEC], ai1[OCFD_MAX_SPEC], d0 = 0.0;
          for (int m = 0; m < NS; m++) { di1[m] = vals[5 + m]; d0 = d0 + di1[m]; }
          for (int m = 0; m < NS; m++) ai1[m] = di1[m] / d0;
          double p1 = ch.P(di1, T[q]);
          double Et1 = ch.E_of_T(di1, T[q]);
          double gamma = p1 / Et1 + 1.0;
          double c1 = std::sqrt(gamma * p1 / d1);  /* comput_soundspeed (CHEM_thermdyn.f90:412-418) */
          if (u[q] < c1) {
            p[q] = p[ih(2, j, k)];
            double dn = ch.Dens(ai1, T[q], p[q]);
            d[q] = dn;
            for (int m = 0; m < NS; m++) di[(long)m * H + q] = dn * ai1[m];
          } else {
            d[q] = d1;
            for (int m = 0; m < NS; m++) di[(long)m * H + q] = di1[m];
          }
        }
      }
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) {
        long q = ih(nx, j, k), q1 = ih(nx - 1, j, k);
        d[q] = d[q1]; u[q] = u[q1]; v[q] = v[q1]; w[q] = w[q1]; T[q] = T[q1]; p[q] = p[q1]; Et[q] = Et[q1];
        for (int m = 0; m < NS; m++) di[(long)m * H + q] = di[(long)m * H + q1];
      }
  }

  /* Flow_Ghost_Extent_2nd (OCFD_GhostCell.f90:166-364) */
  void ghost() {
    const double s1 = 0.8, s2 = 1.2;
    for (int face = 0; face < 6; face++) {
      if (!(P.ghost_cell[face] == 1 || P.ghost_cell[face] == 2)) continue;
      int dir = face / 2, side = face % 2;
      int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
      long s = dir == 0 ? 1 : (dir == 1 ? HX : HX * HY);
      int na = dir == 0 ? ny : nx, nb = dir == 2 ? ny : nz;
      for (int b = 1; b <= nb; b++)
        for (int l = 1; l <= L; l++)
          for (int a = 1; a <= na; a++) {
            int i0 = dir == 0 ? 0 : a, j0 = dir == 0 ? a : (dir == 1 ? 0 : b), k0 = dir == 2 ? 0 : b;
            if (dir == 2) { i0 = a; j0 = b; }
            long base = ih(dir == 0 ? 0 : i0, dir == 1 ? 0 : j0, dir == 2 ? 0 : k0);
            int ig = side == 0 ? 1 - l : n + l;      /* ghost index */
            int ib = side == 0 ? 1 : n;              /* boundary index */
            int im = side == 0 ? 2 - ig : 2 * n - ig; /* mirror */
            long qg = base + ig * s, qb = base + ib * s, qm = base + im * s;
            u[qg] = 2.0 * u[qb] - u[qm]; v[qg] = 2.0 * v[qb] - v[qm]; w[qg] = 2.0 * w[qb] - w[qm];
            d[qg] = 2.0 * d[qb] - d[qm]; T[qg] = 2.0 * T[qb] - T[qm];
            if (d[qg] < s1 * d[qb]) d[qg] = s1 * d[qb];
            if (d[qg] > s2 * d[qb]) d[qg] = s2 * d[qb];
            if (T[qg] < s1 * T[qb]) T[qg] = s1 * T[qb];
            if (T[qg] > s2 * T[qb]) T[qg] = s2 * T[qb];
            double di1[OCFD_MAX_SPEC], d0 = 0.0;
            for (int m = 0; m < NS; m++) { di1[m] = 2.0 * di[(long)m * H + qb] - di[(long)m * H + qm]; d0 = d0 + di1[m]; }
            double dtmp = d[qg] / d0;
            for (int m = 0; m < NS; m++) { di1[m] = di1[m] * dtmp; di[(long)m * H + qg] = di1[m]; }
            Et[qg] = ch.E_of_T(di1, T[qg]);
            p[qg] = ch.P(di1, T[qg]);
          }
    }
  }

  void ocfd_bc(double tt) {
    if (P.ibc == OCFD_BC_BOUNDARYLAYER) bc_boundary_layer(tt);
    if (P.ibc == OCFD_BC_JET) bc_jet();
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) { face_cell(1, j, k); }
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++) { face_cell(nx, j, k); }
    for (int k = 1; k <= nz; k++)
      for (int i = 1; i <= nx; i++) face_cell(i, 1, k);
    for (int k = 1; k <= nz; k++)
      for (int i = 1; i <= nx; i++) face_cell(i, ny, k);
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) face_cell(i, j, 1);
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) face_cell(i, j, nz);
    ghost();
  }

  /* init3d tail (OCFD_init.f90:8-25) + comput_flow_variables + OCFD_bc (OCFD_NS_Solver.f90:17-18) */
  int init_state(const double* prim5, const double* dii, double tt) {
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long a = in(i, j, k), q = ih(i, j, k);
          d[q] = prim5[a]; u[q] = prim5[N + a]; v[q] = prim5[2 * N + a]; w[q] = prim5[3 * N + a]; T[q] = prim5[4 * N + a];
          for (int m = 0; m < NS; m++) di[(long)m * H + q] = dii[(long)m * N + a];
        }
    rescale_di();
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long a = in(i, j, k), q = ih(i, j, k);
          double di1[OCFD_MAX_SPEC];
          cell_di(q, di1);
          f[a] = d[q];
          f[N + a] = d[q] * u[q];
          f[2 * N + a] = d[q] * v[q];
          f[3 * N + a] = d[q] * w[q];
          double Et1 = ch.E_of_T(di1, T[q]);
          f[4 * N + a] = Et1 + d[q] * (u[q] * u[q] + v[q] * v[q] + w[q] * w[q]) * 0.5;
        }
    int e = comput_flow_variables();
    if (e) return e;
    ocfd_bc(tt);
    return 0;
  }

  /* flow_time_advance (OCFD_Time_Adv.f90:7-92) */
  int flow_advance(double dt1, double tt) {
    std::memcpy(fn.data(), f.data(), sizeof(double) * 5 * N);
    for (int m = 0; m < NS; m++)
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) din[(long)m * N + in(i, j, k)] = di[(long)m * H + ih(i, j, k)];
    for (int krk = 1; krk <= 3; krk++) {
      transport_coeffs();
      exch(d.data()); exch(u.data()); exch(v.data()); exch(w.data()); exch(T.data()); exch(p.data()); exch(Et.data());
      if (NS == 1) {
        std::memcpy(di.data(), d.data(), sizeof(double) * H);
      } else {
        for (int m = 0; m < NS; m++) exch(di.data() + (long)m * H);
      }
      if (krk == 1 && P.scheme_invis == OCFD_SCHEME_HYBRID) comput_rhybrid();
      if (NS != 1) {
        for (int m = 0; m < NS; m++) {
          const double* fs = di.data() + (long)m * H;
          inviscid_dir(0, fs, du.data(), 1);
          inviscid_dir(1, fs, du.data(), 1);
          inviscid_dir(2, fs, du.data(), 1);
          if (P.if_viscous == 1) du_scaler_viscous(m, fs, du.data());
          scalar_rk3(krk, m, du.data(), dt1);
        }
      }
      du_inviscous();
      if (P.if_viscous == 1) du_viscous();
      rk3(krk, dt1);
      int e = comput_flow_variables();
      if (e) return e;
      ocfd_bc(tt);
    }
    return 0;
  }

  /* ---------------- filtering (code/others/OCFD_filtering.f90) ---------------- */
  /* F = Para%Filter(100,10) column-major: group m's parameters at F[100 m + 0..12] */
  int filtering(int istep, int nfilt, const double* F, int* applied) {
    if (applied) *applied = 0;
    if (nfilt < 0 || nfilt > 10) { err = "NFiltering must be 0..10"; return OCFD_ERR_PARAM; }
    for (int m = 0; m < nfilt; m++)
      if (std::lround(F[100 * m]) < 1) { err = "filter step interval must be >= 1"; return OCFD_ERR_PARAM; }
    int any = 0;
    for (int m = 0; m < nfilt; m++)
      if (istep % (int)std::lround(F[100 * m]) == 0) any = 1;
    if (!any) return 0;
    if (applied) *applied = 1;
    for (int m = 0; m < nfilt; m++) {
      const double* c = F + 100 * m;
      if (istep % (int)std::lround(c[0]) != 0) continue;
      const int fdir[3] = {(int)std::lround(c[1]), (int)std::lround(c[2]), (int)std::lround(c[3])};
      int b[3][2];
      const int nn3[3] = {nx, ny, nz};
      for (int d = 0; d < 3; d++) {
        b[d][0] = std::max((int)std::lround(c[4 + 2 * d]), 1);
        b[d][1] = std::min((int)std::lround(c[5 + 2 * d]), nn3[d]);
      }
      const int scheme = (int)std::lround(c[10]);
      const double s0 = c[11], rth = c[12];
      for (int d = 0; d < 3; d++) {
        if (fdir[d] != 1) continue;
        if (scheme == 1) filter_fo9p(d, s0, b);
        else if (scheme == 2) {
          int e = filter_shock(d, s0, rth, b);
          if (e) return e;
        }
      }
    }
    return 0;
  }
  /* filter_x3d / filter_y3d / filter_z3d (:78-189): f0 is a fresh halo array (its halo is only
   * read where the exchange filled it), f is overwritten component by component */
  void filter_fo9p(int dir, double s0, const int (&b)[3][2]) {
    const double d0 = 0.243527493120, d1 = -0.204788880640, d2 = 0.120007591680, d3 = -0.045211119360,
                 d4 = 0.008228661760;
    const int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
    int lo[3] = {b[0][0], b[1][0], b[2][0]}, hi[3] = {b[0][1], b[1][1], b[2][1]};
    if (P.iperiodic[dir] != 1) { lo[dir] = std::max(lo[dir], 6); hi[dir] = std::min(hi[dir], n - 5); }
    const long s = dir == 0 ? 1 : (dir == 1 ? HX : HX * HY);
    std::vector<double> f0(H, std::nan(""));
    for (int m = 0; m < 5; m++) {
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) f0[ih(i, j, k)] = f[(long)m * N + in(i, j, k)];
      if (dir == 0) exch_x(f0.data());
      else if (dir == 1) exch_y(f0.data());
      else exch_z(f0.data());
      for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
          for (int i = lo[0]; i <= hi[0]; i++) {
            const double* q = f0.data() + ih(i, j, k);
            f[(long)m * N + in(i, j, k)] =
                q[0] - s0 * (d0 * q[0] + d1 * (q[-s] + q[s]) + d2 * (q[-2 * s] + q[2 * s]) + d3 * (q[-3 * s] + q[3 * s]) +
                             d4 * (q[-4 * s] + q[4 * s]));
          }
    }
  }
  /* filter_x3d_shock / _y3d_ / _z3d_ (:194-360) */
  int filter_shock(int dir, double s0, double rth, const int (&b)[3][2]) {
    const double c1 = -0.210383, c2 = 0.039617;
    const int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
    int lo[3] = {b[0][0], b[1][0], b[2][0]}, hi[3] = {b[0][1], b[1][1], b[2][1]};
    if (P.iperiodic[dir] != 1) { lo[dir] = std::max(lo[dir], 4); hi[dir] = std::min(hi[dir], n - 3); }
    int e = comput_flow_variables();
    if (e) return e;
    if (dir == 0) exch_x(p.data());
    else if (dir == 1) exch_y(p.data());
    else exch_z(p.data());
    const long s = dir == 0 ? 1 : (dir == 1 ? HX : HX * HY);
    std::vector<double> f0(H, std::nan("")), sc0(n + 2);
    for (int m = 0; m < 5; m++) {
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) f0[ih(i, j, k)] = f[(long)m * N + in(i, j, k)];
      if (dir == 0) exch_x(f0.data());
      else if (dir == 1) exch_y(f0.data());
      else exch_z(f0.data());
      /* one line at a time: the two cross indices run over the box, the line index over
       * lo-1 .. hi+1 for sc0 and lo .. hi for the update */
      const int a0 = dir == 0 ? 1 : 0, a1 = dir == 2 ? 1 : 2;
      for (int cb = lo[a1]; cb <= hi[a1]; cb++)
        for (int ca = lo[a0]; ca <= hi[a0]; ca++) {
          auto at = [&](int t) {
            int ijk[3];
            ijk[dir] = t; ijk[a0] = ca; ijk[a1] = cb;
            return ih(ijk[0], ijk[1], ijk[2]);
          };
          for (int t = lo[dir] - 1; t <= hi[dir] + 1; t++) {
            const double* pq = p.data() + at(t);
            double dp0 = 0.25 * (-pq[s] + 2.0 * pq[0] - pq[-s]);
            double dp1 = 0.25 * (-pq[2 * s] + 2.0 * pq[s] - pq[0]);
            double dp2 = 0.25 * (-pq[0] + 2.0 * pq[-s] - pq[-2 * s]);
            double ri = 0.5 * (p2(dp0 - dp1) + p2(dp0 - dp2)) / (pq[0] * pq[0]) + 1.0e-16;
            sc0[t] = 0.5 * (1.0 - rth / ri + std::fabs(1.0 - rth / ri));
          }
          for (int t = lo[dir]; t <= hi[dir]; t++) {
            double sc1 = 0.5 * (sc0[t] + sc0[t + 1]);
            double sc2 = 0.5 * (sc0[t] + sc0[t - 1]);
            const long qh = at(t);
            const double* q = f0.data() + qh;
            int ijk[3];
            ijk[dir] = t; ijk[a0] = ca; ijk[a1] = cb;
            f[(long)m * N + in(ijk[0], ijk[1], ijk[2])] =
                q[0] - s0 * (sc1 * (c1 * (q[s] - q[0]) + c2 * (q[2 * s] - q[-s])) -
                             sc2 * (c1 * (q[0] - q[-s]) + c2 * (q[s] - q[-2 * s])));
          }
        }
    }
    return 0;
  }

  /* ---------------- OCFD_analysis pieces (code/others/OCFD_ANA.f90) ---------------- */
  /* ana_box (:197-303): out = tt, Re_lamda, Re_lamdax, Amt, vv_rms, u_rms, v_rms, w_rms,
   * u_skewness, u_flatness, ux_skewness, ux_flatness, E_kinetic, d_rms, T_aver, Amu_aver, d_aver,
   * Ux_rms, Alamdax; sums in the reference's serial loop order */
  void ana_box(double tt, double* out) {
    exch(u.data());
    std::vector<double> uk(N), ui(N), us(N);
    dxyz(0, u.data(), uk.data()); dxyz(1, u.data(), ui.data()); dxyz(2, u.data(), us.data());
    double c_aver = 0, d_aver = 0, amu_aver = 0, T_aver = 0, u_rms = 0, v_rms = 0, w_rms = 0, ux_rms = 0,
           ux_sk = 0, ux_fl = 0, u_sk = 0, u_fl = 0, ek = 0;
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long q = ih(i, j, k), a = in(i, j, k);
          double ux = uk[a] * M[M_AKX][q] + ui[a] * M[M_AIX][q] + us[a] * M[M_ASX][q];
          double gamma = p[q] / Et[q] + 1.0;
          double c1 = std::sqrt(gamma * p[q] / d[q]);
          c_aver = c_aver + c1;
          d_aver = d_aver + d[q];
          amu_aver = amu_aver + Amu[a];
          T_aver = T_aver + T[q];
          u_rms = u_rms + u[q] * u[q];
          v_rms = v_rms + v[q] * v[q];
          w_rms = w_rms + w[q] * w[q];
          ux_rms = ux_rms + ux * ux;
          ux_sk = ux_sk + p3(ux);
          ux_fl = ux_fl + p4(ux);
          u_sk = u_sk + p3(u[q]);
          u_fl = u_fl + p4(u[q]);
          ek = ek + (u[q] * u[q] + v[q] * v[q] + w[q] * w[q]) * d[q] * 0.5;
        }
    double sums[13] = {u_rms, v_rms, w_rms, ux_rms, ux_sk, ux_fl, d_aver, c_aver, amu_aver, ek, T_aver, u_sk, u_fl};
    const double nn = (double)((long)nx * ny * nz);
    for (double& x : sums) x = x / nn;
    double d_rms = 0.0;
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) d_rms = d_rms + p2(d[ih(i, j, k)] - sums[6]);
    ana_box_finish(tt, sums, d_rms, nn, out);
  }
  static void ana_box_finish(double tt, const double* s, double d_rms_sum, double nn, double* out) {
    double u_rms = s[0], v_rms = s[1], w_rms = s[2], ux_rms = s[3], ux_sk = s[4], ux_fl = s[5], d_aver = s[6],
           c_aver = s[7], amu_aver = s[8], ek = s[9], T_aver = s[10], u_sk = s[11], u_fl = s[12];
    double vv_rms = std::sqrt((u_rms + v_rms + w_rms) / 3.0);
    double amt = std::sqrt(u_rms + v_rms + w_rms) / c_aver;
    u_rms = std::sqrt(u_rms); v_rms = std::sqrt(v_rms); w_rms = std::sqrt(w_rms); ux_rms = std::sqrt(ux_rms);
    double alamda = vv_rms / ux_rms, alamdax = u_rms / ux_rms;
    double re_l = vv_rms * alamda * d_aver / amu_aver, re_lx = vv_rms * alamdax * d_aver / amu_aver;
    ux_sk = ux_sk / p3(ux_rms); ux_fl = ux_fl / p4(ux_rms);
    u_sk = u_sk / p3(u_rms); u_fl = u_fl / p4(u_rms);
    double d_rms = std::sqrt(d_rms_sum / nn);
    const double o[19] = {tt, re_l, re_lx, amt, vv_rms, u_rms, v_rms, w_rms, u_sk, u_fl, ux_sk, ux_fl, ek, d_rms,
                          T_aver, amu_aver, d_aver, ux_rms, alamdax};
    for (int m = 0; m < 19; m++) out[m] = o[m];
  }
  /* ana_getQ (:143-190): Q = II of the velocity gradient, interior array */
  void ana_q(double* tk) {
    exch(u.data()); exch(v.data()); exch(w.data());
    std::vector<double> g[9];
    for (auto& x : g) x.resize(N);
    const double* vel[3] = {u.data(), v.data(), w.data()};
    for (int c = 0; c < 3; c++)
      for (int d = 0; d < 3; d++) dxyz(d, vel[c], g[3 * c + d].data());
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long q = ih(i, j, k), a = in(i, j, k);
          auto dd = [&](int c, int x) {  /* d(vel c)/d(x): uk*Akx + ui*Aix + us*Asx for x */
            return g[3 * c][a] * M[M_AKX + x][q] + g[3 * c + 1][a] * M[M_AIX + x][q] + g[3 * c + 2][a] * M[M_ASX + x][q];
          };
          double ux = dd(0, 0), vx = dd(1, 0), wx = dd(2, 0), uy = dd(0, 1), vy = dd(1, 1), wy = dd(2, 1);
          double uz = dd(0, 2), vz = dd(1, 2), wz = dd(2, 2);
          tk[a] = ux * vy + ux * wz + vy * wz - uy * vx - uz * wx - vz * wy;
        }
  }
  /* ana_time_average (:39-140): running means of d, u, v, w, T, di(m), interior arrays */
  std::vector<double> avg;
  int k_average = 0;
  double t_average = 0.0;
  void ana_time_average(double dt) {
    if (avg.empty()) avg.assign((size_t)(5 + NS) * N, 0.0);
    const double K = (double)k_average;
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          long q = ih(i, j, k), a = in(i, j, k);
          const double* src[5] = {d.data(), u.data(), v.data(), w.data(), T.data()};
          for (int m = 0; m < 5; m++) avg[(long)m * N + a] = (K * avg[(long)m * N + a] + src[m][q]) / (K + 1.0);
          for (int m = 0; m < NS; m++)
            avg[(long)(5 + m) * N + a] = (K * avg[(long)(5 + m) * N + a] + di[(long)m * H + q]) / (K + 1.0);
        }
    k_average = k_average + 1;
    t_average = t_average + dt;
  }

  /* nsub x Chemical_time_advance + comput_T_P */
  int chem_advance(double dt2, int nsub) {
    if (!ch.have_kin) { err = "no kinetics"; return OCFD_ERR_PARAM; }
    for (int s = 0; s < nsub; s++) {
#pragma omp parallel for collapse(2)
      for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
          for (int i = 1; i <= nx; i++) {
            long q = ih(i, j, k), a = in(i, j, k);
            double di1[OCFD_MAX_SPEC];
            cell_di(q, di1);
            double Et1 = Et[q], Et0 = Et1;
            ch.time_adv(di1, Et1, dt2);
            for (int m = 0; m < NS; m++) di[(long)m * H + q] = di1[m];
            f[4 * N + a] = f[4 * N + a] + (Et1 - Et0);
            Et[q] = Et1;
          }
    }
    comput_T_P();
    return 0;
  }
};

Oracle* g = nullptr;
std::string g_err;

}  // namespace

extern "C" {

int ocfd_cpu_init(const ocfd_params* p, const ocfd_thermo* th, const ocfd_kinetics* kin, const ocfd_transport* tr,
                  const ocfd_bcdata* bc, const double* coords, const double* metrics) {
  delete g;
  g = new Oracle();
  int e = g->init(p, th, kin, tr, bc, coords, metrics);
  if (e) { g_err = g->err; delete g; g = nullptr; }
  return e;
}

int ocfd_cpu_upload_state(const double* f, const double* di, const double* prims) {
  if (!g) return OCFD_ERR_STATE;
  std::memcpy(g->f.data(), f, sizeof(double) * 5 * g->N);
  std::memcpy(g->di.data(), di, sizeof(double) * g->NS * g->H);
  std::vector<double>* pr[7] = {&g->d, &g->u, &g->v, &g->w, &g->T, &g->p, &g->Et};
  for (int m = 0; m < 7; m++) std::memcpy(pr[m]->data(), prims + (long)m * g->H, sizeof(double) * g->H);
  return 0;
}

int ocfd_cpu_init_state(const double* prim5, const double* di, double tt) {
  if (!g) return OCFD_ERR_STATE;
  int e = g->init_state(prim5, di, tt);
  if (e) g_err = g->err;
  return e;
}

int ocfd_cpu_flow_advance(double dt1, double tt) {
  if (!g) return OCFD_ERR_STATE;
  int e = g->flow_advance(dt1, tt);
  if (e) g_err = g->err;
  return e;
}

int ocfd_cpu_chem_advance(double dt2, int nsub) {
  if (!g) return OCFD_ERR_STATE;
  int e = g->chem_advance(dt2, nsub);
  if (e) g_err = g->err;
  return e;
}

int ocfd_cpu_step(double dt, double tt, int if_reaction, int nsub) {
  if (!g) return OCFD_ERR_STATE;
  double dt1 = 0.5 * dt;
  int e = g->flow_advance(dt1, tt);
  if (!e && if_reaction) e = g->chem_advance(dt / nsub, nsub);
  if (!e) e = g->flow_advance(dt1, tt);
  if (e) g_err = g->err;
  return e;
}

int ocfd_cpu_download_state(double* f, double* di, double* prims) {
  if (!g) return OCFD_ERR_STATE;
  if (f) std::memcpy(f, g->f.data(), sizeof(double) * 5 * g->N);
  if (di) std::memcpy(di, g->di.data(), sizeof(double) * g->NS * g->H);
  if (prims) {
    std::vector<double>* pr[7] = {&g->d, &g->u, &g->v, &g->w, &g->T, &g->p, &g->Et};
    for (int m = 0; m < 7; m++) std::memcpy(prims + (long)m * g->H, pr[m]->data(), sizeof(double) * g->H);
  }
  return 0;
}

int ocfd_cpu_download_rhybrid(double* r) {
  if (!g) return OCFD_ERR_STATE;
  std::memcpy(r, g->Rh.data(), sizeof(double) * g->H);
  return 0;
}

int ocfd_cpu_download_metrics(double* m) {
  if (!g) return OCFD_ERR_STATE;
  for (int k = 0; k < 10; k++) std::memcpy(m + (long)k * g->H, g->M[k].data(), sizeof(double) * g->H);
  return 0;
}

/* show_flow_msg (OCFD_Time_Adv.f90:210-223), serial summation order */
int ocfd_cpu_diag(double* e_mean, double* k_mean) {
  if (!g) return OCFD_ERR_STATE;
  double E1 = 0.0, E2 = 0.0;
  for (int k = 1; k <= g->nz; k++)
    for (int j = 1; j <= g->ny; j++)
      for (int i = 1; i <= g->nx; i++) {
        long q = g->ih(i, j, k), a = g->in(i, j, k);
        double tmp0 = 1.0 / g->M[M_AJAC][q];
        E1 = E1 + g->f[4 * g->N + a] * tmp0;
        E2 = E2 + g->d[q] * (g->u[q] * g->u[q] + g->v[q] * g->v[q] + g->w[q] * g->w[q]) * 0.5 * tmp0;
      }
  double nn = (double)g->nx * g->ny * g->nz;
  *e_mean = E1 / nn;
  *k_mean = E2 / nn;
  return 0;
}

/* Batched 0-D reactors: chemical_timeAdv applied nsub[r] times with dt[r]/nsub[r]. Standalone:
 * needs only thermo + kinetics (no grid). const_p = 1: constant-pressure reactors (cp_restore
 * after every sub-step), 0: the reference's constant-volume reactor. */
int ocfd_cpu_chem_batch(const ocfd_thermo* th, const ocfd_kinetics* kin, int realgas, int timeadv, int n,
                        double* di, double* e, const double* dt, const int* nsub, int nthreads, int const_p) {
  static Chem ch;
  ch.set_thermo(th, realgas);
  ch.kin = *kin;
  ch.nreac = kin->n_reac;
  ch.have_kin = true;
  ch.timeadv = timeadv;
  int ns = th->n_spec;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 64)
  for (int r = 0; r < n; r++) {
    int ks = nsub ? nsub[r] : 1;
    double dt2 = dt[r] / ks;
    double* dr = di + (long)r * ns;
    double h0 = 0.0, p0 = 0.0;
    if (const_p) ch.cp_reference(dr, e[r], h0, p0);
    for (int s = 0; s < ks; s++) {
      ch.time_adv(dr, e[r], dt2);
      if (const_p) ch.cp_restore(dr, e[r], h0, p0);
    }
  }
  return 0;
}

/* Per-species thermo probes for known-answer tests */
double ocfd_cpu_probe(const ocfd_thermo* th, int realgas, int what, const double* di, double x) {
  static Chem ch;
  ch.set_thermo(th, realgas);
  switch (what) {
    case 0: return ch.E_of_T(di, x);
    case 1: return ch.T_of_E(di, x);
    case 2: return ch.P(di, x);
    case 3: { double d = 0; for (int k = 0; k < th->n_spec; k++) d += di[k]; return ch.Cp(d, di, x); }
    default: return ch.gibbs((int)di[0], x);
  }
}

/* Known-answer probes of single building blocks */
int ocfd_cpu_flux_line(int scheme, int plus, const double* v, int n, int bnd0, int bnd1, int sb0, int sb1,
                       const int* scm, double ud7l_diss, double theta1, double theta2, double* hh) {
  SchemeSet S;
  S.scheme = scheme;
  switch (scheme) {
    case 1: S.Ka1 = -2; S.Kb1 = 2; S.Ka2 = -1; S.Kb2 = 3; break;
    case 2: S.Ka1 = -3; S.Kb1 = 3; S.Ka2 = -2; S.Kb2 = 4; break;
    default: S.Ka1 = -3; S.Kb1 = 4; S.Ka2 = -3; S.Kb2 = 4;
  }
  const double UD7[8] = {-3.0, 25.0, -101.0, 319.0, 214.0, -38.0, 4.0, 0.0};
  const double CD8[8] = {-3.0, 29.0, -139.0, 533.0, 533.0, -139.0, 29.0, -3.0};
  for (int k = 0; k < 8; k++) S.UD7L[k] = ud7l_diss * UD7[k] / 420.0 + (1.0 - ud7l_diss) * CD8[k] / 840.0;
  S.theta1 = theta1;
  S.theta2 = theta2;
  int bnd[2] = {bnd0, bnd1}, sb[2] = {sb0, sb1};
  std::vector<int> sc(n + 1, 3);
  if (scm) for (int i = 0; i <= n; i++) sc[i] = scm[i];
  flux_pencil(plus != 0, S, v + 3, hh, n, bnd, sb, sc.data()); /* v[0] is f(1-LAP) */
  return 0;
}

int ocfd_cpu_split(int split, const double* in, double* fp, double* fm) {
  Oracle o;
  o.P.flux_splitting = split;
  double c1 = std::sqrt((in[1] / in[0] + 1.0) * in[1] / in[2]);
  o.split(in[0], in[1], c1, in[2], in[3], in[4], in[5], in[6], in[7], in[8], fp, fm);
  return 0;
}

int ocfd_cpu_gauss(int n, const double* A, const double* b, double* x) {
  Chem c;
  double a[OCFD_MAX_SPEC][OCFD_MAX_SPEC], bb[OCFD_MAX_SPEC];
  for (int i = 0; i < n; i++) {
    bb[i] = b[i];
    for (int j = 0; j < n; j++) a[i][j] = A[i * n + j];
  }
  c.gauss(n, a, bb, x);
  return 0;
}

int ocfd_cpu_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

long long ocfd_cpu_neg_et(void) { return g ? g->neg_et : 0; }
const char* ocfd_cpu_last_error(void) { return g_err.c_str(); }
/* filtering after step istep (OCFD_NS_Solver.f90:48); filter = Para%Filter(100,10) */
int ocfd_cpu_filtering(int istep, int nfiltering, const double* filter, int* applied) {
  if (!g) return OCFD_ERR_STATE;
  int e = g->filtering(istep, nfiltering, filter, applied);
  if (e) g_err = g->err;
  return e;
}
int ocfd_cpu_ana_box(double tt, double* out) {
  if (!g) return OCFD_ERR_STATE;
  g->ana_box(tt, out);
  return 0;
}
int ocfd_cpu_ana_q(double* q) {
  if (!g) return OCFD_ERR_STATE;
  g->ana_q(q);
  return 0;
}
int ocfd_cpu_ana_time_average(double dt, int* k_average, double* t_average) {
  if (!g) return OCFD_ERR_STATE;
  g->ana_time_average(dt);
  if (k_average) *k_average = g->k_average;
  if (t_average) *t_average = g->t_average;
  return 0;
}
int ocfd_cpu_ana_average_download(double* fields) {
  if (!g) return OCFD_ERR_STATE;
  if (g->avg.empty()) return OCFD_ERR_STATE;
  std::memcpy(fields, g->avg.data(), sizeof(double) * g->avg.size());
  return 0;
}

int ocfd_cpu_finalize(void) {
  delete g;
  g = nullptr;
  return 0;
}

}  // extern "C"
