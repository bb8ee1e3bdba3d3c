// Filtering and analysis kernels: the reference's `filtering` (code/others/OCFD_filtering.f90),
// called after every step (OCFD_NS_Solver.f90:48), and the device parts of OCFD_analysis
// (code/others/OCFD_ANA.f90: ana_box statistics, ana_getQ, ana_time_average).
#pragma once
#include "ocfd_flow.cuh"

namespace ocfd {

// a filter pass covers the cells lo..hi (inclusive, per direction) after the reference's clamps
struct FilterBox {
  int lo[3], hi[3];
};

// index s + o along a sweep of n cells; a periodic direction wraps, which is what the halo
// exchange of a single rank (exchange_boundary_x/y/z, OCFD_mpi.f90:201-236) puts in the halo
__device__ __forceinline__ int wrap_index(int s, int n, bool per) {
  if (!per) return s;
  return s < 1 ? s + n : (s > n ? s - n : s);
}

__device__ __forceinline__ bool box_cell(const FilterBox& b, long long t, int& i, int& j, int& k) {
  const int ni = b.hi[0] - b.lo[0] + 1, nj = b.hi[1] - b.lo[1] + 1, nk = b.hi[2] - b.lo[2] + 1;
  if (t >= (long long)ni * nj * nk) return false;
  i = b.lo[0] + (int)(t % ni);
  j = b.lo[1] + (int)((t / ni) % nj);
  k = b.lo[2] + (int)(t / ni / nj);
  return true;
}

// filter_x3d / filter_y3d / filter_z3d (OCFD_filtering.f90:78-189): 9-point Bogey-Bailly filter of
// the five conserved variables; f0 is the unfiltered copy (interior layout of f), the box already
// excludes the last five points of a non-periodic direction, so no halo point is read there
template <int DIR>
__global__ void k_filter_fo9p(double* f, const double* f0, FilterBox b, double s0) {
  int i, j, k;
  if (!box_cell(b, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const double d0 = 0.243527493120, d1 = -0.204788880640, d2 = 0.120007591680, d3 = -0.045211119360,
               d4 = 0.008228661760;
  const int n = DIR == 0 ? cC.nx : (DIR == 1 ? cC.ny : cC.nz);
  const bool per = cC.iper[DIR];
  const int s = DIR == 0 ? i : (DIR == 1 ? j : k);
  int idx[9];  // interior offsets of the points s-4 .. s+4
#pragma unroll
  for (int o = -4; o <= 4; o++) {
    const int t = wrap_index(s + o, n, per);
    idx[o + 4] = DIR == 0 ? nidx(t, j, k) : (DIR == 1 ? nidx(i, t, k) : nidx(i, j, t));
  }
  const long long N = cC.N;
#pragma unroll
  for (int m = 0; m < 5; m++) {
    const double* g = f0 + (size_t)m * N;
    const double c = g[idx[4]];
    f[(size_t)m * N + idx[4]] =
        c - s0 * (d0 * c + d1 * (g[idx[3]] + g[idx[5]]) + d2 * (g[idx[2]] + g[idx[6]]) +
                  d3 * (g[idx[1]] + g[idx[7]]) + d4 * (g[idx[0]] + g[idx[8]]));
  }
}

// filter_x3d_shock / _y3d_ / _z3d_ (OCFD_filtering.f90:194-360): the switch sc0 at s-1, s, s+1
// from the pressure (comput_flow_variables has just run), then the 4-point dissipative filter.
// Each thread evaluates its three sc0 values itself; sc0 is a function of p alone, so every
// cell sees the values the reference's line array holds.
template <int DIR>
__global__ void k_filter_shock(double* f, const double* f0, const double* p, FilterBox b, double s0, double rth) {
  int i, j, k;
  if (!box_cell(b, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const double c1 = -0.210383, c2 = 0.039617;
  const int n = DIR == 0 ? cC.nx : (DIR == 1 ? cC.ny : cC.nz);
  const bool per = cC.iper[DIR];
  const int s = DIR == 0 ? i : (DIR == 1 ? j : k);
  auto P = [&](int o) {
    const int t = wrap_index(s + o, n, per);
    return p[DIR == 0 ? hidx(t, j, k) : (DIR == 1 ? hidx(i, t, k) : hidx(i, j, t))];
  };
  double sc[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int o = c - 1;
    const double pm2 = P(o - 2), pm1 = P(o - 1), p0 = P(o), pp1 = P(o + 1), pp2 = P(o + 2);
    const double dp0 = 0.25 * (-pp1 + 2.0 * p0 - pm1);
    const double dp1 = 0.25 * (-pp2 + 2.0 * pp1 - p0);
    const double dp2 = 0.25 * (-p0 + 2.0 * pm1 - pm2);
    const double ri = 0.5 * (q2(dp0 - dp1) + q2(dp0 - dp2)) / (p0 * p0) + 1.0e-16;
    sc[c] = 0.5 * (1.0 - rth / ri + fabs(1.0 - rth / ri));
  }
  const double sc1 = 0.5 * (sc[1] + sc[2]);
  const double sc2 = 0.5 * (sc[1] + sc[0]);
  int idx[5];  // s-2 .. s+2
#pragma unroll
  for (int o = -2; o <= 2; o++) {
    const int t = wrap_index(s + o, n, per);
    idx[o + 2] = DIR == 0 ? nidx(t, j, k) : (DIR == 1 ? nidx(i, t, k) : nidx(i, j, t));
  }
  const long long N = cC.N;
#pragma unroll
  for (int m = 0; m < 5; m++) {
    const double* g = f0 + (size_t)m * N;
    const double fm2 = g[idx[0]], fm1 = g[idx[1]], f00 = g[idx[2]], fp1 = g[idx[3]], fp2 = g[idx[4]];
    f[(size_t)m * N + idx[2]] =
        f00 - s0 * (sc1 * (c1 * (fp1 - f00) + c2 * (fp2 - fm1)) - sc2 * (c1 * (f00 - fm1) + c2 * (fp1 - fm2)));
  }
}

// comput_vis_coeff for one species (the Amu that comput_Amu_Amk_AMD, OCFD_Time_Adv.f90:35,
// leaves at the start of a stage), kept for ana_box: the single-species stage computes it inline
__global__ void k_amu1(const double* T, const double* di, double* amu) {
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const int q = hidx(i, j, k);
  double Xi[1];
  Xi[0] = di[q] / cC.Mi[0];
  const double X0 = Xi[0];
  Xi[0] = Xi[0] / X0;
  amu[nidx(i, j, k)] = dev_viscosity<1>(T[q], Xi);
}

// fixed-order block sums of NQ per-thread values (256 threads) into partial[NQ * block + m]
template <int NQ>
__device__ __forceinline__ void block_sums(double (&v)[NQ], double* partial) {
  __shared__ double s[NQ][256];
#pragma unroll
  for (int m = 0; m < NQ; m++) s[m][threadIdx.x] = v[m];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
#pragma unroll
      for (int m = 0; m < NQ; m++) s[m][threadIdx.x] = s[m][threadIdx.x] + s[m][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < NQ) partial[(size_t)NQ * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

// ana_box (OCFD_ANA.f90:219-243): the thirteen cell sums, in the reference's atmp1 order
// u^2, v^2, w^2, ux^2, ux^3, ux^4, d, c, Amu, kinetic energy, T, u^3, u^4
template <bool SEP>
__global__ void __launch_bounds__(256) k_ana_box(const double* d, const double* u, const double* v, const double* w,
                                                 const double* T, const double* p, const double* Et,
                                                 const double* amu, double* partial, Geo g) {
  double s[13];
#pragma unroll
  for (int m = 0; m < 13; m++) s[m] = 0.0;
  int i, j, k;
  if (cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) {
    const int q = hidx(i, j, k);
    const double uk = cdiff(u, q, 0, i, cC.nx), ui = cdiff(u, q, 1, j, cC.ny), us = cdiff(u, q, 2, k, cC.nz);
    double A[9], A1[9];
    metric_all<SEP>(g, i, j, k, q, A, A1);
    const double ux = uk * A[0] + ui * A[3] + us * A[6];
    const double gamma = p[q] / Et[q] + 1.0;
    const double c1 = sqrt(gamma * p[q] / d[q]);
    const double uq = u[q], vq = v[q], wq = w[q], dq = d[q];
    s[0] = uq * uq;
    s[1] = vq * vq;
    s[2] = wq * wq;
    s[3] = ux * ux;
    s[4] = q3(ux);
    s[5] = q4(ux);
    s[6] = dq;
    s[7] = c1;
    s[8] = amu[nidx(i, j, k)];
    s[9] = (uq * uq + vq * vq + wq * wq) * dq * 0.5;
    s[10] = T[q];
    s[11] = q3(uq);
    s[12] = q4(uq);
  }
  block_sums<13>(s, partial);
}

// d_rms (OCFD_ANA.f90:277-286): sum of (d - d_aver)^2
__global__ void __launch_bounds__(256) k_ana_drms(const double* d, double d_aver, double* partial) {
  double s[1] = {0.0};
  int i, j, k;
  if (cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) s[0] = q2(d[hidx(i, j, k)] - d_aver);
  block_sums<1>(s, partial);
}

// ana_getQ (OCFD_ANA.f90:152-181): Q = ux vy + ux wz + vy wz - uy vx - uz wx - vz wy
template <bool SEP>
__global__ void k_ana_q(const double* u, const double* v, const double* w, double* tk, Geo g) {
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const int q = hidx(i, j, k);
  double A[9], A1[9];
  metric_all<SEP>(g, i, j, k, q, A, A1);
  const double* vel[3] = {u, v, w};
  double gr[3][3];  // gr[c][x] = d(vel c)/dx
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const double dk = cdiff(vel[c], q, 0, i, cC.nx), di = cdiff(vel[c], q, 1, j, cC.ny),
                 ds = cdiff(vel[c], q, 2, k, cC.nz);
#pragma unroll
    for (int x = 0; x < 3; x++) gr[c][x] = dk * A[x] + di * A[3 + x] + ds * A[6 + x];
  }
  const double ux = gr[0][0], vx = gr[1][0], wx = gr[2][0], uy = gr[0][1], vy = gr[1][1], wy = gr[2][1];
  const double uz = gr[0][2], vz = gr[1][2], wz = gr[2][2];
  tk[nidx(i, j, k)] = ux * vy + ux * wz + vy * wz - uy * vx - uz * wx - vz * wy;
}

// ana_time_average (OCFD_ANA.f90:92-111): running means of d, u, v, w, T and every di
template <int NS>
__global__ void k_ana_average(const double* d, const double* u, const double* v, const double* w, const double* T,
                              const double* di, double* avg, double K) {
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const int q = hidx(i, j, k), nn = nidx(i, j, k);
  const long long N = cC.N;
  const double* src[5] = {d, u, v, w, T};
#pragma unroll
  for (int m = 0; m < 5; m++) avg[(size_t)m * N + nn] = (K * avg[(size_t)m * N + nn] + src[m][q]) / (K + 1.0);
#pragma unroll
  for (int m = 0; m < NS; m++)
    avg[(size_t)(5 + m) * N + nn] = (K * avg[(size_t)(5 + m) * N + nn] + di[(size_t)m * cC.H + q]) / (K + 1.0);
}

// save_flow_data's content (OCFD_IO.f90:39-64): d, u, v, w, T and every di, as interior arrays,
// packed into one buffer for a single device-to-host copy
__global__ void k_pack_snapshot(const double* d, const double* u, const double* v, const double* w, const double* T,
                                const double* di, int ns, double* out) {
  int i, j, k;
  if (!cell_of((long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const int q = hidx(i, j, k), nn = nidx(i, j, k);
  const long long N = cC.N;
  out[nn] = d[q];
  out[N + nn] = u[q];
  out[2 * N + nn] = v[q];
  out[3 * N + nn] = w[q];
  out[4 * N + nn] = T[q];
  for (int m = 0; m < ns; m++) out[(size_t)(5 + m) * N + nn] = di[(size_t)m * cC.H + q];
}

// final sums of NQ per-block partials on the device (one block of 256 threads, fixed order:
// thread t adds blocks t, t + 256, ... in turn, then a tree), so that a reduction needs no host
// round trip
template <int NQ>
__global__ void __launch_bounds__(256) k_sum_partials(const double* partial, int nb, double* out) {
  double v[NQ];
#pragma unroll
  for (int m = 0; m < NQ; m++) v[m] = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
    for (int m = 0; m < NQ; m++) v[m] = v[m] + partial[(size_t)NQ * b + m];
  block_sums<NQ>(v, out);
}

}  // namespace ocfd
