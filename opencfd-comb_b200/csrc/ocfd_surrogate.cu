// Learned chemistry surrogate: a BF16 MLP (12 -> 256 -> 256 -> 256 -> 10 for the 9-species H2-air
// mechanism, GELU) that maps one reactor state (T, log p, Y_k, log dt) to its increments (dY_k, dT)
// over dt, trained on the GPU with the tcgen05 GEMM of ocfd_mlp.cu on states that the FP64 implicit
// integrator itself produced, and applied behind a gate with FP64 fallback.
//
// Conservation: the predicted dY is projected onto the null space of the element-mass matrix
// (element and total mass are conserved exactly), the energy update follows update_et (the
// reference's formation-enthalpy bookkeeping) and T comes from the conserved energy with the FP64
// Newton inversion. The predicted dT is therefore not used for the state: it is the error proxy.
// A reactor is accepted when |dT_pred - dT_energy| <= tol_T, no mass fraction falls below -1e-6
// (trace radicals may dip below zero by the network's error) and the input lies inside the training
// range; the others run through the FP64 integrator (work queue).
// No counterpart in the reference.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "ocfd_chem.cuh"
#include "ocfd_mlp.h"

namespace ocfd {
void launch_chem_batch(int ns, int sms, int n, double* di, double* e, const double* dt, const int* nsub,
                       const int* perm, int* counter, int* nfail, cudaStream_t st);
int current_nspec();
int current_const_p();
cudaStream_t current_stream();

namespace sg {

constexpr int HID = 256, PAD = 16;  // hidden width; padded input / output width
constexpr int NLAYER = 4;
constexpr double Y_STD_FLOOR = 1.0e-3;  // smallest normalisation scale of a mass fraction input

struct Norm {  // per-column affine maps and the training range of the raw inputs
  float in_mean[PAD], in_std[PAD], out_mean[PAD], out_std[PAD];
  float in_min[PAD], in_max[PAD];
};

struct State {
  int ns = 0, nin = 0, nout = 0;
  bool trained = false;
  float *w[NLAYER] = {}, *b[NLAYER] = {}, *mw[NLAYER] = {}, *vw[NLAYER] = {}, *mb[NLAYER] = {}, *vb[NLAYER] = {};
  __nv_bfloat16* wb[NLAYER] = {};
  int rows[NLAYER] = {HID, HID, HID, PAD}, cols[NLAYER] = {PAD, HID, HID, HID};
  Norm norm{};
  Norm* d_norm = nullptr;
  double* d_proj = nullptr;  // ns x ns element projection
  int* d_err = nullptr;
  unsigned char* d_wpack = nullptr;  // weights packed for the fused inference kernel
  long long adam_t = 0;
};
State S;

__host__ __device__ inline size_t wsize(int l) { return (size_t)(l == 3 ? PAD : HID) * (l == 0 ? PAD : HID); }

// ---------------------------------------------------------------- per-reactor features
// raw inputs: T, log p, Y_1..Y_ns, log dt (T from the energy by the FP64 Newton inversion)
template <int NS>
__global__ void k_raw_inputs(int n, const double* __restrict__ di, const double* __restrict__ e,
                             const double* __restrict__ dt, float* __restrict__ raw, double* __restrict__ T0,
                             int* nfail) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double d[NS], rho = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    d[k] = di[(size_t)r * NS + k];
    rho += d[k];
  }
  const double T = dev_T<NS>(d, e[r], nfail);
  const double p = dev_P<NS>(d, T);
  float* o = raw + (size_t)r * PAD;
  o[0] = (float)T;
  o[1] = (float)log(p);
#pragma unroll
  for (int k = 0; k < NS; k++) o[2 + k] = (float)(d[k] / rho);
  o[2 + NS] = (float)log(dt[r]);
  for (int c = NS + 3; c < PAD; c++) o[c] = 0.0f;
  T0[r] = T;
}
// raw targets: dY_k, dT of the FP64 integrator
template <int NS>
__global__ void k_raw_targets(int n, const double* __restrict__ di0, const double* __restrict__ di1,
                              const double* __restrict__ e1, const double* __restrict__ T0, float* __restrict__ raw,
                              int* nfail) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double a[NS], b[NS], ra = 0.0, rb = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    a[k] = di0[(size_t)r * NS + k];
    b[k] = di1[(size_t)r * NS + k];
    ra += a[k];
    rb += b[k];
  }
  const double T1 = dev_T<NS>(b, e1[r], nfail);
  float* o = raw + (size_t)r * PAD;
#pragma unroll
  for (int k = 0; k < NS; k++) o[k] = (float)(b[k] / rb - a[k] / ra);
  o[NS] = (float)(T1 - T0[r]);
  for (int c = NS + 1; c < PAD; c++) o[c] = 0.0f;
}
// per-block partial column statistics: part[block][0..3][PAD] = sum, sum of squares, min, max
constexpr int STAT_THREADS = 256;
__global__ void __launch_bounds__(STAT_THREADS) k_colstats(int n, const float* __restrict__ x, double* part) {
  __shared__ double red[4][PAD][STAT_THREADS / 32];
  double s1[PAD], s2[PAD], mn[PAD], mx[PAD];
#pragma unroll
  for (int c = 0; c < PAD; c++) { s1[c] = 0.0; s2[c] = 0.0; mn[c] = 1.0e300; mx[c] = -1.0e300; }
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < PAD; c++) {
      const double v = x[(size_t)r * PAD + c];
      s1[c] += v; s2[c] += v * v; mn[c] = fmin(mn[c], v); mx[c] = fmax(mx[c], v);
    }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < PAD; c++) {
    for (int o = 16; o > 0; o >>= 1) {
      s1[c] += __shfl_down_sync(0xffffffffu, s1[c], o);
      s2[c] += __shfl_down_sync(0xffffffffu, s2[c], o);
      mn[c] = fmin(mn[c], __shfl_down_sync(0xffffffffu, mn[c], o));
      mx[c] = fmax(mx[c], __shfl_down_sync(0xffffffffu, mx[c], o));
    }
    if (lane == 0) { red[0][c][w] = s1[c]; red[1][c][w] = s2[c]; red[2][c][w] = mn[c]; red[3][c][w] = mx[c]; }
  }
  __syncthreads();
  if (threadIdx.x < 4 * PAD) {
    const int q = threadIdx.x / PAD, c = threadIdx.x % PAD;
    double acc = red[q][c][0];
    for (int k = 1; k < STAT_THREADS / 32; k++) {
      const double v = red[q][c][k];
      acc = q < 2 ? acc + v : (q == 2 ? fmin(acc, v) : fmax(acc, v));
    }
    part[((size_t)blockIdx.x * 4 + q) * PAD + c] = acc;
  }
}
// affine map of the columns into BF16 network inputs (or FP32 targets); columns >= ncol are zero
__global__ void k_normalize(int n, int ncol, const float* __restrict__ raw, const float* __restrict__ mean,
                            const float* __restrict__ sd, __nv_bfloat16* __restrict__ xb, float* __restrict__ xf) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * PAD) return;
  const int c = (int)(t % PAD);
  const float v = c < ncol ? (raw[t] - mean[c]) / sd[c] : 0.0f;
  if (xb) xb[t] = __float2bfloat16(v);
  if (xf) xf[t] = v;
}
// gather rows (training shuffle)
__global__ void k_gather_rows(int n, const int* __restrict__ perm, const __nv_bfloat16* __restrict__ xs,
                              const float* __restrict__ ts, __nv_bfloat16* __restrict__ xd, float* __restrict__ td) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * PAD) return;
  const long long r = t / PAD, c = t % PAD;
  const long long src = (long long)perm[r] * PAD + c;
  xd[t] = xs[src];
  td[t] = ts[src];
}
// mean-squared-error gradient over the used output columns (and the loss, summed in double)
__global__ void k_loss_grad(int B, int nout, const float* __restrict__ out, const float* __restrict__ tgt,
                            float* __restrict__ gf, __nv_bfloat16* __restrict__ gb, double* loss) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)B * PAD) return;
  const int c = (int)(t % PAD);
  float g = 0.0f;
  if (c < nout) {
    const float d = out[t] - tgt[t];
    g = 2.0f * d / (float)((long long)B * nout);
    atomicAdd(loss, (double)d * (double)d / ((double)B * nout));
  }
  gf[t] = g;
  gb[t] = __float2bfloat16(g);
}
// bias gradient: column sums of an FP32 B x ncol matrix; block = one column, threads over rows
__global__ void k_colsum(int B, int ncol, const float* __restrict__ g, float* __restrict__ out) {
  __shared__ float red[8];
  const int c = blockIdx.x;
  float s = 0.0f;
  for (int r = threadIdx.x; r < B; r += blockDim.x) s += g[(size_t)r * ncol + c];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    out[c] = t;
  }
}
// Adam step on FP32 master parameters, refreshing the BF16 copy
__global__ void k_adam(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, __nv_bfloat16* __restrict__ pb, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.0f - b1) * gt, vt = b2 * v[t] + (1.0f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  const float pt = p[t] - lr * (mt / c1) / (sqrtf(vt / c2) + eps);
  p[t] = pt;
  if (pb) pb[t] = __float2bfloat16(pt);
}
__global__ void k_to_bf16(long long n, const float* __restrict__ p, __nv_bfloat16* __restrict__ pb) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) pb[t] = __float2bfloat16(p[t]);
}

// network output -> reactor update. dY is de-normalised and projected on the element-conserving
// subspace, the energy follows update_et, T comes from the energy; the gate compares that T with
// the network's own dT. mode 0: write every reactor to the outputs (ungated); mode 1: write the
// accepted reactors in place and list the others for the FP64 integrator.
// every mass fraction input inside its training range widened by half a normalised unit (its
// training standard deviation, at least Y_STD_FLOOR): the network sees no input far outside what
// it was trained on. A trace species whose level grows past what the training states held (radicals
// of a mixture that starts to react) would otherwise reach the network as tens or thousands of
// normalised units.
template <int NS>
__device__ __forceinline__ bool mass_fractions_in_range(const float* ri, const Norm* nm) {
  bool in = true;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    const int c = 2 + k;
    const float w = 0.5f * nm->in_std[c];
    in = in && ri[c] >= nm->in_min[c] - w && ri[c] <= nm->in_max[c] + w;
  }
  return in;
}

template <int NS>
__global__ void k_post(int n, int mode, double* __restrict__ di, double* __restrict__ e,
                       const double* __restrict__ T0, const float* __restrict__ raw, const float* __restrict__ out,
                       const Norm* __restrict__ nm, const double* __restrict__ proj, double tol_T,
                       double* __restrict__ di_out, double* __restrict__ e_out, double* __restrict__ T_pred,
                       double* __restrict__ T_energy, int* __restrict__ fb_list, int* __restrict__ fb_count,
                       int base, int* nfail) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double d0[NS], rho = 0.0, dy[NS], d1[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) {
    d0[k] = di[(size_t)r * NS + k];
    rho += d0[k];
  }
  const float* o = out + (size_t)r * PAD;
#pragma unroll
  for (int k = 0; k < NS; k++) dy[k] = (double)o[k] * nm->out_std[k] + nm->out_mean[k];
  const double dTp = (double)o[NS] * nm->out_std[NS] + nm->out_mean[NS];
  bool ok = true;
#pragma unroll
  for (int i = 0; i < NS; i++) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < NS; j++) s += proj[i * NS + j] * dy[j];
    const double y1 = d0[i] / rho + s;
    if (y1 < -1.0e-6) ok = false;  // trace species may dip below zero by the network's own error
    d1[i] = y1 * rho;
  }
  const double e1 = update_et<NS>(d0, d1, e[r]);
  const double T1 = dev_T<NS>(d1, e1, nfail);
  const double T = T0[r];
  if (!(fabs(T1 - T - dTp) <= tol_T)) ok = false;  // also rejects NaN
  const float* ri = raw + (size_t)r * PAD;
  const int chk[3] = {0, 1, NS + 2};  // T, log p, log dt inside the training range
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const int c = chk[q];
    if (!(ri[c] >= nm->in_min[c] && ri[c] <= nm->in_max[c])) ok = false;
  }
  if (!mass_fractions_in_range<NS>(ri, nm)) ok = false;
  if (T_pred) T_pred[r] = T + dTp;
  if (T_energy) T_energy[r] = T1;
  if (mode == 0) {
#pragma unroll
    for (int k = 0; k < NS; k++) di_out[(size_t)r * NS + k] = d1[k];
    e_out[r] = e1;
    return;
  }
  if (ok) {
#pragma unroll
    for (int k = 0; k < NS; k++) di[(size_t)r * NS + k] = d1[k];
    e[r] = e1;
  } else {
    fb_list[atomicAdd(fb_count, 1)] = base + r;
  }
}

// ---------------------------------------------------------------- host side
inline unsigned nb(long long n, int b) { return (unsigned)((n + b - 1) / b); }

struct Gemm {
  int rc = 0;
  void operator()(const __nv_bfloat16* A, long long sam, long long sak, const __nv_bfloat16* B, long long sbn,
                  long long sbk, int M, int N, int K, float* C, long long ldc, __nv_bfloat16* Cb, long long ldcb,
                  float* pre, const float* bias, int beta, int act, cudaStream_t st) {
    mlp::GemmArgs g{};
    g.A = A; g.sam = sam; g.sak = sak;
    g.B = B; g.sbn = sbn; g.sbk = sbk;
    g.C = C; g.ldc = ldc; g.Cb = Cb; g.ldcb = ldcb; g.pre = pre; g.bias = bias;
    g.M = M; g.N = N; g.K = K; g.beta = beta; g.act = act; g.err = S.d_err;
    if (rc == 0) rc = mlp::launch_gemm(g, st);
  }
};

bool g_fused = true;  // inference through the fused four-layer kernel (ocfd_gpu_surrogate_fused)

// forward pass of rows rows of x (BF16, PAD wide): hidden activations into h[0..2] (BF16, HID wide,
// and their pre-activations into pre[0..2] when given), outputs into out (FP32, PAD wide). Without
// pre-activations (inference) the four layers run as one fused kernel; the hidden activations then
// stay on chip and h is not written.
void forward(Gemm& gemm, int rows, const __nv_bfloat16* x, __nv_bfloat16* const* h, float* const* pre, float* out,
             cudaStream_t st) {
  if (!pre && g_fused) {
    mlp::MlpArgs m{};
    m.x = x;
    for (int l = 0; l < NLAYER; l++) {
      m.w[l] = S.wb[l];
      m.b[l] = S.b[l];
    }
    m.out = out;
    m.M = rows;
    m.err = S.d_err;
    m.pack = S.d_wpack;
    if (gemm.rc == 0) gemm.rc = mlp::launch_mlp_fused(m, st);
    return;
  }
  const __nv_bfloat16* in = x;
  long long ld = PAD;
  for (int l = 0; l < 3; l++) {
    gemm(in, ld, 1, S.wb[l], S.cols[l], 1, rows, HID, S.cols[l], nullptr, HID, h[l], HID, pre ? pre[l] : nullptr,
         S.b[l], 0, 1, st);
    in = h[l];
    ld = HID;
  }
  gemm(in, HID, 1, S.wb[3], HID, 1, rows, PAD, HID, out, PAD, nullptr, 0, nullptr, S.b[3], 0, 0, st);
}

int ensure_params(int ns, unsigned seed) {
  S.ns = ns;
  S.nin = ns + 3;
  S.nout = ns + 1;
  if (S.nin > PAD || S.nout > PAD) return -1;
  if (!S.w[0]) {
    for (int l = 0; l < NLAYER; l++) {
      const size_t nw = wsize(l), nbias = S.rows[l];
      if (cudaMalloc(&S.w[l], nw * 4) || cudaMalloc(&S.wb[l], nw * 2) || cudaMalloc(&S.mw[l], nw * 4) ||
          cudaMalloc(&S.vw[l], nw * 4) || cudaMalloc(&S.b[l], nbias * 4) || cudaMalloc(&S.mb[l], nbias * 4) ||
          cudaMalloc(&S.vb[l], nbias * 4))
        return -2;
    }
    if (cudaMalloc(&S.d_norm, sizeof(Norm)) || cudaMalloc(&S.d_proj, sizeof(double) * PAD * PAD) ||
        cudaMalloc(&S.d_err, sizeof(int)) || cudaMalloc(&S.d_wpack, mlp::MLP_PACK_BYTES))
      return -2;
  }
  // He initialisation over the used fan-in; padded rows / columns start (and stay) at zero
  std::mt19937_64 rng(seed);
  for (int l = 0; l < NLAYER; l++) {
    const int R = S.rows[l], Cn = S.cols[l];
    const int fan_in = l == 0 ? S.nin : HID, used_rows = l == 3 ? S.nout : R;
    std::normal_distribution<float> nd(0.0f, (l == 3 ? 0.5f : 1.0f) * std::sqrt(2.0f / fan_in));
    std::vector<float> w((size_t)R * Cn, 0.0f), zb(R, 0.0f);
    for (int i = 0; i < used_rows; i++)
      for (int j = 0; j < (l == 0 ? S.nin : Cn); j++) w[(size_t)i * Cn + j] = nd(rng);
    cudaMemcpy(S.w[l], w.data(), w.size() * 4, cudaMemcpyHostToDevice);
    cudaMemset(S.mw[l], 0, w.size() * 4);
    cudaMemset(S.vw[l], 0, w.size() * 4);
    cudaMemcpy(S.b[l], zb.data(), R * 4, cudaMemcpyHostToDevice);
    cudaMemset(S.mb[l], 0, R * 4);
    cudaMemset(S.vb[l], 0, R * 4);
    k_to_bf16<<<nb(w.size(), 256), 256>>>((long long)w.size(), S.w[l], S.wb[l]);
  }
  S.adam_t = 0;
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}

template <int NS>
__global__ void k_temperature(int n, const double* __restrict__ di, const double* __restrict__ e, double* __restrict__ T,
                              int* nfail) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double d[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) d[k] = di[(size_t)r * NS + k];
  T[r] = dev_T<NS>(d, e[r], nfail);
}
template <int NS>
void launch_temperature(int n, const double* di, const double* e, double* T, int* nf, cudaStream_t st) {
  k_temperature<NS><<<nb(n, 128), 128, 0, st>>>(n, di, e, T, nf);
}
template <int NS>
void launch_raw_inputs(int n, const double* di, const double* e, const double* dt, float* raw, double* T0, int* nf,
                       cudaStream_t st) {
  k_raw_inputs<NS><<<nb(n, 128), 128, 0, st>>>(n, di, e, dt, raw, T0, nf);
}
template <int NS>
void launch_raw_targets(int n, const double* di0, const double* di1, const double* e1, const double* T0, float* raw,
                        int* nf, cudaStream_t st) {
  k_raw_targets<NS><<<nb(n, 128), 128, 0, st>>>(n, di0, di1, e1, T0, raw, nf);
}
template <int NS>
void launch_post(int n, int mode, double* di, double* e, const double* T0, const float* raw, const float* out,
                 double tol, double* dio, double* eo, double* Tp, double* Te, int* fb, int* fbn, int base, int* nf,
                 cudaStream_t st) {
  k_post<NS><<<nb(n, 128), 128, 0, st>>>(n, mode, di, e, T0, raw, out, S.d_norm, S.d_proj, tol, dio, eo, Tp, Te, fb,
                                         fbn, base, nf);
}
#define SG_DISPATCH(NSV, CALL)                                           \
  switch (NSV) {                                                         \
    case 2: { constexpr int NSC = 2; CALL; } break;                      \
    case 3: { constexpr int NSC = 3; CALL; } break;                      \
    case 4: { constexpr int NSC = 4; CALL; } break;                      \
    case 5: { constexpr int NSC = 5; CALL; } break;                      \
    case 6: { constexpr int NSC = 6; CALL; } break;                      \
    case 7: { constexpr int NSC = 7; CALL; } break;                      \
    case 8: { constexpr int NSC = 8; CALL; } break;                      \
    case 9: { constexpr int NSC = 9; CALL; } break;                      \
    default: return -1;                                                  \
  }

// column statistics of a raw n x PAD FP32 array (host reduction of per-block partials)
// sd_floor replaces the standard deviation of a column that does not vary (above the rounding of
// the variance): 1 for inputs, so that a constant input maps to 0
int column_stats(int n, const float* raw, double* mean, double* sd, double* mn, double* mx, double sd_floor,
                 cudaStream_t st) {
  const int blocks = 592;
  double* part = nullptr;
  if (cudaMalloc(&part, sizeof(double) * blocks * 4 * PAD)) return -2;
  k_colstats<<<blocks, STAT_THREADS, 0, st>>>(n, raw, part);
  std::vector<double> h((size_t)blocks * 4 * PAD);
  cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) { cudaFree(part); return -2; }
  cudaFree(part);
  for (int c = 0; c < PAD; c++) {
    double s1 = 0, s2 = 0, a = 1e300, b = -1e300;
    for (int k = 0; k < blocks; k++) {
      s1 += h[((size_t)k * 4 + 0) * PAD + c];
      s2 += h[((size_t)k * 4 + 1) * PAD + c];
      a = std::min(a, h[((size_t)k * 4 + 2) * PAD + c]);
      b = std::max(b, h[((size_t)k * 4 + 3) * PAD + c]);
    }
    mean[c] = s1 / n;
    const double var = std::max(s2 / n - mean[c] * mean[c], 0.0);
    // a column varies when its variance stands above the rounding of s2 / n - mean^2
    const bool varies = var > 1e-20 * mean[c] * mean[c] && var > 1e-60;
    sd[c] = varies ? std::sqrt(var) : sd_floor;
    mn[c] = a;
    mx[c] = b;
  }
  return 0;
}


// ---------------------------------------------------------------- flow cells (Chemical_time_advance)
// the surrogate inside the Strang step: cells are read in place from the halo arrays, the gate
// decides per cell, rejected cells go to a device list that k_chem_cells_list advances with the
// FP64 sub-steps of the plain path; no host synchronisation, so the step stays one CUDA graph
template <int NS>
__global__ void k_cell_inputs(int c0, int rows, const double* __restrict__ di, const double* __restrict__ Et,
                              double dtc, const Norm* __restrict__ nm, int nin, float* __restrict__ raw,
                              double* __restrict__ T0, __nv_bfloat16* __restrict__ xb, int* nfail) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const int t = c0 + r;
  const int i = t % cC.nx + 1, j = (t / cC.nx) % cC.ny + 1, k = t / cC.nx / cC.ny + 1;
  const int q = hidx(i, j, k);
  double d[NS], rho = 0.0;
#pragma unroll
  for (int m = 0; m < NS; m++) {
    d[m] = di[(size_t)m * cC.H + q];
    rho += d[m];
  }
  const double T = dev_T<NS>(d, Et[q], nfail);
  const double p = dev_P<NS>(d, T);
  float v[PAD];
  v[0] = (float)T;
  v[1] = (float)log(p);
#pragma unroll
  for (int m = 0; m < NS; m++) v[2 + m] = (float)(d[m] / rho);
  v[2 + NS] = (float)log(dtc);
  for (int c = NS + 3; c < PAD; c++) v[c] = 0.0f;
  float* o = raw + (size_t)r * PAD;
#pragma unroll
  for (int c = 0; c < PAD; c++) {
    o[c] = v[c];
    xb[(size_t)r * PAD + c] = __float2bfloat16(c < nin ? (v[c] - nm->in_mean[c]) / nm->in_std[c] : 0.0f);
  }
  T0[r] = T;
}
template <int NS>
__global__ void k_cell_post(int c0, int rows, double* __restrict__ f, double* __restrict__ Et, double* __restrict__ Tf,
                            double* __restrict__ pf, double* __restrict__ di, const double* __restrict__ T0,
                            const float* __restrict__ raw, const float* __restrict__ out, const Norm* __restrict__ nm,
                            const double* __restrict__ proj, double tol_T, int* __restrict__ list,
                            int* __restrict__ count, int* nfail) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const int t = c0 + r;
  const int i = t % cC.nx + 1, j = (t / cC.nx) % cC.ny + 1, k = t / cC.nx / cC.ny + 1;
  const int q = hidx(i, j, k);
  double d0[NS], rho = 0.0, dy[NS], d1[NS];
#pragma unroll
  for (int m = 0; m < NS; m++) {
    d0[m] = di[(size_t)m * cC.H + q];
    rho += d0[m];
  }
  const float* o = out + (size_t)r * PAD;
#pragma unroll
  for (int m = 0; m < NS; m++) dy[m] = (double)o[m] * nm->out_std[m] + nm->out_mean[m];
  const double dTp = (double)o[NS] * nm->out_std[NS] + nm->out_mean[NS];
  // rejection reasons, counted in count[2..7]: negative composition, temperature check, T, log p and
  // log dt outside the training range, a mass fraction outside its (widened) training range
  int why = 0;
#pragma unroll
  for (int a = 0; a < NS; a++) {
    double sacc = 0.0;
#pragma unroll
    for (int b = 0; b < NS; b++) sacc += proj[a * NS + b] * dy[b];
    const double y1 = d0[a] / rho + sacc;
    // the flow path tolerates larger dips: Rescaling_di clips negative densities at the next stage
    if (y1 < -1.0e-4) why |= 1;
    d1[a] = y1 * rho;
  }
  const double e0 = Et[q];
  const double e1 = update_et<NS>(d0, d1, e0);
  const double T1 = dev_T<NS>(d1, e1, nfail);
  if (!(fabs(T1 - T0[r] - dTp) <= tol_T)) why |= 2;
  const float* ri = raw + (size_t)r * PAD;
  const int chk[3] = {0, 1, NS + 2};
#pragma unroll
  for (int qq = 0; qq < 3; qq++) {
    const int c = chk[qq];
    if (!(ri[c] >= nm->in_min[c] && ri[c] <= nm->in_max[c])) why |= 4 << qq;
  }
  if (!mass_fractions_in_range<NS>(ri, nm)) why |= 32;
  if (why) {
    list[atomicAdd(count, 1)] = t;
#pragma unroll
    for (int b = 0; b < 6; b++)
      if (why >> b & 1) atomicAdd(count + 2 + b, 1);
    return;
  }
#pragma unroll
  for (int m = 0; m < NS; m++) di[(size_t)m * cC.H + q] = d1[m];
  Et[q] = e1;
  f[4 * cC.N + t] = f[4 * cC.N + t] + (e1 - e0);
  Tf[q] = T1;
  pf[q] = dev_P<NS>(d1, T1);
}
// Chemical_time_advance + comput_T_P for the listed cells (k_chem_cells on a cell list whose length
// is read on the device)
template <int NS>
__global__ void __launch_bounds__(OCFD_CHEM_TPB, OCFD_CHEM_MINB) k_chem_cells_list(
    const int* __restrict__ list, const int* __restrict__ count, double* f, double* Et, double* T, double* p,
    double* di, double dt2, int nsub, int* nfail) {
  __shared__ double sA[NS * NS * OCFD_CHEM_TPB];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= *count) return;
  const int t = list[idx];
  const int i = t % cC.nx + 1, j = (t / cC.nx) % cC.ny + 1, k = t / cC.nx / cC.ny + 1;
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
    zero = chem_step<NS, OCFD_CHEM_TPB>(d1, e, dt2, nfail, slab) || zero;
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

struct Cells {
  long long N = 0;
  int chunk = 0;
  float* raw = nullptr;
  double* T0 = nullptr;
  __nv_bfloat16 *xb = nullptr, *hA = nullptr, *hB = nullptr;
  float* out = nullptr;
  int* list = nullptr;
  int* count = nullptr;  // [0] rejected cells of the current call, [1] their total since set-up
  double tol = 5.0;
};
Cells CS;

template <int NS>
int cells_chem_t(double* f, double* Et, double* T, double* p, double* di, double dt2, int nsub, int* nfail,
                 cudaStream_t st) {
  const long long N = CS.N;
  cudaMemsetAsync(CS.count, 0, 8 * sizeof(int), st);
  Gemm gemm;
  __nv_bfloat16* hs[3] = {CS.hA, CS.hB, CS.hA};
  for (long long c0 = 0; c0 < N; c0 += CS.chunk) {
    const int rows = (int)std::min<long long>(CS.chunk, N - c0);
    k_cell_inputs<NS><<<nb(rows, 128), 128, 0, st>>>((int)c0, rows, di, Et, dt2 * nsub, S.d_norm, S.nin, CS.raw,
                                                    CS.T0, CS.xb, nfail);
    forward(gemm, rows, CS.xb, hs, nullptr, CS.out, st);
    if (gemm.rc) return gemm.rc;  // the network did not run: its outputs would be stale
    k_cell_post<NS><<<nb(rows, 128), 128, 0, st>>>((int)c0, rows, f, Et, T, p, di, CS.T0, CS.raw, CS.out, S.d_norm,
                                                  S.d_proj, CS.tol, CS.list, CS.count, nfail);
  }
  k_chem_cells_list<NS><<<nb(N, OCFD_CHEM_TPB), OCFD_CHEM_TPB, 0, st>>>(CS.list, CS.count, f, Et, T, p, di, dt2, nsub, nfail);
  return 0;
}

// mode 1: allocate the chunk buffers for N cells (called outside any stream capture)
int cells_setup(long long N, double tol) {
  if (!S.trained) return -5;
  if (g_fused && mlp::prepare_mlp_fused() != 0) return -2;
  if (CS.N != N) {
    void* ptrs[] = {CS.raw, CS.T0, CS.xb, CS.hA, CS.hB, CS.out, CS.list, CS.count};
    for (void* q : ptrs)
      if (q) cudaFree(q);
    CS = Cells{};
    CS.N = N;
    CS.chunk = (int)std::min<long long>(N, 1 << 20);
    const size_t ch = CS.chunk;
    if (cudaMalloc(&CS.raw, ch * PAD * 4) || cudaMalloc(&CS.T0, ch * 8) || cudaMalloc(&CS.xb, ch * PAD * 2) ||
        cudaMalloc(&CS.hA, ch * HID * 2) || cudaMalloc(&CS.hB, ch * HID * 2) || cudaMalloc(&CS.out, ch * PAD * 4) ||
        cudaMalloc(&CS.list, (size_t)N * 4) || cudaMalloc(&CS.count, 64))
      return -2;
  }
  CS.tol = tol;
  return 0;
}

}  // namespace sg

// the flow solver's chemistry through the gated surrogate (ocfd_gpu.cu, chemistry mode 1)
int sg_cells_chem(int ns, double* f, double* Et, double* T, double* p, double* di, double dt2, int nsub, int* nfail,
                  cudaStream_t st) {
  using namespace sg;
  if (!S.trained || S.ns != ns || CS.N <= 0) return -5;
  int rc = 0;
  SG_DISPATCH(ns, rc = cells_chem_t<NSC>(f, Et, T, p, di, dt2, nsub, nfail, st));
  return rc;
}
// 1 when a network kernel ran out of a bounded wait since the last call (the word is cleared)
int sg_device_error(cudaStream_t st) {
  using namespace sg;
  if (!S.d_err) return 0;
  int h = 0;
  cudaMemcpyAsync(&h, S.d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  if (h) cudaMemsetAsync(S.d_err, 0, sizeof(int), st);
  return h ? 1 : 0;
}
int sg_cells_setup(int ns, long long N, double tol) {
  using namespace sg;
  if (!S.trained || S.ns != ns) return -5;
  return cells_setup(N, tol);
}
long long sg_cells_rejected(long long* reasons) {
  using namespace sg;
  int h[8] = {};
  if (CS.count) cudaMemcpy(h, CS.count, sizeof(h), cudaMemcpyDeviceToHost);
  if (reasons)
    for (int b = 0; b < 6; b++) reasons[b] = h[2 + b];
  return h[0];
}
}  // namespace ocfd

// ---------------------------------------------------------------- C ABI
namespace {
using namespace ocfd;
using namespace ocfd::sg;

constexpr long long NPARAM = (long long)HID * PAD + HID + 2LL * ((long long)HID * HID + HID) + (long long)PAD * HID + PAD;
constexpr long long NBLOB = NPARAM + (long long)sizeof(Norm) / 4 + 2LL * PAD * PAD;

float* norm_field(int which) {  // device address of one of the Norm arrays
  char* b = reinterpret_cast<char*>(S.d_norm);
  const size_t off[6] = {offsetof(Norm, in_mean), offsetof(Norm, in_std), offsetof(Norm, out_mean),
                         offsetof(Norm, out_std), offsetof(Norm, in_min), offsetof(Norm, in_max)};
  return reinterpret_cast<float*>(b + off[which]);
}
int finish(int rc) {
  if (rc) return rc;
  if (cudaDeviceSynchronize() != cudaSuccess) return -2;
  int herr = 0;
  cudaMemcpy(&herr, S.d_err, sizeof(int), cudaMemcpyDeviceToHost);
  return herr ? -6 : 0;
}
template <class T>
T* dalloc(size_t n, std::vector<void*>& keep) {
  void* p = nullptr;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
  keep.push_back(p);
  return static_cast<T*>(p);
}
struct Freer {
  std::vector<void*> v;
  ~Freer() {
    for (void* p : v) cudaFree(p);
  }
};

// raw inputs, normalised BF16 inputs and T0 of n reactors (chunk of a larger batch)
int features(int n, const double* di, const double* e, const double* dt, float* raw, double* T0, __nv_bfloat16* xb,
             int* nf, cudaStream_t st) {
  SG_DISPATCH(S.ns, launch_raw_inputs<NSC>(n, di, e, dt, raw, T0, nf, st));
  k_normalize<<<nb((long long)n * PAD, 256), 256, 0, st>>>(n, S.nin, raw, norm_field(0), norm_field(1), xb, nullptr);
  return 0;
}

// predict (mode 0: outputs only) or apply with the gate (mode 1) over all reactors, in chunks
int run_surrogate(int n, int mode, double* di, double* e, const double* dt, const int* nsub, double tol, double* dio,
                  double* eo, double* Tp, double* Te, int* n_fallback) {
  if (!S.trained) return -5;
  cudaStream_t st = current_stream();
  // scratch kept between calls (grown when a larger batch arrives), so no call allocates twice
  static const int CH = 1 << 18;
  static float* raw = nullptr;
  static double* T0 = nullptr;
  static __nv_bfloat16 *xb = nullptr, *hA = nullptr, *hB = nullptr;
  static float* out = nullptr;
  static int* fb = nullptr;
  static int* cnt = nullptr;  // [0] fallback count, [1] nfail, [32..] work-queue counter + nfail
  static int fb_cap = 0;
  if (!raw) {
    if (cudaMalloc(&raw, (size_t)CH * PAD * 4) || cudaMalloc(&T0, (size_t)CH * 8) ||
        cudaMalloc(&xb, (size_t)CH * PAD * 2) || cudaMalloc(&hA, (size_t)CH * HID * 2) ||
        cudaMalloc(&hB, (size_t)CH * HID * 2) || cudaMalloc(&out, (size_t)CH * PAD * 4) || cudaMalloc(&cnt, 256))
      return -2;
  }
  if (n > fb_cap) {
    if (fb) cudaFree(fb);
    if (cudaMalloc(&fb, (size_t)n * 4)) { fb = nullptr; fb_cap = 0; return -2; }
    fb_cap = n;
  }
  cudaMemsetAsync(cnt, 0, 64 * sizeof(int), st);
  cudaMemsetAsync(S.d_err, 0, sizeof(int), st);
  Gemm gemm;
  __nv_bfloat16* hs[3] = {hA, hB, hA};
  for (int c0 = 0; c0 < n; c0 += CH) {
    const int rows = std::min(CH, n - c0);
    double* dic = di + (size_t)c0 * S.ns;
    double* ec = e + c0;
    int rc = features(rows, dic, ec, dt + c0, raw, T0, xb, cnt + 1, st);
    if (rc) return rc;
    forward(gemm, rows, xb, hs, nullptr, out, st);
    if (gemm.rc) return gemm.rc;
    SG_DISPATCH(S.ns, launch_post<NSC>(rows, mode, dic, ec, T0, raw, out, tol,
                                        dio ? dio + (size_t)c0 * S.ns : nullptr, eo ? eo + c0 : nullptr,
                                        Tp ? Tp + c0 : nullptr, Te ? Te + c0 : nullptr, fb, cnt, c0, cnt + 1, st));
  }
  int nfb = 0;
  if (mode == 1) {
    cudaMemcpyAsync(&nfb, cnt, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -2;
    if (nfb > 0) {
      int dev = 0, sms = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      launch_chem_batch(S.ns, sms, nfb, di, e, dt, nsub, fb, cnt + 32, cnt + 33, st);
    }
  }
  if (n_fallback) *n_fallback = nfb;
  return finish(cudaGetLastError() == cudaSuccess ? 0 : -2);
}
}  // namespace

extern "C" {
int ocfd_gpu_surrogate_fused(int on) {
  const int was = g_fused ? 1 : 0;
  if (on >= 0) g_fused = on != 0;
  return was;
}

int ocfd_gpu_surrogate_init(unsigned seed) {
  const int ns = current_nspec();
  if (ns < 2) return -5;
  return ensure_params(ns, seed);
}

int ocfd_gpu_surrogate_train(int n, const double* d_di0, const double* d_e0, const double* d_dt, const double* d_di1,
                             const double* d_e1, const double* proj, int epochs, int batch, double lr, unsigned seed,
                             double* loss_history) {
  const int ns = current_nspec();
  if (ns < 2) return -5;
  if (n <= 0 || batch <= 0 || batch % 128 != 0 || n < batch || epochs <= 0 || !proj) return -1;
  cudaStream_t st = current_stream();
  int rc = ensure_params(ns, seed);
  if (rc) return rc;
  {
    std::vector<double> P((size_t)PAD * PAD, 0.0);
    for (int i = 0; i < ns; i++)
      for (int j = 0; j < ns; j++) P[(size_t)i * ns + j] = proj[(size_t)i * ns + j];
    cudaMemcpy(S.d_proj, P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice);
  }
  Freer fr;
  float* raw_in = dalloc<float>((size_t)n * PAD, fr.v);
  float* raw_out = dalloc<float>((size_t)n * PAD, fr.v);
  double* T0 = dalloc<double>(n, fr.v);
  __nv_bfloat16* X = dalloc<__nv_bfloat16>((size_t)n * PAD, fr.v);
  float* Tt = dalloc<float>((size_t)n * PAD, fr.v);
  __nv_bfloat16* Xs = dalloc<__nv_bfloat16>((size_t)n * PAD, fr.v);
  float* Ts = dalloc<float>((size_t)n * PAD, fr.v);
  int* perm = dalloc<int>(n, fr.v);
  int* nf = dalloc<int>(1, fr.v);
  const int B = batch;
  float* pre[3];
  __nv_bfloat16* h[3];
  for (int l = 0; l < 3; l++) {
    pre[l] = dalloc<float>((size_t)B * HID, fr.v);
    h[l] = dalloc<__nv_bfloat16>((size_t)B * HID, fr.v);
  }
  float* out = dalloc<float>((size_t)B * PAD, fr.v);
  float* gf = dalloc<float>((size_t)B * PAD, fr.v);
  __nv_bfloat16* gbf = dalloc<__nv_bfloat16>((size_t)B * PAD, fr.v);
  float* dzf = dalloc<float>((size_t)B * HID, fr.v);
  __nv_bfloat16* dzb[2] = {dalloc<__nv_bfloat16>((size_t)B * HID, fr.v), dalloc<__nv_bfloat16>((size_t)B * HID, fr.v)};
  float *gW[NLAYER], *gB[NLAYER];
  for (int l = 0; l < NLAYER; l++) {
    gW[l] = dalloc<float>(wsize(l), fr.v);
    gB[l] = dalloc<float>(S.rows[l], fr.v);
  }
  double* dloss = dalloc<double>(1, fr.v);
  if (!raw_in || !raw_out || !T0 || !X || !Tt || !Xs || !Ts || !perm || !nf || !out || !gf || !gbf || !dzf ||
      !dzb[0] || !dzb[1] || !dloss || !gW[3] || !gB[3] || !pre[2] || !h[2])
    return -2;
  cudaMemsetAsync(nf, 0, sizeof(int), st);
  cudaMemsetAsync(S.d_err, 0, sizeof(int), st);
  SG_DISPATCH(ns, launch_raw_inputs<NSC>(n, d_di0, d_e0, d_dt, raw_in, T0, nf, st));
  SG_DISPATCH(ns, launch_raw_targets<NSC>(n, d_di0, d_di1, d_e1, T0, raw_out, nf, st));
  double mean[PAD], sd[PAD], mn[PAD], mx[PAD];
  if ((rc = column_stats(n, raw_in, mean, sd, mn, mx, 1.0, st))) return rc;
  for (int c = 0; c < PAD; c++) {
    // a mass fraction's scale is at least Y_STD_FLOOR: differences far below it (trace species
    // near zero in every training state) do not become O(1) inputs
    if (c >= 2 && c < 2 + ns && sd[c] < Y_STD_FLOOR) sd[c] = Y_STD_FLOOR;
    S.norm.in_mean[c] = (float)mean[c];
    S.norm.in_std[c] = (float)sd[c];
    S.norm.in_min[c] = (float)mn[c];
    S.norm.in_max[c] = (float)mx[c];
  }
  // outputs whose spread is below the FP64 rounding noise of the state (std < 1e-15, e.g. an inert
  // species) are inactive: trained against 0 and applied as their mean (stored scale 0)
  if ((rc = column_stats(n, raw_out, mean, sd, mn, mx, 0.0, st))) return rc;
  float out_train_std[PAD];
  for (int c = 0; c < PAD; c++) {
    const bool active = sd[c] > 1e-15;
    S.norm.out_mean[c] = (float)mean[c];
    S.norm.out_std[c] = active ? (float)sd[c] : 0.0f;
    out_train_std[c] = active ? (float)sd[c] : 1.0f;
  }
  float* d_tstd = dalloc<float>(PAD, fr.v);
  if (!d_tstd) return -2;
  cudaMemcpyAsync(d_tstd, out_train_std, sizeof(out_train_std), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(S.d_norm, &S.norm, sizeof(Norm), cudaMemcpyHostToDevice, st);
  k_normalize<<<nb((long long)n * PAD, 256), 256, 0, st>>>(n, S.nin, raw_in, norm_field(0), norm_field(1), X, nullptr);
  k_normalize<<<nb((long long)n * PAD, 256), 256, 0, st>>>(n, S.nout, raw_out, norm_field(2), d_tstd, nullptr, Tt);

  Gemm gemm;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const int nbatch = n / B;
  std::vector<int> hp(n);
  for (int i = 0; i < n; i++) hp[i] = i;
  for (int ep = 0; ep < epochs; ep++) {
    std::mt19937_64 rng(seed * 1000003ULL + ep);
    std::shuffle(hp.begin(), hp.end(), rng);
    cudaMemcpyAsync(perm, hp.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st);
    k_gather_rows<<<nb((long long)n * PAD, 256), 256, 0, st>>>(n, perm, X, Tt, Xs, Ts);
    cudaMemsetAsync(dloss, 0, sizeof(double), st);
    const float lr_ep = (float)(lr * 0.5 * (1.0 + std::cos(M_PI * ep / epochs)));  // cosine decay
    for (int bi = 0; bi < nbatch; bi++) {
      const __nv_bfloat16* x = Xs + (size_t)bi * B * PAD;
      const float* t = Ts + (size_t)bi * B * PAD;
      forward(gemm, B, x, h, pre, out, st);
      k_loss_grad<<<nb((long long)B * PAD, 256), 256, 0, st>>>(B, S.nout, out, t, gf, gbf, dloss);
      // output layer
      gemm(gbf, 1, PAD, h[2], 1, HID, PAD, HID, B, gW[3], HID, nullptr, 0, nullptr, nullptr, 0, 0, st);
      k_colsum<<<PAD, 256, 0, st>>>(B, PAD, gf, gB[3]);
      gemm(gbf, PAD, 1, S.wb[3], 1, HID, B, HID, PAD, dzf, HID, dzb[0], HID, pre[2], nullptr, 0, 2, st);
      int cur = 0;
      for (int l = 2; l >= 0; l--) {
        const __nv_bfloat16* hin = l > 0 ? h[l - 1] : x;
        const int Kin = S.cols[l];
        gemm(dzb[cur], 1, HID, hin, 1, Kin, HID, Kin, B, gW[l], Kin, nullptr, 0, nullptr, nullptr, 0, 0, st);
        k_colsum<<<HID, 256, 0, st>>>(B, HID, dzf, gB[l]);
        if (l > 0) {
          gemm(dzb[cur], HID, 1, S.wb[l], 1, Kin, B, Kin, HID, dzf, HID, dzb[1 - cur], HID, pre[l - 1], nullptr, 0, 2,
               st);
          cur = 1 - cur;
        }
      }
      S.adam_t++;
      const float c1 = 1.0f - std::pow(b1, (float)S.adam_t), c2 = 1.0f - std::pow(b2, (float)S.adam_t);
      for (int l = 0; l < NLAYER; l++) {
        k_adam<<<nb(wsize(l), 256), 256, 0, st>>>((long long)wsize(l), S.w[l], gW[l], S.mw[l], S.vw[l], S.wb[l], lr_ep,
                                                 b1, b2, eps, c1, c2);
        k_adam<<<nb(S.rows[l], 256), 256, 0, st>>>(S.rows[l], S.b[l], gB[l], S.mb[l], S.vb[l], nullptr, lr_ep, b1, b2,
                                                  eps, c1, c2);
      }
      if (gemm.rc) return gemm.rc;
    }
    double lh = 0.0;
    cudaMemcpyAsync(&lh, dloss, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -2;
    if (loss_history) loss_history[ep] = lh / nbatch;
  }
  S.trained = true;
  return finish(0);
}

// ungated predictions: the state each reactor would get (di_out, e_out), the network's temperature
// T0 + dT_pred and the temperature of the conserved energy (T_energy)
int ocfd_gpu_surrogate_predict(int n, const double* d_di, const double* d_e, const double* d_dt, double* d_di_out,
                               double* d_e_out, double* d_T_pred, double* d_T_energy) {
  if (n <= 0) return 0;
  return run_surrogate(n, 0, const_cast<double*>(d_di), const_cast<double*>(d_e), d_dt, nullptr, 0.0, d_di_out,
                       d_e_out, d_T_pred, d_T_energy, nullptr);
}

// gated surrogate chemistry: reactors that pass the gate are advanced by the network, the others by
// the FP64 implicit integrator (its sub-step counts in d_nsub); n_fallback gets their number
int ocfd_gpu_chem_batch_surrogate(int n, double* d_di, double* d_e, const double* d_dt, const int* d_nsub,
                                  double tol_T, int* n_fallback) {
  if (n <= 0) return 0;
  if (current_const_p()) return -7;  // the network replaces the constant-volume integrator only
  return run_surrogate(n, 1, d_di, d_e, d_dt, d_nsub, tol_T, nullptr, nullptr, nullptr, nullptr, n_fallback);
}

// temperature of n reactors from their densities and energy (comput_T), on device pointers
int ocfd_gpu_chem_temperature(int n, const double* d_di, const double* d_e, double* d_T) {
  const int ns = current_nspec();
  if (ns < 2) return -5;
  if (n <= 0) return 0;
  cudaStream_t st = current_stream();
  int* nf = nullptr;
  if (cudaMalloc(&nf, sizeof(int)) != cudaSuccess) return -2;
  cudaMemsetAsync(nf, 0, sizeof(int), st);
  SG_DISPATCH(ns, launch_temperature<NSC>(n, d_di, d_e, d_T, nf, st));
  const int rc = cudaStreamSynchronize(st) == cudaSuccess ? 0 : -2;
  cudaFree(nf);
  return rc;
}

// parameter blob: weights and biases (layer order, row-major), the normalisation record and the
// element projection; host == NULL returns the number of floats
long long ocfd_gpu_surrogate_blob(float* host, long long nfloats, int set) {
  if (!host) return NBLOB;
  if (nfloats < NBLOB || !S.w[0]) return -1;
  float* p = host;
  for (int l = 0; l < NLAYER; l++) {
    const size_t nw = wsize(l);
    if (set) {
      cudaMemcpy(S.w[l], p, nw * 4, cudaMemcpyHostToDevice);
      k_to_bf16<<<nb(nw, 256), 256>>>((long long)nw, S.w[l], S.wb[l]);
    } else {
      cudaMemcpy(p, S.w[l], nw * 4, cudaMemcpyDeviceToHost);
    }
    p += nw;
    if (set) cudaMemcpy(S.b[l], p, S.rows[l] * 4, cudaMemcpyHostToDevice);
    else cudaMemcpy(p, S.b[l], S.rows[l] * 4, cudaMemcpyDeviceToHost);
    p += S.rows[l];
  }
  if (set) {
    std::memcpy(&S.norm, p, sizeof(Norm));
    cudaMemcpy(S.d_norm, &S.norm, sizeof(Norm), cudaMemcpyHostToDevice);
  } else {
    std::memcpy(p, &S.norm, sizeof(Norm));
  }
  p += sizeof(Norm) / 4;
  if (set) {
    cudaMemcpy(S.d_proj, p, sizeof(double) * PAD * PAD, cudaMemcpyHostToDevice);
    S.trained = true;
  } else {
    cudaMemcpy(p, S.d_proj, sizeof(double) * PAD * PAD, cudaMemcpyDeviceToHost);
  }
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}

// one forward + backward pass on a host batch of normalised inputs x (B x 16) and targets t
// (B x 16), without an update: the loss and the gradients (blob layout of the weights and biases)
int ocfd_gpu_surrogate_grad(int B, const float* x, const float* t, float* grads, double* loss) {
  if (!S.w[0] || B <= 0 || B % 128 != 0) return -1;
  cudaStream_t st = current_stream();
  Freer fr;
  std::vector<__nv_bfloat16> xh((size_t)B * PAD);
  for (size_t i = 0; i < xh.size(); i++) xh[i] = __float2bfloat16(x[i]);
  __nv_bfloat16* xd = dalloc<__nv_bfloat16>((size_t)B * PAD, fr.v);
  float* td = dalloc<float>((size_t)B * PAD, fr.v);
  float* pre[3];
  __nv_bfloat16* h[3];
  for (int l = 0; l < 3; l++) {
    pre[l] = dalloc<float>((size_t)B * HID, fr.v);
    h[l] = dalloc<__nv_bfloat16>((size_t)B * HID, fr.v);
  }
  float* out = dalloc<float>((size_t)B * PAD, fr.v);
  float* gf = dalloc<float>((size_t)B * PAD, fr.v);
  __nv_bfloat16* gbf = dalloc<__nv_bfloat16>((size_t)B * PAD, fr.v);
  float* dzf = dalloc<float>((size_t)B * HID, fr.v);
  __nv_bfloat16* dzb[2] = {dalloc<__nv_bfloat16>((size_t)B * HID, fr.v), dalloc<__nv_bfloat16>((size_t)B * HID, fr.v)};
  float *gW[NLAYER], *gB[NLAYER];
  for (int l = 0; l < NLAYER; l++) {
    gW[l] = dalloc<float>(wsize(l), fr.v);
    gB[l] = dalloc<float>(S.rows[l], fr.v);
  }
  double* dloss = dalloc<double>(1, fr.v);
  if (!xd || !td || !out || !gf || !gbf || !dzf || !dzb[1] || !dloss || !gB[3]) return -2;
  cudaMemcpyAsync(xd, xh.data(), xh.size() * 2, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(td, t, sizeof(float) * B * PAD, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(dloss, 0, sizeof(double), st);
  cudaMemsetAsync(S.d_err, 0, sizeof(int), st);
  Gemm gemm;
  forward(gemm, B, xd, h, pre, out, st);
  k_loss_grad<<<nb((long long)B * PAD, 256), 256, 0, st>>>(B, S.nout, out, td, gf, gbf, dloss);
  gemm(gbf, 1, PAD, h[2], 1, HID, PAD, HID, B, gW[3], HID, nullptr, 0, nullptr, nullptr, 0, 0, st);
  k_colsum<<<PAD, 256, 0, st>>>(B, PAD, gf, gB[3]);
  gemm(gbf, PAD, 1, S.wb[3], 1, HID, B, HID, PAD, dzf, HID, dzb[0], HID, pre[2], nullptr, 0, 2, st);
  int cur = 0;
  for (int l = 2; l >= 0; l--) {
    const __nv_bfloat16* hin = l > 0 ? h[l - 1] : xd;
    const int Kin = S.cols[l];
    gemm(dzb[cur], 1, HID, hin, 1, Kin, HID, Kin, B, gW[l], Kin, nullptr, 0, nullptr, nullptr, 0, 0, st);
    k_colsum<<<HID, 256, 0, st>>>(B, HID, dzf, gB[l]);
    if (l > 0) {
      gemm(dzb[cur], HID, 1, S.wb[l], 1, Kin, B, Kin, HID, dzf, HID, dzb[1 - cur], HID, pre[l - 1], nullptr, 0, 2, st);
      cur = 1 - cur;
    }
  }
  if (gemm.rc) return gemm.rc;
  float* p = grads;
  for (int l = 0; l < NLAYER; l++) {
    cudaMemcpyAsync(p, gW[l], wsize(l) * 4, cudaMemcpyDeviceToHost, st);
    p += wsize(l);
    cudaMemcpyAsync(p, gB[l], S.rows[l] * 4, cudaMemcpyDeviceToHost, st);
    p += S.rows[l];
  }
  cudaMemcpyAsync(loss, dloss, sizeof(double), cudaMemcpyDeviceToHost, st);
  return finish(0);
}
}
