// Dense-layer GEMM of the chemistry surrogate (tcgen05, ocfd_mlp.cu), shared with the surrogate's
// training and inference code (ocfd_surrogate.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace ocfd {
namespace mlp {

struct GemmArgs {
  const __nv_bfloat16* A;
  long long sam, sak;  // A(m, k) = A[m * sam + k * sak]
  const __nv_bfloat16* B;
  long long sbn, sbk;  // B(n, k) = B[n * sbn + k * sbk]
  float* C;            // C(m, n) = C[m * ldc + n], FP32 (may be null when only Cb is wanted)
  long long ldc;
  __nv_bfloat16* Cb;  // optional BF16 copy of the epilogue output
  long long ldcb;
  float* pre;  // act 1: FP32 copy before the activation is written here; act 2: read from here
  const float* bias;
  int M, N, K;
  int beta;  // 1: C = C + A . B^T
  int act;   // 0: none, 1: GELU, 2: multiply by GELU'(pre) (backward through the activation)
  int* err;  // set to 1 when an mbarrier wait runs out
};

// launches k_gemm_bf16 on stream st; 0 or -2 (CUDA error)
int launch_gemm(const GemmArgs& g, cudaStream_t st);

// the whole inference pass of the surrogate's network 16 -> 256 -> 256 -> 256 -> 16 (GELU after
// the three hidden layers) in one kernel: W0 (256 x 16), W1, W2 (256 x 256), W3 (16 x 256) BF16
// row-major (row = output neuron), biases FP32, x (M x 16) BF16, out (M x 16) FP32
struct MlpArgs {
  const __nv_bfloat16* x;
  const __nv_bfloat16* w[4];
  const float* b[4];
  float* out;
  int M;
  int* err;            // set to 1 when an mbarrier wait runs out
  unsigned char* pack; // MLP_PACK_BYTES of device scratch for the weights in shared-memory image form
};
constexpr int MLP_PACK_BYTES = (2 + 2 * 16) * 8192;  // W0, 16 + 16 chunks of W1 / W2, W3
// packs the weights (launch on the same stream before the kernel), then runs the kernel
int launch_mlp_fused(const MlpArgs& a, cudaStream_t st);
// one-time kernel attribute set-up of the fused kernel (call outside stream capture)
int prepare_mlp_fused();

}  // namespace mlp
}  // namespace ocfd
