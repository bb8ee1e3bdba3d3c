"""The surrogate's tensor-core GEMM (tcgen05, BF16 operands, FP32 accumulation in TMEM) against a
float64 product of the same BF16-rounded operands. Products of two BF16 numbers are exact in FP32,
so the only differences are FP32 accumulation roundings: relative 1e-5 of the largest entry."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    from ocfd_b200 import solver
    return torch, solver.lib()


def _gemm(env, A, B, trans_a=False, trans_b=False, bias=None, beta=0, act=0, C0=None):
    torch, L = env
    M, K = A.shape
    N = B.shape[0]
    dev = torch.device("cuda")
    # store A / B transposed in memory when asked, and pass strides that undo it
    a_t = torch.from_numpy(A.T.copy() if trans_a else A.copy()).to(dev, torch.bfloat16).contiguous()
    b_t = torch.from_numpy(B.T.copy() if trans_b else B.copy()).to(dev, torch.bfloat16).contiguous()
    sam, sak = (1, M) if trans_a else (K, 1)
    sbn, sbk = (1, N) if trans_b else (K, 1)
    C = torch.zeros((M, N), dtype=torch.float32, device=dev) if C0 is None else torch.from_numpy(C0).to(dev).contiguous()
    bt = None if bias is None else torch.from_numpy(bias).to(dev, torch.float32)
    rc = L.ocfd_gpu_gemm_bf16(M, N, K, a_t.data_ptr(), sam, sak, b_t.data_ptr(), sbn, sbk, C.data_ptr(), N,
                              None if bt is None else bt.data_ptr(), beta, act)
    assert rc == 0, rc
    Ar = a_t.float().cpu().numpy().astype(np.float64)
    Br = b_t.float().cpu().numpy().astype(np.float64)
    Ar = Ar.T if trans_a else Ar
    Br = Br.T if trans_b else Br
    return C.cpu().numpy(), Ar, Br


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 150, 200), (1000, 256, 12), (77, 10, 256)])
@pytest.mark.parametrize("trans", [(False, False), (True, False), (False, True)])
def test_gemm_matches_float64(env, M, N, K, trans):
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    C, Ar, Br = _gemm(env, A, B, *trans)
    ref = Ar @ Br.T
    assert np.abs(C - ref).max() <= 1e-5 * np.abs(ref).max()


def test_gemm_epilogue_bias_beta_gelu(env):
    from math import pi, sqrt
    rng = np.random.default_rng(7)
    M, N, K = 260, 200, 96
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    bias = rng.standard_normal(N).astype(np.float32)
    C0 = rng.standard_normal((M, N)).astype(np.float32)
    C, Ar, Br = _gemm(env, A, B, bias=bias, beta=1, act=1, C0=C0)
    pre = Ar @ Br.T + bias + C0
    ref = 0.5 * pre * (1.0 + np.tanh(sqrt(2.0 / pi) * pre * (1.0 + 0.044715 * pre * pre)))  # GELU, tanh form
    # the kernel evaluates tanh with the hardware approximation (absolute error about 5e-4 on tanh,
    # i.e. up to 2.5e-4 |x| on GELU); the GEMM itself agrees to 1e-5 (test above)
    assert np.abs(C - ref).max() <= 1e-3 * np.abs(ref).max()
