"""tcgen05 BF16 GEMM (omm_gpu_gemm_bf16) against a torch reference on the same bf16 values.

The reference multiplies the bf16 operands in FP64 (exact products); the kernel
accumulates in FP32 in TMEM, so the bar is 2e-6 of sum_k |a_ik b_jk| (K up to 2^14
FP32 additions), and 1e-5 relative for the 3-segment split product against FP64 inputs."""
import ctypes as ct

import numpy as np
import pytest

import ommgpu as G

pytestmark = pytest.mark.gpu


def _fn():
    L = G.lib()
    f = L.omm_gpu_gemm_bf16
    f.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int,
                  ct.c_int, ct.c_double, ct.c_double, ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    return f, L


def _run(M, N, K, nseg=1, alpha=1.0, beta=0.0, seed=0):
    import torch

    f, L = _fn()
    g = torch.Generator(device="cuda").manual_seed(seed)
    lda = (K + 7) // 8 * 8
    A64 = torch.randn(M, K, generator=g, device="cuda", dtype=torch.float64)
    B64 = torch.randn(N, K, generator=g, device="cuda", dtype=torch.float64)
    Ah = torch.zeros(M, lda, device="cuda", dtype=torch.bfloat16)
    Bh = torch.zeros(N, lda, device="cuda", dtype=torch.bfloat16)
    Ah[:, :K] = A64.to(torch.bfloat16)
    Bh[:, :K] = B64.to(torch.bfloat16)
    Al = torch.zeros_like(Ah)
    Bl = torch.zeros_like(Bh)
    Al[:, :K] = (A64 - Ah[:, :K].double()).to(torch.bfloat16)
    Bl[:, :K] = (B64 - Bh[:, :K].double()).to(torch.bfloat16)
    out0 = torch.randn(N, M, generator=g, device="cuda", dtype=torch.float64)  # column-major M x N storage
    out = out0.clone()
    torch.cuda.synchronize()
    rc = f(M, N, K, Ah.data_ptr(), Al.data_ptr(), lda, Bh.data_ptr(), Bl.data_ptr(), lda, nseg, alpha, beta,
           out.data_ptr(), M)
    assert rc == 0, L.omm_gpu_last_error().decode()
    torch.cuda.synchronize()
    got = out.t()  # M x N
    ah, bh = Ah[:, :K].double(), Bh[:, :K].double()
    if nseg == 1:
        ref = alpha * (ah @ bh.t()) + beta * out0.t()
        scale = alpha * (ah.abs() @ bh.abs().t())
        err = ((got - ref).abs() / (scale + 1e-30)).max().item()
        return err
    al_, bl_ = Al[:, :K].double(), Bl[:, :K].double()
    ref_split = alpha * (ah @ bh.t() + ah @ bl_.t() + al_ @ bh.t()) + beta * out0.t()
    ref_exact = alpha * (A64 @ B64.t()) + beta * out0.t()
    scale = alpha * (A64.abs() @ B64.abs().t())
    e_split = ((got - ref_split).abs() / scale).max().item()
    e_exact = ((got - ref_exact).abs() / scale).max().item()
    return e_split, e_exact


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (256, 512, 1024), (300, 500, 1000), (129, 257, 72),
                                   (3072, 1536, 4096), (64, 64, 8), (1536, 4096, 3072)])
def test_gemm_bf16(M, N, K):
    err = _run(M, N, K)
    assert err <= 2e-6, err


def test_gemm_bf16_alpha_beta():
    err = _run(200, 300, 256, alpha=-2.0, beta=0.5)
    assert err <= 2e-6, err


@pytest.mark.parametrize("M,N,K", [(256, 256, 512), (300, 700, 2000)])
def test_gemm_bf16x3_split(M, N, K):
    e_split, e_exact = _run(M, N, K, nseg=3)
    assert e_split <= 2e-6, e_split
    assert e_exact <= 1e-5, e_exact


def test_gemm_bf16_rejects_misaligned_ld():
    f, L = _fn()
    out = np.zeros(4)
    rc = f(2, 2, 5, 16, 0, 5, 16, 0, 5, 1, 1.0, 0.0, out.ctypes.data, 2)
    assert rc == -1


@pytest.mark.parametrize("pairs", [0, 1], ids=["one_sm", "sm_pairs"])
@pytest.mark.parametrize("M,N,K,nseg", [(300, 500, 1000, 1), (3072, 1536, 4096, 1), (257, 300, 520, 3)])
def test_gemm_bf16_tilings(pairs, M, N, K, nseg):
    """Both tilings -- 128 x 256 tiles on single SMs and 256 x 256 tiles on SM pairs
    (omm_gpu_tc_set_pairs) -- meet the same bars."""
    _, L = _fn()
    assert L.omm_gpu_tc_set_pairs(pairs) == 0
    try:
        r = _run(M, N, K, nseg=nseg, seed=M + nseg)
    finally:
        assert L.omm_gpu_tc_set_pairs(1) == 0
    if nseg == 1:
        assert r <= 2e-6, r
    else:
        assert r[0] <= 2e-6 and r[1] <= 1e-5, r
