"""The timed-out-wait path of the tcgen05 kernels, exercised without faulting or hanging the GPU.

Every mbarrier wait of the tensor-core GEMM and SpMM gives up after a limit (2 s by
default), sets an error bit, stops issuing, lets issued copies land and frees its TMEM.
Here the limit is cut to 5 ms and the copy producers are told to issue nothing
(omm_gpu_tc_set_wait), so the MMA warp's first wait on every CTA runs out while no copy
is in flight.  The call must return OMM_ERR_CUDA naming the error bits, and the next
normal call must succeed with the same result as before (TMEM was released and the
context is intact)."""
import ctypes as ct
import re

import numpy as np
import pytest

import ommgpu as G
from ommgpu import synth

pytestmark = pytest.mark.gpu

OMM_ERR_CUDA = -2
SHORT_NS = 5_000_000  # 5 ms
DEFAULT_NS = 2_000_000_000


def _lib():
    L = G.lib()
    L.omm_gpu_tc_set_wait.argtypes = [ct.c_ulonglong, ct.c_int]
    L.omm_gpu_tc_set_wait.restype = ct.c_int
    L.omm_gpu_last_error.restype = ct.c_char_p
    f = L.omm_gpu_gemm_bf16
    f.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int,
                  ct.c_int, ct.c_double, ct.c_double, ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    return L, f


def _bits(msg: str) -> int:
    m = re.search(r"error bits (\d+)", msg)
    assert m, msg
    return int(m.group(1))


def test_set_wait_rejects_zero():
    L, _ = _lib()
    assert L.omm_gpu_tc_set_wait(0, 0) == -1


@pytest.mark.parametrize("pairs", [1, 0], ids=["sm_pairs", "one_sm"])
def test_gemm_wait_times_out_and_recovers(pairs):
    """The bf16 GEMM on SM pairs and on single SMs with its copies withheld."""
    L, _ = _lib()
    assert L.omm_gpu_tc_set_pairs(pairs) == 0
    try:
        _bf16_wait_case()
    finally:
        assert L.omm_gpu_tc_set_pairs(1) == 0


def _bf16_wait_case():
    import torch

    L, f = _lib()
    M, N, K = 256, 512, 128  # 2 x 2 CTAs
    g = torch.Generator(device="cuda").manual_seed(1)
    A = torch.randn(M, K, generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn(N, K, generator=g, device="cuda").to(torch.bfloat16)
    out = torch.zeros(N, M, device="cuda", dtype=torch.float64)

    def call():
        return f(M, N, K, A.data_ptr(), None, K, B.data_ptr(), None, K, 1, 1.0, 0.0, out.data_ptr(), M)

    assert call() == 0
    torch.cuda.synchronize()
    good = out.clone()
    ref = A.double() @ B.double().t()
    assert float((good.t() - ref).abs().max()) <= 1e-4 * float(ref.abs().max())
    out.fill_(0.0)
    try:
        assert L.omm_gpu_tc_set_wait(SHORT_NS, 1) == 0
        rc = call()
        msg = L.omm_gpu_last_error().decode()
    finally:
        assert L.omm_gpu_tc_set_wait(DEFAULT_NS, 0) == 0
    assert rc == OMM_ERR_CUDA, (rc, msg)
    bits = _bits(msg)
    assert bits & 4, bits          # the MMA warp's operand wait ran out
    assert not bits & 2, bits      # no copy was in flight to drain
    assert float(out.abs().max()) == 0.0  # no tile was written
    # the library and the context are intact: the same product again, bit for bit
    assert call() == 0
    torch.cuda.synchronize()
    assert G.tc_errors() == 0
    assert torch.equal(out, good)


def test_spmm_wait_times_out_and_recovers():
    L, _ = _lib()
    p = synth.lattice((5, 5, 5), seed=201, compute_mu=False)  # 24 x 24 atom blocks: the tensor-core path
    rng = np.random.default_rng(9)
    A = np.asfortranarray(rng.standard_normal((256, p.m)))
    Ag, Bg = G.Matrix.from_numpy(A), G.Matrix.from_csc(p.H)
    Cg = G.Matrix.allocate(256, p.m)
    path = ct.c_int(-1)
    assert L.omm_gpu_spmm_lowp(Ag.h, Bg.h, Cg.h, None, None, 1, ct.byref(path)) == 0
    assert path.value == 2
    good = Cg.numpy()
    try:
        assert L.omm_gpu_tc_set_wait(SHORT_NS, 1) == 0
        rc = L.omm_gpu_spmm_lowp(Ag.h, Bg.h, Cg.h, None, None, 1, ct.byref(path))
        msg = L.omm_gpu_last_error().decode()
    finally:
        assert L.omm_gpu_tc_set_wait(DEFAULT_NS, 0) == 0
    assert rc == OMM_ERR_CUDA, (rc, msg)
    bits = _bits(msg)
    assert bits & 64, bits         # the MMA warp's stage wait ran out
    assert not bits & 32, bits     # nothing to drain
    assert L.omm_gpu_spmm_lowp(Ag.h, Bg.h, Cg.h, None, None, 1, ct.byref(path)) == 0
    assert G.tc_errors() == 0
    assert np.array_equal(Cg.numpy(), good)


@pytest.mark.parametrize("pairs", [1, 0], ids=["sm_pairs", "one_sm"])
def test_fp64_int8_gemm_wait_times_out_and_recovers(pairs):
    """The persistent int8 GEMM of the FP64 products, on SM pairs and on single SMs: with its copies withheld the MMA warp's slab wait and the epilogue's accumulator
    wait run out (bits 1024, 2048), nothing is left to drain (512 clear), TMEM is released, and
    the next product is correct again."""
    import torch

    L, _ = _lib()
    assert L.omm_gpu_tc_set_pairs(pairs) == 0
    try:
        _fp64_wait_case(L, torch)
    finally:
        assert L.omm_gpu_tc_set_pairs(1) == 0


def _fp64_wait_case(L, torch):
    f = L.omm_gpu_gemm_f64
    f.argtypes = [ct.c_char, ct.c_char, ct.c_int, ct.c_int, ct.c_int, ct.c_double, ct.c_void_p, ct.c_int,
                  ct.c_void_p, ct.c_int, ct.c_double, ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    M, N, K = 256, 512, 300
    g = torch.Generator(device="cuda").manual_seed(2)
    A = torch.randn(K, M, generator=g, device="cuda", dtype=torch.float64)  # column-major M x K
    B = torch.randn(N, K, generator=g, device="cuda", dtype=torch.float64)  # column-major K x N
    out = torch.zeros(N, M, device="cuda", dtype=torch.float64)

    def call():
        return f(b"n", b"n", M, N, K, 1.0, A.data_ptr(), M, B.data_ptr(), K, 0.0, out.data_ptr(), M)

    assert call() == 0
    torch.cuda.synchronize()
    good = out.clone()
    ref = A.t() @ B.t()
    assert float((good.t() - ref).abs().max()) <= 1e-12 * float(ref.abs().max())
    try:
        assert L.omm_gpu_tc_set_wait(SHORT_NS, 1) == 0
        rc = call()
        msg = L.omm_gpu_last_error().decode()
    finally:
        assert L.omm_gpu_tc_set_wait(DEFAULT_NS, 0) == 0
    assert rc == OMM_ERR_CUDA, (rc, msg)
    bits = _bits(msg)
    assert bits & 1024 and bits & 2048, bits
    assert not bits & 512, bits
    assert call() == 0
    torch.cuda.synchronize()
    assert G.tc_errors() == 0
    assert torch.equal(out, good)


@pytest.mark.parametrize("form", [3, 2, 1, 0],
                         ids=["sm_pairs", "two_groups_per_cta", "three_pairs_per_stage", "one_pair_per_stage"])
def test_fp64_int8_spmm_wait_times_out_and_recovers(form):
    """The int8 SpMM of the FP64 CG step with its copies withheld, in each form of the kernel:
    the MMA warp's chunk wait and the epilogue's accumulator wait run out (bits 131072, 262144),
    nothing is left to drain (32768 clear), TMEM is released, and the next product is correct."""
    L, _ = _lib()
    assert L.omm_gpu_set_oz_spmm_form(form) == 0
    try:
        _fp64_spmm_wait_case(L)
    finally:
        assert L.omm_gpu_set_oz_spmm_form(1) == 0


def _fp64_spmm_wait_case(L):
    import torch

    f = L.omm_gpu_spmm_f64
    f.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    p = synth.lattice((5, 5, 5), seed=211, compute_mu=False)
    n = 256
    g = torch.Generator(device="cuda").manual_seed(4)
    A = torch.randn(p.m, n, generator=g, device="cuda", dtype=torch.float64)  # column-major n x m
    Hg, Sg = G.Matrix.from_csc(p.H), G.Matrix.from_csc(p.S)
    Y = torch.zeros(p.m, 2 * n, device="cuda", dtype=torch.float64)

    def call():
        return f(A.data_ptr(), n, n, Hg.h, Sg.h, Y.data_ptr(), 2 * n)

    assert call() == 0
    good = Y.clone()
    try:
        assert L.omm_gpu_tc_set_wait(SHORT_NS, 1) == 0
        rc = call()
        msg = L.omm_gpu_last_error().decode()
    finally:
        assert L.omm_gpu_tc_set_wait(DEFAULT_NS, 0) == 0
    assert rc == OMM_ERR_CUDA, (rc, msg)
    bits = _bits(msg)
    assert bits & 131072 and bits & 262144, bits
    assert not bits & 32768, bits
    assert call() == 0
    assert G.tc_errors() == 0
    assert torch.equal(Y, good)
