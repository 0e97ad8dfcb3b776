"""GPU test of omm_gpu_mm_trace_noalloc, the mm_trace that allocates nothing.

That entry point exists for callers that cannot let the library allocate
device memory (an application whose own memory manager owns the GPU, loops
that cannot take cudaMalloc's synchronisation).  Its result must equal the
allocating entry point msw_mm_[dz]trace on the same data, call after call,
since every call reuses one fixed scratch array; the complex and the largest
cases are also checked against the oracle's mm_trace / numpy on the host.

This file is named so that pytest collects it after every other test file; it
passes alone in a fresh process as well as after the others.
"""
import ctypes as ct

import numpy as np
import pytest

import ommgpu as G

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the tolerance of the FP64 parity tests


def _entry():
    L = G.lib()
    f = L.omm_gpu_mm_trace_noalloc
    f.argtypes = [ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p,
                  ct.c_void_p]
    f.restype = ct.c_int
    L.omm_gpu_noalloc_last_error.restype = ct.c_char_p
    return f, L


def _rnd(rng, shape, cplx):
    a = rng.standard_normal(shape)
    if cplx:
        a = a + 1j * rng.standard_normal(shape)
    return np.asfortranarray(a)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("shape", [(1536, 1536), (777, 3001), (1, 1)])
def test_noalloc_trace_equals_mm_trace_twice(cplx, shape):
    import torch

    f, L = _entry()
    rng = np.random.default_rng(2024 + shape[0])
    A, B = _rnd(rng, shape, cplx), _rnd(rng, shape, cplx)
    Ag, Bg = G.Matrix.from_numpy(A), G.Matrix.from_numpy(B)
    ref = G.mm_trace(Ag, Bg)  # allocating entry point
    scale = max(1.0, float(np.sum(np.abs(A) * np.abs(B))))
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(2):  # two calls in a row share the scratch array
        rc = f(shape[0], shape[1], Ag.device_ptr(), shape[0], Bg.device_ptr(), shape[0], int(cplx), out.data_ptr(),
               stream.cuda_stream)
        assert rc == 0, L.omm_gpu_noalloc_last_error().decode()
        torch.cuda.synchronize()
        got = complex(out[0].item(), out[1].item())
        assert abs(got - complex(ref)) <= RTOL * scale, (got, ref)


def test_noalloc_trace_leading_dimension():
    """A sub-block of a larger matrix (lda > rows), checked against numpy."""
    import torch

    f, L = _entry()
    rng = np.random.default_rng(7)
    big_a, big_b = _rnd(rng, (500, 300), False), _rnd(rng, (500, 300), False)
    Ag, Bg = G.Matrix.from_numpy(big_a), G.Matrix.from_numpy(big_b)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    rc = f(123, 300, Ag.device_ptr(), 500, Bg.device_ptr(), 500, 0, out.data_ptr(), None)
    assert rc == 0, L.omm_gpu_noalloc_last_error().decode()
    torch.cuda.synchronize()
    ref = float(np.sum(big_a[:123] * big_b[:123]))
    assert abs(out[0].item() - ref) <= RTOL * float(np.sum(np.abs(big_a[:123] * big_b[:123])))


def test_noalloc_trace_complex_against_oracle():
    """Complex input, checked against the oracle's mm_trace (Re sum conj(A) B) and numpy's vdot."""
    import torch

    import oracle as O

    f, L = _entry()
    rng = np.random.default_rng(11)
    A, B = _rnd(rng, (641, 257), True), _rnd(rng, (641, 257), True)
    Ag, Bg = G.Matrix.from_numpy(A), G.Matrix.from_numpy(B)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    scale = float(np.sum(np.abs(A) * np.abs(B)))
    for _ in range(2):
        rc = f(641, 257, Ag.device_ptr(), 641, Bg.device_ptr(), 641, 1, out.data_ptr(), None)
        assert rc == 0, L.omm_gpu_noalloc_last_error().decode()
        torch.cuda.synchronize()
        assert abs(out[0].item() - O.mm_trace(A, B)) <= RTOL * scale
        assert abs(out[1].item() - np.vdot(A, B).imag) <= RTOL * scale


def test_noalloc_trace_empty_writes_zero():
    """rows > 0, cols = 0: only the final kernel runs, and it must write {0, 0} over stale values."""
    import torch

    f, L = _entry()
    Ag = G.Matrix.from_numpy(np.ones((8, 8)))
    out = torch.full((2,), 7.0, dtype=torch.float64, device="cuda")
    # fill the scratch array with a non-trivial call first, so stale records exist
    rc = f(8, 8, Ag.device_ptr(), 8, Ag.device_ptr(), 8, 0, out.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert out[0].item() == 64.0
    out.fill_(7.0)
    rc = f(8, 0, Ag.device_ptr(), 8, Ag.device_ptr(), 8, 0, out.data_ptr(), None)
    assert rc == 0, L.omm_gpu_noalloc_last_error().decode()
    torch.cuda.synchronize()
    assert out[0].item() == 0.0 and out[1].item() == 0.0


def test_noalloc_trace_at_the_limit():
    """Exactly OMM_NOALLOC_MAX_ELEMS elements (every record of the array in use), real, against
    msw_mm_dtrace and against a float64 sum on the host."""
    import torch

    f, L = _entry()
    rows, cols = 8192, 16384  # 2^27 elements = OMM_NOALLOC_MAX_ELEMS, 1 GiB per operand
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.rand(cols, rows, generator=g, device="cuda", dtype=torch.float64) * 1e-3
    B = torch.rand(cols, rows, generator=g, device="cuda", dtype=torch.float64) * 1e-3
    Ag = G.Matrix.register_gden(A.data_ptr(), rows, cols, False, keep=A)
    Bg = G.Matrix.register_gden(B.data_ptr(), rows, cols, False, keep=B)
    ref = G.mm_trace(Ag, Bg)  # allocating entry point
    host = float(np.sum(A.cpu().numpy() * B.cpu().numpy()))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for _ in range(2):
        rc = f(rows, cols, A.data_ptr(), rows, B.data_ptr(), rows, 0, out.data_ptr(), None)
        assert rc == 0, L.omm_gpu_noalloc_last_error().decode()
        torch.cuda.synchronize()
        assert abs(out[0].item() - ref) <= RTOL * abs(ref)
        assert abs(out[0].item() - host) <= RTOL * abs(host)
    del Ag, Bg, A, B
    torch.cuda.empty_cache()


def test_noalloc_trace_rejects_oversize():
    import torch

    f, L = _entry()
    Ag = G.Matrix.from_numpy(np.ones((4, 4)))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    # 20000 x 20000 elements exceed OMM_NOALLOC_MAX_ELEMS: rejected before anything is launched
    rc = f(20000, 20000, Ag.device_ptr(), 20000, Ag.device_ptr(), 20000, 0, out.data_ptr(), None)
    assert rc == -1  # OMM_ERR_ARG
    assert "exceeds" in L.omm_gpu_noalloc_last_error().decode()
