"""GPU test of omm_gpu_mm_trace_noalloc, the mm_trace that allocates nothing.

That entry point exists for callers that cannot let the library allocate
device memory (stream capture into a CUDA graph, an application-owned memory
manager, loops that cannot take cudaMalloc's synchronisation).  Its result
must equal the allocating entry point msw_mm_[dz]trace on the same data, call
after call, since every call reuses one fixed scratch array.

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


def test_noalloc_trace_rejects_oversize():
    import torch

    f, L = _entry()
    Ag = G.Matrix.from_numpy(np.ones((4, 4)))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    # 20000 x 20000 elements exceed OMM_NOALLOC_MAX_ELEMS: rejected before anything is launched
    rc = f(20000, 20000, Ag.device_ptr(), 20000, Ag.device_ptr(), 20000, 0, out.data_ptr(), None)
    assert rc == -1  # OMM_ERR_ARG
    assert "exceeds" in L.omm_gpu_noalloc_last_error().decode()
