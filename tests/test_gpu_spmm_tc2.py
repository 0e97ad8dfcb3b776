"""The mixed solver's per-step SpMM (omm_gpu_spmm_lowp_apply_f32) in both its forms -- one column
group per CTA, and CTAs of four column groups -- : Y = A [H, S] in FP32 and its row-major bf16
shadows, against the FP64 products.

Bars as for the other reduced-precision SpMM (relative to |A| |B| of each element): bf16
operands with FP32 accumulation 2^-7, hi/lo split 2^-14.  The shadows must be exactly the
bf16 hi part of the returned FP32 values and the bf16 rounding of their remainder."""
import ctypes as ct

import numpy as np
import pytest

import ommgpu as G
from ommgpu import synth

pytestmark = pytest.mark.gpu


def _fn():
    L = G.lib()
    f = L.omm_gpu_spmm_lowp_apply_f32
    f.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_int]
    f.restype = ct.c_int
    L.omm_gpu_last_error.restype = ct.c_char_p
    return f, L


@pytest.fixture(params=[1, 4], ids=["one_group_per_cta", "four_groups_per_cta"], autouse=True)
def groups(request):
    L = G.lib()
    assert L.omm_gpu_set_spmm_groups(request.param) == 0
    yield request.param
    assert L.omm_gpu_set_spmm_groups(1) == 0


def _run(A, H, S, nseg, shadows=True):
    import torch

    f, L = _fn()
    n, m = A.shape
    Ag = G.Matrix.from_numpy(A)
    Hg = G.Matrix.from_csc(H)
    Sg = G.Matrix.from_csc(S) if S is not None else None
    G.spmm_lowp_prepare(Ag, nseg)
    rows = 2 * n if S is not None else n
    Y = torch.full((m, rows), float("nan"), device="cuda", dtype=torch.float32)  # column-major rows x m
    ldt = (m + 7) // 8 * 8
    th = torch.zeros(rows, ldt, device="cuda", dtype=torch.bfloat16) if shadows else None
    tl = torch.zeros(rows, ldt, device="cuda", dtype=torch.bfloat16) if (shadows and nseg == 3) else None
    rc = f(Hg.h, Sg.h if Sg else None, Y.data_ptr(), rows, th.data_ptr() if shadows else None,
           tl.data_ptr() if tl is not None else None, ldt, nseg)
    assert rc == 0, L.omm_gpu_last_error().decode()
    torch.cuda.synchronize()
    assert G.tc_errors() == 0
    return Y.t().cpu().numpy().astype(np.float64), Y, th, tl


def _check(A, H, S, nseg):
    import torch

    Yn, Y, th, tl = _run(A, H, S, nseg)
    n = A.shape[0]
    tol = 2.0 ** -7 if nseg == 1 else 2.0 ** -14
    for k, B in enumerate([H] + ([S] if S is not None else [])):
        Bd = B.to_dense()
        ref = A @ Bd
        mag = np.abs(A) @ np.abs(Bd) + 1e-300
        err = float(np.max(np.abs(Yn[k * n:(k + 1) * n] - ref) / mag))
        assert err <= tol, (k, err)
    # shadows: the hi part of the FP32 result and the rounding of the remainder
    yt = Y.t()  # rows x m, row-major view of the column-major result
    m = A.shape[1]
    hi = yt.to(torch.bfloat16)
    assert torch.equal(th[:, :m], hi)
    if tl is not None:
        assert torch.equal(tl[:, :m], (yt - hi.float()).to(torch.bfloat16))


@pytest.mark.parametrize("nseg", [1, 3])
@pytest.mark.parametrize("n", [256, 300, 1536])
def test_pair_blocks_of_groups(nseg, n):
    p = synth.lattice((5, 5, 5), seed=201, compute_mu=False)  # 24 x 24 atom blocks, H and S one pattern
    rng = np.random.default_rng(n + nseg)
    A = np.asfortranarray(rng.standard_normal((n, p.m)))
    _check(A, p.H, p.S, nseg)


def test_single_matrix_and_narrow_groups():
    p = synth.lattice((5, 5, 6), seed=202, norb=8, nocc=1, compute_mu=False)  # 8-orbital atoms
    rng = np.random.default_rng(3)
    A = np.asfortranarray(rng.standard_normal((200, p.m)))
    _check(A, p.S, None, 3)
    _check(A, p.H, p.S, 1)


def test_agrees_with_per_group_kernel():
    """The FP32 forms against the per-group kernel with FP64 output (spmm_tc.cu) on the same
    bf16 operands: all accumulate exact bf16 products in FP32, at most the order differs."""
    p = synth.lattice((6, 5, 5), seed=7, compute_mu=False)
    rng = np.random.default_rng(11)
    A = np.asfortranarray(rng.standard_normal((512, p.m)))
    Yn, _, _, _ = _run(A, p.H, p.S, 1, shadows=False)
    Ag, Hg, Sg = G.Matrix.from_numpy(A), G.Matrix.from_csc(p.H), G.Matrix.from_csc(p.S)
    C1, C2 = G.Matrix.allocate(512, p.m), G.Matrix.allocate(512, p.m)
    assert G.spmm_lowp(Ag, Hg, C1, 1, B2=Sg, C2=C2) == 2
    old = np.vstack([C1.numpy(), C2.numpy()])
    mag = np.vstack([np.abs(A) @ np.abs(p.H.to_dense()), np.abs(A) @ np.abs(p.S.to_dense())]) + 1e-300
    assert float(np.max(np.abs(Yn - old) / mag)) <= 2.0 ** -16  # FP32 summation order only
