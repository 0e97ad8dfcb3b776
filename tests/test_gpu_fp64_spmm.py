"""FP64 SpMM on the int8 tensor cores (omm_gpu_spmm_f64: Y = A [H, S], the FP64 CG step's
[HG; SG] = D [H, S]) against extended-precision products.

Rows of A and columns of H, S are rounded to 53 bits relative to their largest entry and
multiplied exactly, so each element is within 2^-52 (max_k |a_ik| sum_k |h_kj| +
sum_k |a_ik| max_k |h_kj|) of the 80-bit long-double product; against the FP64 DMMA SpMM the
two agree within 1e-13 of |A| |H|."""
import ctypes as ct

import numpy as np
import pytest

import ommgpu as G
from ommgpu import synth

pytestmark = pytest.mark.gpu

TOL = 2.0 ** -52
OMM_ERR_UNSUPPORTED = -6


FORMS = [3, 2, 1, 0]
FORM_IDS = ["sm_pairs", "two_groups_per_cta", "three_pairs_per_stage", "one_pair_per_stage"]


@pytest.fixture(params=FORMS, ids=FORM_IDS, autouse=True)
def spmm_form(request):
    """Every case runs in each form of the int8 SpMM kernel (omm_gpu_set_oz_spmm_form)."""
    L = G.lib()
    assert L.omm_gpu_set_oz_spmm_form(request.param) == 0
    yield request.param
    assert L.omm_gpu_set_oz_spmm_form(1) == 0


def _fn():
    L = G.lib()
    f = L.omm_gpu_spmm_f64
    f.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    L.omm_gpu_last_error.restype = ct.c_char_p
    return f, L


def _run(A, H, S):
    import torch

    f, L = _fn()
    n, m = A.shape
    At = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()  # column-major n x m
    Hg = G.Matrix.from_csc(H)
    Sg = G.Matrix.from_csc(S) if S is not None else None
    rows = 2 * n if S is not None else n
    Y = torch.full((m, rows), float("nan"), device="cuda", dtype=torch.float64)
    rc = f(At.data_ptr(), n, n, Hg.h, Sg.h if Sg else None, Y.data_ptr(), rows)
    msg = L.omm_gpu_last_error().decode()
    return rc, msg, Y.t().cpu().numpy()


def _bound(A, B):
    la, lb = A.astype(np.longdouble), B.astype(np.longdouble)
    ref = la @ lb
    aa, ab = np.abs(A), np.abs(B)
    mag = aa.max(axis=1)[:, None] * ab.sum(axis=0)[None, :] + aa.sum(axis=1)[:, None] * ab.max(axis=0)[None, :]
    return ref, mag


def _check(A, H, S):
    rc, msg, Y = _run(A, H, S)
    assert rc == 0, msg
    n = A.shape[0]
    for k, B in enumerate([H] + ([S] if S is not None else [])):
        ref, mag = _bound(A, B.to_dense())
        err = np.abs(Y[k * n:(k + 1) * n] - ref.astype(np.float64))
        assert np.all(err <= TOL * mag + 1e-300), (k, float(np.max(err / (mag + 1e-300))))
    return Y


@pytest.mark.parametrize("n", [256, 300, 1024])
def test_pair_against_long_double(n):
    p = synth.lattice((5, 5, 5), seed=301, compute_mu=False)  # 24 x 24 atom blocks, H and S one pattern
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, p.m)) * np.exp(rng.uniform(-4, 4, (n, p.m)))
    _check(A, p.H, p.S)


def test_single_matrix_and_narrow_atoms():
    p = synth.lattice((5, 5, 6), seed=302, norb=8, nocc=1, compute_mu=False)  # 8-orbital atoms
    rng = np.random.default_rng(4)
    A = rng.standard_normal((128, p.m))
    _check(A, p.H, None)
    _check(A, p.H, p.S)


def test_agrees_with_fp64_dmma_spmm():
    """The int8 product and the FP64 DMMA one (psp_gemspm) on the same operands."""
    p = synth.lattice((6, 5, 5), seed=303, compute_mu=False)
    rng = np.random.default_rng(5)
    A = rng.standard_normal((512, p.m))
    Y = _check(A, p.H, p.S)
    Ag, Hg, Sg = G.Matrix.from_numpy(A), G.Matrix.from_csc(p.H), G.Matrix.from_csc(p.S)
    for k, Bg in enumerate((Hg, Sg)):
        C = G.Matrix.allocate(512, p.m)
        G.psp_gemspm(512, p.m, p.m, Ag, "n", Bg, "n", C, 1.0, 0.0)
        mag = np.abs(A) @ np.abs((p.H if k == 0 else p.S).to_dense())
        assert np.max(np.abs(Y[k * 512:(k + 1) * 512] - C.numpy()) / (mag + 1e-300)) <= 1e-13


def test_same_pattern_new_values():
    """A matrix registered afresh with the pattern of an earlier one (as an SCF caller registers H
    every cycle) reuses that pattern's plan structure, but its products use its own values."""
    p = synth.lattice((5, 5, 5), seed=307, compute_mu=False)
    rng = np.random.default_rng(8)
    A = rng.standard_normal((256, p.m))
    _check(A, p.H, p.S)
    H2 = synth.CSCMatrix(p.H.dim1, p.H.dim2, p.H.colptr, p.H.rowind, p.H.val * rng.uniform(0.5, 2.0, p.H.val.shape))
    S2 = synth.CSCMatrix(p.S.dim1, p.S.dim2, p.S.colptr, p.S.rowind, -p.S.val)
    _check(A, H2, S2)
    _check(A, p.H, p.S)


def test_zero_and_nonfinite_rows():
    p = synth.lattice((5, 5, 5), seed=304, compute_mu=False)
    rng = np.random.default_rng(6)
    A = rng.standard_normal((128, p.m))
    A[3, :] = 0.0
    A[9, 17] = np.nan
    rc, msg, Y = _run(A, p.H, p.S)
    assert rc == 0, msg
    assert np.all(Y[3] == 0.0) and np.all(Y[128 + 3] == 0.0)
    assert np.all(np.isnan(Y[9])) and np.all(np.isnan(Y[128 + 9]))


def test_forms_give_the_same_bits(spmm_form):
    """The kernel's forms (one group per CTA with one or three chunk pairs per stage, two groups per
    CTA over their joint union, the same on SM pairs) form every product exactly, so their results
    are bit-identical,
    on a pattern whose unions hold runs of adjacent chunks, odd chunk counts and an odd number of
    groups (the last CTA of the two-group form holds one)."""
    p = synth.lattice((5, 5, 5), seed=306, compute_mu=False)
    rng = np.random.default_rng(7)
    A = rng.standard_normal((512, p.m)) * np.exp(rng.uniform(-3, 3, (512, p.m)))
    L = G.lib()
    rc, msg, Y1 = _run(A, p.H, p.S)
    assert rc == 0, msg
    for other in FORMS:
        if other == spmm_form:
            continue
        assert L.omm_gpu_set_oz_spmm_form(other) == 0
        rc, msg, Y2 = _run(A, p.H, p.S)
        assert rc == 0, msg
        assert np.array_equal(Y1, Y2), other
    assert L.omm_gpu_set_oz_spmm_form(4) == -1  # OMM_ERR_ARG


def test_rejects_rows_not_multiple_of_four():
    p = synth.lattice((5, 5, 5), seed=305, compute_mu=False)
    A = np.ones((130, p.m))
    rc, msg, _ = _run(A, p.H, p.S)
    assert rc == OMM_ERR_UNSUPPORTED, (rc, msg)
    assert G.tc_errors() == 0
