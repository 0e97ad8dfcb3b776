"""Reduced-precision SpMM of the mixed solver (omm_gpu_spmm_lowp) against the FP64 product.

Bars (relative to the |A| |B| magnitude of each output element): bf16 operands with FP32
accumulation 2^-7; the hi/lo split 2^-14.  The block-sparse lattice matrices must take the
tcgen05 path; a pattern without 8-row blocks takes the FP32 path."""
import numpy as np
import pytest

import ommgpu as G
from ommgpu import synth

pytestmark = pytest.mark.gpu


def _check(A, Bc, nseg, expect_path=None):
    Ag = G.Matrix.from_numpy(A)
    Bg = G.Matrix.from_csc(Bc)
    Cg = G.Matrix.allocate(A.shape[0], Bc.dim2)
    path = G.spmm_lowp(Ag, Bg, Cg, nseg)
    got = Cg.numpy()
    Bd = Bc.to_dense()
    ref = A @ Bd
    mag = np.abs(A) @ np.abs(Bd) + 1e-300
    err = float(np.max(np.abs(got - ref) / mag))
    if expect_path is not None:
        assert path == expect_path, path
    return err, path


@pytest.mark.parametrize("n", [256, 300, 1536])
@pytest.mark.parametrize("nseg", [1, 3])
def test_lattice_blocks_tensor_core(n, nseg):
    p = synth.lattice((5, 5, 5), seed=201, compute_mu=False)  # 24 x 24 atom blocks
    rng = np.random.default_rng(n)
    A = np.asfortranarray(rng.standard_normal((n, p.m)))
    err, path = _check(A, p.H, nseg, expect_path=2)
    assert err <= (2.0 ** -7 if nseg == 1 else 2.0 ** -14), err


def test_lattice_norb8():
    p = synth.lattice((5, 5, 6), seed=202, norb=8, nocc=1, compute_mu=False)
    rng = np.random.default_rng(3)
    A = np.asfortranarray(rng.standard_normal((200, p.m)))
    err, path = _check(A, p.S, 3)
    assert path == 2 and err <= 2.0 ** -14, (err, path)


def test_unblocked_pattern_fp32_path():
    import scipy.sparse as sp

    rng = np.random.default_rng(4)
    B = sp.random(900, 900, density=0.05, random_state=np.random.RandomState(5), format="csc")
    B = B + sp.eye(900)
    Bc = synth.CSCMatrix.from_scipy(sp.csc_matrix(B))
    A = np.asfortranarray(rng.standard_normal((100, 900)))
    err, path = _check(A, Bc, 1)
    assert path in (0, 1)
    assert err <= 1e-6 if path == 1 else err <= 1e-12


def test_plan_follows_matrix_changes():
    """The tensor-core form of B (bf16 blocks built once per matrix) is rebuilt after m_scale,
    after m_set_element on a stored entry, and after an insertion that changes the pattern."""
    p = synth.lattice((5, 5, 5), seed=203, compute_mu=False)
    rng = np.random.default_rng(7)
    A = np.asfortranarray(rng.standard_normal((256, p.m)))
    Ag = G.Matrix.from_numpy(A)
    Bg = G.Matrix.from_csc(p.H)
    Cg = G.Matrix.allocate(256, p.m)
    Bd = p.H.to_dense()

    def check(expect_tc):
        path = G.spmm_lowp(Ag, Bg, Cg, 3)
        ref = A @ Bd
        mag = np.abs(A) @ np.abs(Bd) + 1e-300
        err = float(np.max(np.abs(Cg.numpy() - ref) / mag))
        assert (path == 2) == expect_tc, path
        assert err <= 2.0 ** -14, err

    check(True)
    G.m_scale(Bg, 2.0)
    Bd = 2.0 * Bd
    check(True)
    j = 5
    i = int(p.H.rowind[p.H.colptr[j]])  # first stored entry of column j (0-based)
    G.m_set_element(Bg, i + 1, j + 1, 7.5, 0.0)
    Bd[i, j] = 7.5
    check(True)
    # an entry outside the 24 x 24 atom blocks breaks the 8-row runs of its column group
    far = (i + p.m // 2) % p.m
    assert Bd[far, j] == 0.0
    G.m_set_element(Bg, far + 1, j + 1, 3.25, 0.0)
    Bd[far, j] = 3.25
    check(False)


def test_fused_pair_and_prepare_apply():
    """[A H, A S] in one pass (the solver's form) equals two single products, and the
    prepare/apply halves reproduce the synchronous call."""
    p = synth.lattice((5, 5, 5), seed=204, compute_mu=False)
    rng = np.random.default_rng(9)
    n = 300
    A = np.asfortranarray(rng.standard_normal((n, p.m)))
    Ag = G.Matrix.from_numpy(A)
    Hg, Sg = G.Matrix.from_csc(p.H), G.Matrix.from_csc(p.S)
    for nseg in (1, 3):
        C1, C2 = G.Matrix.allocate(n, p.m), G.Matrix.allocate(n, p.m)
        assert G.spmm_lowp(Ag, Hg, C1, nseg, B2=Sg, C2=C2) == 2
        D1, D2 = G.Matrix.allocate(n, p.m), G.Matrix.allocate(n, p.m)
        G.spmm_lowp(Ag, Hg, D1, nseg)
        G.spmm_lowp(Ag, Sg, D2, nseg)
        assert np.array_equal(C1.numpy(), D1.numpy())
        assert np.array_equal(C2.numpy(), D2.numpy())
        E1, E2 = G.Matrix.allocate(n, p.m), G.Matrix.allocate(n, p.m)
        G.spmm_lowp_prepare(Ag, nseg)
        G.spmm_lowp_apply(Hg, E1, nseg, B2=Sg, C2=E2)
        assert G.tc_errors() == 0
        assert np.array_equal(E1.numpy(), C1.numpy())
        assert np.array_equal(E2.numpy(), C2.numpy())
        ref = A @ p.S.to_dense()
        mag = np.abs(A) @ np.abs(p.S.to_dense()) + 1e-300
        assert float(np.max(np.abs(E2.numpy() - ref) / mag)) <= (2.0 ** -7 if nseg == 1 else 2.0 ** -14)


def test_apply_rejects_unprepared_shape():
    p = synth.lattice((5, 5, 5), seed=205, compute_mu=False)
    A = G.Matrix.from_numpy(np.asfortranarray(np.ones((64, p.m))))
    G.spmm_lowp_prepare(A, 1)
    Hg = G.Matrix.from_csc(p.H)
    C = G.Matrix.allocate(65, p.m)
    with pytest.raises(G.OmmError):
        G.spmm_lowp_apply(Hg, C, 1)
    with pytest.raises(G.OmmError):
        G.spmm_lowp_apply(Hg, G.Matrix.allocate(64, p.m), 3)
