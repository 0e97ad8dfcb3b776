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
