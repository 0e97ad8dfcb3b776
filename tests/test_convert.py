"""Format conversions of the registration path against numpy restatements of the reference's loops.

m_copy dense -> CSC (MatrixSwitch_m_copy.F90:495-629): column-major scan, every element
without a threshold, |a| > thr with one (soft: a - thr a/|a|); dense -> dense with threshold
(:102-147) zeroes the rest; psp_den2sp (pspBasicTool.F90:205-421): a != 0 for thre = 0,
|a| >= thre otherwise; COO registration sums repeats.  Bit-exact (integer patterns, copied
or arithmetically identical values)."""
import numpy as np
import pytest
import scipy.sparse as sp

import ommgpu as G


def ref_den2csc(A, keep, shift=0.0):
    """Column-major scan like the reference loops: (colptr, rowind, val)."""
    cp, ri, val = [0], [], []
    for j in range(A.shape[1]):
        for i in range(A.shape[0]):
            a = A[i, j]
            if keep(a):
                ri.append(i)
                val.append(a - shift * a / abs(a) if shift else a)
        cp.append(len(ri))
    return np.array(cp), np.array(ri, dtype=np.int64), np.array(val, dtype=A.dtype)


def rnd(shape, cplx, seed, zeros=0.3):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    if cplx:
        a = a + 1j * rng.standard_normal(shape)
    a[rng.random(shape) < zeros] = 0.0
    return np.asfortranarray(a)


# ------------------------------------------------------------------ host-only (no GPU)
@pytest.mark.parametrize("cplx", [False, True])
def test_coo_registration_sorts_and_sums(cplx):
    rng = np.random.default_rng(5)
    m, n, k = 40, 30, 300
    r = rng.integers(0, m, k)
    c = rng.integers(0, n, k)
    v = rng.standard_normal(k) + (1j * rng.standard_normal(k) if cplx else 0)
    A = G.Matrix.from_coo(r + 1, c + 1, v, m, n, label="szcsc" if cplx else "sdcsc", index_base=1)
    got = A.csc()
    ref = sp.csc_matrix(sp.coo_matrix((v, (r, c)), shape=(m, n)))
    ref.sum_duplicates()
    ref.sort_indices()
    assert np.array_equal(got.colptr, ref.indptr)
    assert np.array_equal(got.rowind, ref.indices)
    assert np.allclose(got.val, ref.data, rtol=0, atol=1e-14)


def test_coo_registration_rejects_bad_indices():
    with pytest.raises(G.OmmError):
        G.Matrix.from_coo([0, 5], [0, 0], [1.0, 2.0], 5, 5, label="sdcsc")
    with pytest.raises(G.OmmError):
        G.Matrix.from_coo([0], [-1], [1.0], 5, 5, label="sdcsc")


# ------------------------------------------------------------------ device conversions
@pytest.mark.gpu
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("shape", [(37, 29), (700, 300)])
def test_mcopy_dense_to_csc(cplx, shape):
    A = rnd(shape, cplx, 11)
    Ag = G.Matrix.from_numpy(A)
    # no threshold: every element (zeros included)
    cp, ri, val = ref_den2csc(A, lambda a: True)
    got = Ag.copy("gzcsc" if cplx else "gdcsc").csc()
    assert np.array_equal(got.colptr, cp) and np.array_equal(got.rowind, ri) and np.array_equal(got.val, val)
    for soft in (False, True):
        thr = 0.7
        cp, ri, val = ref_den2csc(A, lambda a: abs(a) > thr, thr if soft else 0.0)
        got = Ag.copy_thre("gzcsc" if cplx else "gdcsc", -thr, soft).csc()  # |threshold| is used
        assert np.array_equal(got.colptr, cp) and np.array_equal(got.rowind, ri)
        # soft shifts cancel where |a| ~ thr: compare on the scale of A (hypot may differ by an ulp)
        tol = 4e-16 * float(np.max(np.abs(A)))
        assert np.allclose(got.val, val, rtol=0, atol=tol)
        # dense -> dense with threshold, and the CSC scattered back
        D = Ag.copy_thre("gzden" if cplx else "gdden", thr, soft).numpy()
        Dref = np.zeros_like(A)
        mask = np.abs(A) > thr
        Dref[mask] = A[mask] - (thr * A[mask] / np.abs(A[mask]) if soft else 0)
        assert np.allclose(D, Dref, rtol=0, atol=tol)
        back = G.psp_sp2den(Ag.copy_thre("gzcsc" if cplx else "gdcsc", thr, soft)).numpy()
        assert np.allclose(back, Dref, rtol=0, atol=tol)


@pytest.mark.gpu
@pytest.mark.parametrize("cplx", [False, True])
def test_psp_den2sp(cplx):
    A = rnd((513, 257), cplx, 13)
    Ag = G.Matrix.from_numpy(A)
    cp, ri, val = ref_den2csc(A, lambda a: a != 0)
    got = G.psp_den2sp(Ag, 0.0).csc()
    assert np.array_equal(got.colptr, cp) and np.array_equal(got.rowind, ri) and np.array_equal(got.val, val)
    thr = float(np.sort(np.abs(A[A != 0]))[A.size // 3])  # an existing magnitude: tests the >= edge
    cp, ri, val = ref_den2csc(A, lambda a: abs(a) >= thr)
    got = G.psp_den2sp(Ag, thr).csc()
    assert np.array_equal(got.colptr, cp) and np.array_equal(got.rowind, ri) and np.array_equal(got.val, val)
    with pytest.raises(G.OmmError):
        G.psp_den2sp(Ag, -1.0)
    # the converted matrix is a working operand: psp_gemspm against the dense product
    X = rnd((64, 513), cplx, 14, zeros=0.0)
    Xg = G.Matrix.from_numpy(X)
    out = G.Matrix.allocate(64, 257, "gzden" if cplx else "gdden")
    G.psp_gemspm(64, 257, 513, Xg, "n", G.psp_den2sp(Ag, thr), "n", out, 1.0, 0.0)
    Aref = np.where(np.abs(A) >= thr, A, 0)
    assert np.allclose(out.numpy(), X @ Aref, rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_csc_to_csc_threshold_is_rejected_like_the_reference():
    A = G.Matrix.from_numpy(rnd((20, 20), False, 15)).copy("gdcsc")
    with pytest.raises(G.OmmError) as ei:
        A.copy_thre("gdcsc", 0.1)
    assert ei.value.code == -6
