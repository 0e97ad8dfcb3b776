"""The C-ABI library loads without a GPU, exports every declared symbol, and
validates arguments on the host exactly where the reference's die() would fire."""
import re

import numpy as np
import pytest

import ommgpu as G


def test_exports_every_declared_symbol():
    names = G.header_functions()
    assert len(names) >= 40
    L = G.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_header_cites_reference():
    txt = open(G.HEADER).read()
    for routine in ("omm.F90", "MatrixSwitch.F90", "pspMspm.F90", "pspSpmm.F90", "MatrixSwitch_m_register.F90"):
        assert routine in txt


def test_invalid_labels_rejected():
    with pytest.raises(G.OmmError) as e:
        G.Matrix.allocate(2, 2, "xdden")
    assert e.value.code == -1
    with pytest.raises(G.OmmError) as e:
        G.Matrix.allocate(2, 2, "sdcoo")
    assert e.value.code == -6


def test_register_csc_validation():
    from ommgpu.synth import CSCMatrix

    bad = CSCMatrix(3, 3, np.array([0, 1, 1, 2], np.int32), np.array([0, 5], np.int32), np.ones(2))
    with pytest.raises(G.OmmError):
        G.Matrix.from_csc(bad, "sdcsc")
    ok = CSCMatrix(3, 3, np.array([0, 1, 1, 2], np.int32), np.array([0, 2], np.int32), np.ones(2))
    M = G.Matrix.from_csc(ok, "sdcsc", index_base=1)  # passed to the library 1-based (Fortran CSC)
    assert M.dims() == (3, 3, False, True)


def test_register_csc_large_copies_and_checks():
    """The copy and the row-index check of a large registration run on host threads: a bad
    index far from the start is still caught, and a good 1-based matrix (registered twice, the
    second time from pooled memory) exports the same 0-based arrays."""
    from ommgpu.synth import CSCMatrix

    rng = np.random.default_rng(5)
    m, per = 4096, 64
    colptr = np.arange(m + 1, dtype=np.int32) * per
    rowind = np.sort(rng.integers(0, m, size=(m, per)), axis=1).astype(np.int32).ravel()
    val = rng.standard_normal(m * per)
    bad = rowind.copy()
    bad[-5] = m  # out of range, in the last worker's share
    with pytest.raises(G.OmmError):
        G.Matrix.from_csc(CSCMatrix(m, m, colptr, bad, val), "sdcsc")
    for _ in range(2):
        M = G.Matrix.from_csc(CSCMatrix(m, m, colptr, rowind, val), "sdcsc", index_base=1)
        back = M.csc()
        assert np.array_equal(back.colptr, colptr) and np.array_equal(back.rowind, rowind)
        assert np.array_equal(back.val, val)
        del M


def test_host_matrix_elements_without_gpu():
    a = np.asfortranarray(np.arange(6.0).reshape(2, 3))
    M = G.Matrix.register_sden(a)
    assert G.m_get_element(M, 2, 3) == 5.0
    G.m_set_element(M, 1, 1, 7.0, 2.0)  # C = alpha + beta*C
    assert a[0, 0] == 7.0


def test_csc_element_insert_host():
    from ommgpu.synth import CSCMatrix

    M = G.Matrix.from_csc(CSCMatrix(3, 3, np.array([0, 1, 1, 1], np.int32), np.array([0], np.int32),
                                    np.array([2.0])), "sdcsc")
    G.m_set_element(M, 3, 2, 4.0)
    assert G.m_get_element(M, 3, 2) == 4.0
    assert G.m_get_element(M, 1, 1) == 2.0
    assert G.m_get_element(M, 2, 2) == 0.0
