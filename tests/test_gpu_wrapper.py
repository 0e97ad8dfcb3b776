"""libOMM's omm_wrapper (libOMM/src/omm_wrapper.F90:5-96, CBIND logicals) driven through the
MatrixSwitch wrapper's string keys, on the reference's complex two-k-point example
(libOMM/examples/example_kpoints.F90): the sequence of that example -- H and S registered by
key (m_register_szden), D and C allocated by key, two SCF steps per k-point (np = 2), then the
energy-weighted density -- against the example's asserted values and the oracle."""
import ctypes as ct

import numpy as np
import pytest

import oracle as O
import ommgpu as G
from tests.golden.examples import golden, kpoints_HS

pytestmark = pytest.mark.gpu


def _lib():
    L = G.lib()
    L.omm_gpu_last_error.restype = ct.c_char_p
    f = L.omm_wrapper
    f.argtypes = [ct.c_int, ct.c_int, ct.c_char_p, ct.c_char_p, ct.c_bool, ct.POINTER(ct.c_double), ct.c_char_p,
                  ct.c_bool, ct.c_double, ct.c_char_p, ct.c_bool, ct.c_char_p, ct.c_double, ct.c_int, ct.c_int,
                  ct.c_int, ct.c_double, ct.c_bool, ct.c_bool, ct.c_char_p, ct.c_char_p]
    f.restype = ct.c_int
    return L


@pytest.mark.parametrize("flavour", [0, 1])
def test_kpoints_example_through_keys(flavour):
    L = _lib()
    g = golden()["kpoints"]
    tol = g["tolerance"]
    keys = [b"H1", b"S1", b"H2", b"S2", b"D1", b"D2", b"C1", b"C2", b"ED1", b"ED2", b"T"]
    assert L.ms_wrapper_open(len(keys), (ct.c_char_p * len(keys))(*keys)) == 0
    keep = {}
    try:
        orc = O.OmmOracle()
        Ho, So, Co, Do = {}, {}, {}, {}
        for k in (1, 2):
            m, n, h, s = kpoints_HS(k, 1)
            keep["H%d" % k], keep["S%d" % k] = h, s
            assert L.ms_m_register_szden(b"H%d" % k, m, m, h.ctypes.data_as(ct.c_void_p)) == 0
            assert L.ms_m_register_szden(b"S%d" % k, m, m, s.ctypes.data_as(ct.c_void_p)) == 0
            assert L.ms_m_allocate(b"D%d" % k, m, m, b"szden") == 0
            assert L.ms_m_allocate(b"C%d" % k, n, m, b"szden") == 0
            Ho[k], So[k] = h.copy(order="F"), s.copy(order="F")
            Co[k] = np.zeros((n, m), complex, order="F")
            Do[k] = np.zeros((m, m), complex, order="F")
        e = ct.c_double()
        el = (ct.c_double * 2)()
        for i in (1, 2):
            for k in (1, 2):
                if i == 2:
                    h2 = kpoints_HS(k, 2)[2]
                    keep["H%d" % k] = h2
                    assert L.ms_m_register_szden(b"H%d" % k, m, m, h2.ctypes.data_as(ct.c_void_p)) == 0
                    Ho[k] = h2.copy(order="F")
                rc = L.omm_wrapper(m, n, b"H%d" % k, b"S%d" % k, i == 1, ct.byref(e), b"D%d" % k, False, 0.0,
                                   b"C%d" % k, i == 2, b"T", 0.0, flavour, 2, k, -1.0, False, False, b"szden", b"lap")
                assert rc == 0, L.omm_gpu_last_error()
                er, _ = orc.omm(m, n, Ho[k], So[k], i == 1, Do[k], False, 0.0, Co[k], i == 2, flavour=flavour,
                                np_=2, ip=k)
                idx = (k - 1) * 2 + (i - 1)
                assert abs(e.value - g["e_min_check"]["values"][idx]) <= tol
                assert abs(e.value - er) <= 1e-10 * abs(er)
                assert L.ms_m_zget_element(b"D%d" % k, 1, 1, el, b"lap") == 0
                assert abs(el[0] - g["D_el_check"]["values"][idx]) <= tol
        for k in (1, 2):
            assert L.ms_m_allocate(b"ED%d" % k, m, m, b"szden") == 0
            rc = L.omm_wrapper(m, n, b"H%d" % k, b"S%d" % k, False, ct.byref(e), b"ED%d" % k, True, 0.0,
                               b"C%d" % k, True, b"T", 0.0, 0, 2, k, -1.0, False, k == 2, b"szden", b"lap")
            assert rc == 0, L.omm_gpu_last_error()
            assert L.ms_m_zget_element(b"ED%d" % k, 1, 1, el, b"lap") == 0
            assert abs(el[0] - g["ED_el_check"]["values"][k - 1]) <= tol
    finally:
        assert L.ms_wrapper_close() == 0

