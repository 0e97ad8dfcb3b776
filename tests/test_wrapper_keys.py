"""The string-key layer (MatrixSwitch_wrapper / ms_lookup, MatrixSwitch_wrapper_params.F90:47-71)
on host storage, without a GPU: key semantics of Fortran character variables (stored cut to 10
characters, trailing blanks insignificant), unknown keys, uninitialised slots, default label."""
import ctypes as ct

import numpy as np

import ommgpu as G

OMM_ERR_ARG, OMM_ERR_STATE = -1, -5


def _lib():
    L = G.lib()
    L.omm_gpu_last_error.restype = ct.c_char_p
    return L


def _open(L, keys):
    arr = (ct.c_char_p * len(keys))(*[k.encode() for k in keys])
    assert L.ms_wrapper_open(len(keys), arr) == 0


def test_keys_follow_fortran_character_semantics():
    L = _lib()
    _open(L, ["H", "S", "dens_matrix_long"])
    h = ct.c_void_p(1)
    assert L.ms_lookup(b"H", ct.byref(h)) == 0 and h.value is None      # slot exists, no matrix yet
    assert L.ms_lookup(b"H   ", ct.byref(h)) == 0                        # trailing blanks do not count
    assert L.ms_lookup(b"dens_matri", ct.byref(h)) == 0                  # the key was stored cut to 10
    assert L.ms_lookup(b"dens_matrix_long", ct.byref(h)) == OMM_ERR_ARG  # longer than any stored key
    assert L.ms_lookup(b"T", ct.byref(h)) == OMM_ERR_ARG
    assert b"key not found" in L.omm_gpu_last_error()
    ini = ct.c_bool(True)
    assert L.ms_is_initialized(b"S", ct.byref(ini)) == 0 and not ini.value
    assert L.ms_wrapper_close() == 0
    assert L.ms_lookup(b"H", ct.byref(h)) == OMM_ERR_STATE


def test_allocate_default_label_and_queries():
    L = _lib()
    _open(L, ["C", "X"])
    assert L.ms_m_allocate(b"C", 3, 5, None) == 0  # no label: sdden (MatrixSwitch.F90:344-347)
    h = ct.c_void_p()
    assert L.ms_lookup(b"C", ct.byref(h)) == 0 and h.value
    d1, d2, cplx, csc = ct.c_int(), ct.c_int(), ct.c_int(), ct.c_int()
    assert L.msw_dims(h, ct.byref(d1), ct.byref(d2), ct.byref(cplx), ct.byref(csc)) == 0
    assert (d1.value, d2.value, cplx.value, csc.value) == (3, 5, 0, 0)
    b = ct.c_bool()
    for fn, want in ((L.ms_is_initialized, True), (L.ms_is_serial, True), (L.ms_is_real, True),
                     (L.ms_is_square, False), (L.ms_is_sparse, False)):
        assert fn(b"C", ct.byref(b)) == 0 and b.value == want
    n = ct.c_int()
    assert L.ms_dim1(b"C", ct.byref(n)) == 0 and n.value == 3
    assert L.ms_dim2(b"C", ct.byref(n)) == 0 and n.value == 5
    assert L.ms_is_real(b"X", ct.byref(b)) == OMM_ERR_ARG  # uninitialised slot
    a = np.asfortranarray(np.arange(6.0).reshape(2, 3))
    assert L.ms_m_register_sdden(b"X", 2, 3, a.ctypes.data_as(ct.POINTER(ct.c_double))) == 0
    assert L.ms_lookup(b"X", ct.byref(h)) == 0
    out = np.zeros((2, 3), order="F")
    assert L.msw_download(h, out.ctypes.data_as(ct.c_void_p)) == 0  # aliases the caller's array
    assert np.array_equal(out, a)
    assert L.ms_m_deallocate(b"C") == 0
    assert L.ms_is_initialized(b"C", ct.byref(b)) == 0 and not b.value
    assert L.ms_wrapper_close() == 0


def test_omm_wrapper_resolves_keys_first():
    """omm_wrapper looks its keys up before anything runs (ms_lookup dies on an unknown key);
    an allocated-key check follows for H, D_min and C_min (S and T may be uninitialised)."""
    L = _lib()
    f = L.omm_wrapper
    f.argtypes = [ct.c_int, ct.c_int, ct.c_char_p, ct.c_char_p, ct.c_bool, ct.POINTER(ct.c_double), ct.c_char_p,
                  ct.c_bool, ct.c_double, ct.c_char_p, ct.c_bool, ct.c_char_p, ct.c_double, ct.c_int, ct.c_int,
                  ct.c_int, ct.c_double, ct.c_bool, ct.c_bool, ct.c_char_p, ct.c_char_p]
    _open(L, ["H", "S", "D", "C", "T"])
    try:
        e = ct.c_double()
        rc = f(4, 2, b"Q", b"S", True, ct.byref(e), b"D", False, 0.0, b"C", False, b"T", 0.0, 0, 1, 1, -1.0, False,
               True, b"sdden", b"ref")
        assert rc == OMM_ERR_ARG and b"key not found" in L.omm_gpu_last_error()
        rc = f(4, 2, b"H", b"S", True, ct.byref(e), b"D", False, 0.0, b"C", False, b"T", 0.0, 0, 1, 1, -1.0, False,
               True, b"sdden", b"ref")
        assert rc == OMM_ERR_ARG and b"not allocated" in L.omm_gpu_last_error()
    finally:
        assert L.ms_wrapper_close() == 0
