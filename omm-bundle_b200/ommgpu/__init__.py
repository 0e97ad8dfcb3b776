"""Thin Python binding of the B200 libOMM / MatrixSwitch / pspBLAS C ABI (include/ommgpu.h).

The names mirror the reference's Fortran API so that tests read like the
reference's example programs:

    H = Matrix.from_csc(csc, "gdcsc")          # m_register_pcsc
    C = Matrix.allocate(n, m, "gdden")          # m_allocate
    e, rc = omm(m, n, H, S, True, D, False, 0.0, C, False, m_operation="gpu")

Everything computes on the GPU through ``lib/libommgpu.so``; there is no CPU
fallback.  Importing works without a GPU (so the exported symbols can be
checked), but every call then fails with the CUDA error the library reports.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libommgpu.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(_HERE)), "include", "ommgpu.h")

OMM_OK = 0
OMM_NOT_CONVERGED = 1
ERRORS = {-1: "OMM_ERR_ARG", -2: "OMM_ERR_CUDA", -3: "OMM_ERR_ALLOC", -4: "OMM_ERR_NOT_SPD", -5: "OMM_ERR_STATE",
          -6: "OMM_ERR_UNSUPPORTED", -7: "OMM_ERR_NONFINITE", -8: "OMM_ERR_CALLBACK"}

_lib = None


class OmmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, msg))
        self.code = code


class omm_gpu_stats(ct.Structure):
    _fields_ = [("icg", ct.c_int), ("icg_low", ct.c_int), ("icg_fp64", ct.c_int), ("ls_fail", ct.c_int),
                ("converged", ct.c_int), ("e_min", ct.c_double), ("e_diff", ct.c_double), ("trqs", ct.c_double),
                ("seconds", ct.c_double), ("t_setup", ct.c_double), ("t_loop", ct.c_double), ("t_final", ct.c_double),
                ("t_loop_sync", ct.c_double)]


def lib():
    """Load lib/libommgpu.so (raises if it has not been built: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libommgpu.so is not built (%s); run `make -C omm-bundle_b200` or "
                           "__graft_entry__.build()" % LIB_PATH)
    L = ct.CDLL(LIB_PATH)
    P = ct.c_void_p
    I, D, CP, B = ct.c_int, ct.c_double, ct.c_char_p, ct.c_bool
    PD = ct.POINTER(ct.c_double)
    sig = {
        "omm_gpu_last_error": ([], ct.c_char_p),
        "omm_gpu_set_device": ([I], I),
        "omm_gpu_set_stream": ([P], I),
        "omm_gpu_finalize": ([], I),
        "omm_gpu_kernel_launches": ([], ct.c_longlong),
        "omm_gpu_pool_stats": ([ct.POINTER(ct.c_longlong)], ct.c_int),
        "omm_gpu_set_oz_spmm_form": ([I], I),
        "msw_allocate": ([ct.POINTER(P), I, I, CP], I),
        "msw_deallocate": ([ct.POINTER(P)], I),
        "msw_register_sden": ([ct.POINTER(P), I, I, P, I], I),
        "msw_register_gden": ([ct.POINTER(P), I, I, P, I], I),
        "msw_register_csc": ([ct.POINTER(P), CP, I, I, I, P, P, P, I], I),
        "msw_copy": ([ct.POINTER(P), P, CP], I),
        "msw_upload": ([P, P], I),
        "msw_download": ([P, P], I),
        "msw_device_ptr": ([P], P),
        "msw_dims": ([P, ct.POINTER(I), ct.POINTER(I), ct.POINTER(I), ct.POINTER(I)], I),
        "msw_mm_dmultiply": ([P, ct.c_char, P, ct.c_char, P, D, D, CP], I),
        "msw_mm_zmultiply": ([P, ct.c_char, P, ct.c_char, P, PD, PD, CP], I),
        "msw_m_dadd": ([P, ct.c_char, P, D, D, CP], I),
        "msw_m_zadd": ([P, ct.c_char, P, PD, PD, CP], I),
        "msw_m_dtrace": ([P, PD, CP], I),
        "msw_m_ztrace": ([P, PD, CP], I),
        "msw_mm_dtrace": ([P, P, PD, CP], I),
        "msw_mm_ztrace": ([P, P, PD, CP], I),
        "msw_m_dscale": ([P, D, CP], I),
        "msw_m_zscale": ([P, PD, CP], I),
        "msw_m_dset": ([P, ct.c_char, D, D, CP], I),
        "msw_m_zset": ([P, ct.c_char, PD, PD, CP], I),
        "msw_m_dset_element": ([P, I, I, D, D, CP], I),
        "msw_m_zset_element": ([P, I, I, PD, PD, CP], I),
        "msw_m_dget_element": ([P, I, I, PD, CP], I),
        "msw_m_zget_element": ([P, I, I, PD, CP], I),
        "psp_gpu_dgemspm": ([I, I, I, P, ct.c_char, P, ct.c_char, P, D, D], I),
        "psp_gpu_zgemspm": ([I, I, I, P, ct.c_char, P, ct.c_char, P, PD, PD], I),
        "psp_gpu_dgespmm": ([I, I, I, P, ct.c_char, P, ct.c_char, P, D, D], I),
        "psp_gpu_zgespmm": ([I, I, I, P, ct.c_char, P, ct.c_char, P, PD, PD], I),
        "omm_gpu": ([I, I, P, P, B, PD, P, B, D, P, B, P, D, I, I, I, D, B, B, CP, CP], I),
        "msw_copy_thre": ([ct.POINTER(P), P, CP, D, B], I),
        "msw_register_coo": ([ct.POINTER(P), CP, I, I, I, P, P, P, I], I),
        "psp_gpu_den2sp": ([P, D, CP, ct.POINTER(P)], I),
        "psp_gpu_sp2den": ([P, CP, ct.POINTER(P)], I),
        "msw_csc_arrays": ([P, ct.POINTER(I), P, P, P], I),
        "omm_gpu_callback": ([I, I, H_FN, P, P, B, PD, P, B, D, P, B, P, D, I, I, I, D, B, B, CP, CP], I),
        "omm_gpu_get_stats": ([ct.POINTER(omm_gpu_stats)], I),
        "omm_gpu_set_log": ([CP], I),
        "omm_gpu_set_mixed": ([D, D, D], I),
        "omm_gpu_functional_grad": ([I, I, P, P, P, P, PD], I),
        "omm_gpu_energy_adjoint": ([I, I, P, P, I, ct.POINTER(P), PD], I),
        "omm_gpu_spmm_lowp": ([P, P, P, P, P, I, ct.POINTER(I)], I),
        "omm_gpu_spmm_lowp_prepare": ([P, I], I),
        "omm_gpu_spmm_lowp_apply": ([P, P, P, P, I], I),
        "omm_gpu_tc_errors": ([ct.POINTER(ct.c_uint)], I),
        "omm_gpu_spmm_plan_info": ([P, ct.POINTER(I), ct.POINTER(I), PD, ct.POINTER(I)], I),
        "tomato_gpu_TB": ([CP, CP, B, PD, ct.POINTER(I), B, ct.POINTER(I), ct.POINTER(I), B, PD, PD,
                           ct.POINTER(I), B, PD, B, D, ct.POINTER(P), ct.POINTER(P), CP, B], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _check(rc: int) -> int:
    if rc < 0:
        raise OmmError(rc, lib().omm_gpu_last_error().decode())
    return rc


def _lbl(s: str, k: int) -> bytes:
    b = s.encode()
    if len(b) != k:
        raise ValueError("label %r must have %d characters" % (s, k))
    return b


def _z(v) -> ct.Array:
    v = complex(v)
    return (ct.c_double * 2)(v.real, v.imag)


# omm_callback's H routine: int H(const msw_matrix* C, msw_matrix* HC, void* user)
H_FN = ct.CFUNCTYPE(ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p)


class Matrix:
    """Handle of a MatrixSwitch-like matrix (type(matrix), MatrixSwitch_ops.F90:62-97)."""

    def __init__(self, handle: int, keep=None, owned: bool = True):
        self.h = ct.c_void_p(handle)
        self._keep = keep  # host/device memory aliased by the handle
        self._owned = owned  # False for handles the library lends (omm_callback's C and HC)

    def __del__(self):
        try:
            if self._owned and self.h and self.h.value:
                lib().msw_deallocate(ct.byref(self.h))
        except Exception:
            pass

    @property
    def _as_arg(self):
        return self.h

    # ---------------------------------------------------------- constructors
    @classmethod
    def allocate(cls, dim1: int, dim2: int, label: str = "gdden") -> "Matrix":
        h = ct.c_void_p()
        _check(lib().msw_allocate(ct.byref(h), dim1, dim2, _lbl(label, 5)))
        return cls(h.value)

    @classmethod
    def register_sden(cls, a: np.ndarray) -> "Matrix":
        """m_register_sden: alias a Fortran-ordered host array (float64 or complex128)."""
        if not a.flags.f_contiguous or a.dtype not in (np.float64, np.complex128):
            raise ValueError("m_register_sden needs a Fortran-ordered float64/complex128 array")
        h = ct.c_void_p()
        _check(lib().msw_register_sden(ct.byref(h), a.shape[0], a.shape[1], a.ctypes.data,
                                       int(a.dtype == np.complex128)))
        return cls(h.value, keep=a)

    @classmethod
    def register_gden(cls, ptr: int, dim1: int, dim2: int, is_complex: bool, keep=None) -> "Matrix":
        h = ct.c_void_p()
        _check(lib().msw_register_gden(ct.byref(h), dim1, dim2, ct.c_void_p(ptr), int(is_complex)))
        return cls(h.value, keep=keep)

    @classmethod
    def from_numpy(cls, a: np.ndarray, label: str | None = None) -> "Matrix":
        a = np.asfortranarray(a)
        cplx = np.iscomplexobj(a)
        a = a.astype(np.complex128 if cplx else np.float64, copy=False)
        label = label or ("gzden" if cplx else "gdden")
        M = cls.allocate(a.shape[0], a.shape[1], label)
        _check(lib().msw_upload(M.h, a.ctypes.data))
        return M

    @classmethod
    def from_csc(cls, csc, label: str | None = None, index_base: int = 0) -> "Matrix":
        val = np.ascontiguousarray(csc.val)
        cplx = np.iscomplexobj(val)
        val = val.astype(np.complex128 if cplx else np.float64, copy=False)
        label = label or ("gzcsc" if cplx else "gdcsc")
        cp = np.ascontiguousarray(csc.colptr, dtype=np.int32)
        ri = np.ascontiguousarray(csc.rowind, dtype=np.int32)
        if index_base:
            cp, ri = cp + index_base, ri + index_base
        h = ct.c_void_p()
        _check(lib().msw_register_csc(ct.byref(h), _lbl(label, 5), csc.dim1, csc.dim2, int(cp[-1] - index_base),
                                      cp.ctypes.data, ri.ctypes.data, val.ctypes.data, index_base))
        return cls(h.value)

    @classmethod
    def from_coo(cls, rows, cols, vals, dim1: int, dim2: int, label: str | None = None,
                 index_base: int = 0) -> "Matrix":
        """COO registration (psp_register_spm 'coo' + psp_coo2csc); repeats are summed."""
        vals = np.ascontiguousarray(vals)
        cplx = np.iscomplexobj(vals)
        vals = vals.astype(np.complex128 if cplx else np.float64, copy=False)
        label = label or ("gzcsc" if cplx else "gdcsc")
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.ascontiguousarray(cols, dtype=np.int32)
        h = ct.c_void_p()
        _check(lib().msw_register_coo(ct.byref(h), _lbl(label, 5), dim1, dim2, len(r), r.ctypes.data, c.ctypes.data,
                                      vals.ctypes.data, index_base))
        return cls(h.value)

    def copy_thre(self, label: str, threshold: float, soft: bool = False) -> "Matrix":
        """m_copy with threshold (MatrixSwitch.F90:630-900)."""
        h = ct.c_void_p()
        _check(lib().msw_copy_thre(ct.byref(h), self.h, _lbl(label, 5), float(threshold), bool(soft)))
        return Matrix(h.value)

    def csc(self):
        """The CSC arrays as a synth.CSCMatrix (host copy)."""
        from .synth import CSCMatrix

        d1, d2, z, s = self.dims()
        if not s:
            raise ValueError("csc() of a dense matrix")
        nnz = ct.c_int(0)
        _check(lib().msw_csc_arrays(self.h, ct.byref(nnz), None, None, None))
        cp = np.zeros(d2 + 1, dtype=np.int32)
        ri = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value, dtype=np.complex128 if z else np.float64)
        _check(lib().msw_csc_arrays(self.h, ct.byref(nnz), cp.ctypes.data, ri.ctypes.data, val.ctypes.data))
        return CSCMatrix(d1, d2, cp, ri, val)

    def copy(self, label: str) -> "Matrix":
        h = ct.c_void_p()
        _check(lib().msw_copy(ct.byref(h), self.h, _lbl(label, 5)))
        return Matrix(h.value)

    # ---------------------------------------------------------- accessors
    def dims(self):
        d1, d2, z, s = ct.c_int(), ct.c_int(), ct.c_int(), ct.c_int()
        _check(lib().msw_dims(self.h, ct.byref(d1), ct.byref(d2), ct.byref(z), ct.byref(s)))
        return d1.value, d2.value, bool(z.value), bool(s.value)

    @property
    def shape(self):
        d = self.dims()
        return d[0], d[1]

    @property
    def is_complex(self) -> bool:
        return self.dims()[2]

    def numpy(self) -> np.ndarray:
        d1, d2, z, s = self.dims()
        if s:
            raise ValueError("numpy() of a CSC matrix: use copy('gdden') first")
        out = np.zeros((d1, d2), dtype=np.complex128 if z else np.float64, order="F")
        _check(lib().msw_download(self.h, out.ctypes.data))
        return out

    def upload(self, a: np.ndarray):
        d1, d2, z, _ = self.dims()
        a = np.asfortranarray(a, dtype=np.complex128 if z else np.float64)
        assert a.shape == (d1, d2)
        _check(lib().msw_upload(self.h, a.ctypes.data))

    def device_ptr(self) -> int:
        return lib().msw_device_ptr(self.h) or 0


# ---------------------------------------------------------------- MatrixSwitch ops
def mm_multiply(A, opA, B, opB, C, alpha=1.0, beta=0.0, label="gpu"):
    if C.is_complex and (isinstance(alpha, complex) or isinstance(beta, complex)):
        _check(lib().msw_mm_zmultiply(A.h, opA.encode(), B.h, opB.encode(), C.h, _z(alpha), _z(beta), _lbl(label, 3)))
    else:
        _check(lib().msw_mm_dmultiply(A.h, opA.encode(), B.h, opB.encode(), C.h, float(np.real(alpha)),
                                      float(np.real(beta)), _lbl(label, 3)))


def m_add(A, opA, C, alpha=1.0, beta=0.0, label="gpu"):
    if isinstance(alpha, complex) or isinstance(beta, complex):
        _check(lib().msw_m_zadd(A.h, opA.encode(), C.h, _z(alpha), _z(beta), _lbl(label, 3)))
    else:
        _check(lib().msw_m_dadd(A.h, opA.encode(), C.h, float(alpha), float(beta), _lbl(label, 3)))


def m_trace(A, label="gpu"):
    o = (ct.c_double * 2)()
    _check(lib().msw_m_ztrace(A.h, o, _lbl(label, 3)))
    return complex(o[0], o[1]) if A.is_complex else o[0]


def mm_trace(A, B, label="gpu"):
    o = (ct.c_double * 2)()
    _check(lib().msw_mm_ztrace(A.h, B.h, o, _lbl(label, 3)))
    return complex(o[0], o[1]) if A.is_complex else o[0]


def m_scale(C, beta, label="gpu"):
    _check(lib().msw_m_zscale(C.h, _z(beta), _lbl(label, 3)))


def m_set(C, seC, alpha, beta, label="gpu"):
    _check(lib().msw_m_zset(C.h, seC.encode(), _z(alpha), _z(beta), _lbl(label, 3)))


def m_set_element(C, i, j, alpha, beta=0.0, label="gpu"):
    _check(lib().msw_m_zset_element(C.h, i, j, _z(alpha), _z(beta), _lbl(label, 3)))


def m_get_element(C, i, j, label="gpu"):
    o = (ct.c_double * 2)()
    _check(lib().msw_m_zget_element(C.h, i, j, o, _lbl(label, 3)))
    return complex(o[0], o[1]) if C.is_complex else o[0]


# ---------------------------------------------------------------- pspBLAS
def psp_gemspm(M, N, K, A, opA, B, opB, C, alpha=1.0, beta=0.0):
    if C.is_complex:
        _check(lib().psp_gpu_zgemspm(M, N, K, A.h, opA.encode(), B.h, opB.encode(), C.h, _z(alpha), _z(beta)))
    else:
        _check(lib().psp_gpu_dgemspm(M, N, K, A.h, opA.encode(), B.h, opB.encode(), C.h, float(alpha), float(beta)))


def psp_gespmm(M, N, K, A, opA, B, opB, C, alpha=1.0, beta=0.0):
    if C.is_complex:
        _check(lib().psp_gpu_zgespmm(M, N, K, A.h, opA.encode(), B.h, opB.encode(), C.h, _z(alpha), _z(beta)))
    else:
        _check(lib().psp_gpu_dgespmm(M, N, K, A.h, opA.encode(), B.h, opB.encode(), C.h, float(alpha), float(beta)))


# ---------------------------------------------------------------- libOMM
def omm(m, n, H, S, new_S, D_min, calc_ED, eta, C_min, init_C, T=None, scale_T=0.0, flavour=0, np_=1, ip=1,
        cg_tol=-1.0, long_out=False, dealloc=False, m_storage=None, m_operation="gpu"):
    """omm (libOMM/src/omm.F90:5-51); returns (e_min, status) with status OMM_OK or OMM_NOT_CONVERGED."""
    if m_storage is None:
        m_storage = "gzden" if C_min.is_complex else "gdden"
    e = ct.c_double(0.0)
    rc = lib().omm_gpu(m, n, H.h, S.h if S is not None else None, bool(new_S), ct.byref(e), D_min.h, bool(calc_ED),
                       float(eta), C_min.h, bool(init_C), T.h if T is not None else None, float(scale_T),
                       int(flavour), int(np_), int(ip), float(cg_tol), bool(long_out), bool(dealloc),
                       _lbl(m_storage, 5), _lbl(m_operation, 3))
    _check(rc)
    return e.value, rc


def psp_den2sp(den: "Matrix", thre: float = 0.0, label: str | None = None) -> "Matrix":
    """psp_den2sp (pspBasicTool.F90:205-421): nonzeros (thre = 0) or |a| >= thre."""
    label = label or ("gzcsc" if den.is_complex else "gdcsc")
    h = ct.c_void_p()
    _check(lib().psp_gpu_den2sp(den.h, float(thre), _lbl(label, 5), ct.byref(h)))
    return Matrix(h.value)


def psp_sp2den(sp: "Matrix", label: str | None = None) -> "Matrix":
    """psp_sp2den (pspBasicTool.F90:423-533)."""
    label = label or ("gzden" if sp.is_complex else "gdden")
    h = ct.c_void_p()
    _check(lib().psp_gpu_sp2den(sp.h, _lbl(label, 5), ct.byref(h)))
    return Matrix(h.value)


def tomato_TB(template_basedir, system_label, switch1, frac_occ, num_orbs_per_atom, switch2, num_orbs,
              num_cells_dir, switch3, sparsity, orb_r_cut, gamma_point, k_point, defect, defect_perturbation,
              m_storage="sdden", build_matrix=True) -> dict:
    """tomato_TB (tomato/src/tomato_TB.F90:1-636) on the GPU: the reference's arguments, with the
    in/out scalars returned in a dict beside H and S (Matrix handles in m_storage, or None: S
    without an overlap, both with build_matrix False)."""
    fo, nopa, no = ct.c_double(frac_occ), ct.c_int(num_orbs_per_atom), ct.c_int(num_orbs)
    ncd = (ct.c_int * 3)(*num_cells_dir)
    sp, orc, nocc = ct.c_double(sparsity), ct.c_double(orb_r_cut), ct.c_int(0)
    kp = (ct.c_double * 3)(*k_point)
    h, s_ = ct.c_void_p(), ct.c_void_p()
    _check(lib().tomato_gpu_TB(str(template_basedir).encode(), str(system_label).encode(), bool(switch1),
                               ct.byref(fo), ct.byref(nopa), bool(switch2), ct.byref(no), ncd, bool(switch3),
                               ct.byref(sp), ct.byref(orc), ct.byref(nocc), bool(gamma_point),
                               ct.cast(kp, ct.POINTER(ct.c_double)), bool(defect), float(defect_perturbation),
                               ct.byref(h), ct.byref(s_), _lbl(m_storage, 5), bool(build_matrix)))
    return dict(num_orbs_per_atom=nopa.value, frac_occ=fo.value, num_orbs=no.value, num_cells_dir=list(ncd),
                orb_r_cut=orc.value, num_occ_states=nocc.value, k_point=list(kp), sparsity=sp.value,
                H=Matrix(h.value) if h.value else None, S=Matrix(s_.value) if s_.value else None)


def omm_callback(m, n, H, S, new_S, D_min, calc_ED, eta, C_min, init_C, T=None, scale_T=0.0, flavour=0, np_=1,
                 ip=1, cg_tol=-1.0, long_out=False, dealloc=False, m_storage=None, m_operation="gpu"):
    """omm_callback (libOMM/src/omm_callback.F90:5-673): H is a Python routine H(C, HC) that sets
    HC = C*H on the lent device matrices (through this module's functions).  Returns
    (e_min, status); an exception inside H aborts the solve with OMM_ERR_CALLBACK."""
    if m_storage is None:
        m_storage = "gzden" if C_min.is_complex else "gdden"
    failure = []

    def trampoline(c, hc, _user):
        try:
            H(Matrix(c, owned=False), Matrix(hc, owned=False))
            return 0
        except Exception as exc:  # reported after the library returns
            failure.append(exc)
            return 1

    fn = H_FN(trampoline)
    e = ct.c_double(0.0)
    rc = lib().omm_gpu_callback(m, n, fn, None, S.h if S is not None else None, bool(new_S), ct.byref(e),
                                D_min.h, bool(calc_ED), float(eta), C_min.h, bool(init_C),
                                T.h if T is not None else None, float(scale_T), int(flavour), int(np_), int(ip),
                                float(cg_tol), bool(long_out), bool(dealloc), _lbl(m_storage, 5),
                                _lbl(m_operation, 3))
    if rc < 0 and failure:
        raise OmmError(rc, "%s (raised in H: %r)" % (lib().omm_gpu_last_error().decode(), failure[0]))
    _check(rc)
    return e.value, rc


def stats() -> dict:
    s = omm_gpu_stats()
    _check(lib().omm_gpu_get_stats(ct.byref(s)))
    return {k: getattr(s, k) for k, _ in omm_gpu_stats._fields_}


def set_log(path):
    _check(lib().omm_gpu_set_log(path.encode() if path else None))


def set_mixed(bf16_tol=1e-5, split_tol=1e-8, refine_factor=0.1):
    """Stage tolerances of the "gmx" solver (see omm_gpu_set_mixed in include/ommgpu.h)."""
    _check(lib().omm_gpu_set_mixed(float(bf16_tol), float(split_tol), float(refine_factor)))


def kernel_launches() -> int:
    return int(lib().omm_gpu_kernel_launches())


def pool_stats() -> dict:
    """Device pool counters: cudaMalloc calls and bytes since start-up, blocks freed, bytes held."""
    out = (ct.c_longlong * 4)()
    _check(lib().omm_gpu_pool_stats(out))
    return {"mallocs": out[0], "malloc_bytes": out[1], "frees": out[2], "cached_bytes": out[3]}


def set_stream(stream_ptr: int):
    _check(lib().omm_gpu_set_stream(ct.c_void_p(stream_ptr)))


def finalize():
    _check(lib().omm_gpu_finalize())


def functional_grad(m, n, H, S, C, G) -> float:
    om = ct.c_double(0.0)
    _check(lib().omm_gpu_functional_grad(m, n, H.h, S.h if S is not None else None, C.h, G.h, ct.byref(om)))
    return om.value


def energy_adjoint(m, n, S, C, V) -> np.ndarray:
    arr = (ct.c_void_p * max(1, len(V)))(*[v.h.value for v in V])
    out = np.zeros(len(V))
    _check(lib().omm_gpu_energy_adjoint(m, n, S.h if S is not None else None, C.h, len(V), arr,
                                        out.ctypes.data_as(ct.POINTER(ct.c_double))))
    return out


def spmm_lowp(A, B, C, nseg=1, B2=None, C2=None) -> int:
    """C = A*B (and C2 = A*B2) with the reduced-precision SpMM; returns the kernel path
    (2 tensor cores, 1 FP32, 0 FP64)."""
    path = ct.c_int(-1)
    _check(lib().omm_gpu_spmm_lowp(A.h, B.h, C.h, B2.h if B2 is not None else None,
                                   C2.h if C2 is not None else None, int(nseg), ct.byref(path)))
    return path.value


def spmm_lowp_prepare(A, nseg=1):
    _check(lib().omm_gpu_spmm_lowp_prepare(A.h, int(nseg)))


def spmm_lowp_apply(B, C, nseg=1, B2=None, C2=None):
    _check(lib().omm_gpu_spmm_lowp_apply(B.h, C.h, B2.h if B2 is not None else None,
                                         C2.h if C2 is not None else None, int(nseg)))


def spmm_plan_info(B) -> dict:
    """The column-group plan of a CSC matrix: G, ngroups, fill, column_groups."""
    g, ng, cg = ct.c_int(0), ct.c_int(0), ct.c_int(0)
    fill = ct.c_double(0.0)
    _check(lib().omm_gpu_spmm_plan_info(B.h, ct.byref(g), ct.byref(ng), ct.byref(fill), ct.byref(cg)))
    return {"G": g.value, "ngroups": ng.value, "fill": fill.value, "column_groups": bool(cg.value)}


def tc_errors() -> int:
    bits = ct.c_uint(0)
    _check(lib().omm_gpu_tc_errors(ct.byref(bits)))
    return bits.value


def header_functions(path: str = HEADER) -> list:
    """Names of the functions declared in include/ommgpu.h."""
    import re

    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = re.sub(r"^\s*typedef[^;]*;", "", txt, flags=re.M | re.S)  # function-pointer types are not symbols
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*([a-z_][a-z0-9_]*)\s*\(", txt,
                                 flags=re.M)))
