"""TEST INFRASTRUCTURE — the CPU FP64 oracle for libOMM's omm() and its products.

ctypes binding of ``oracle/build/liboracle.so`` (built from ``omm_oracle.cpp`` by
``oracle/Makefile``).  Only tests, ``__graft_entry__.smoke()`` and the CPU arms
of ``bench.py`` use this module, as the checker; the GPU library never does.

Conventions follow the reference: C is n x m column-major (rows are Wannier
functions, libOMM/src/omm.F90:50), H and S are m x m, and a CSC matrix holds
0-based column offsets and 0-based row indices (MatrixSwitch's serial CSC,
MatrixSwitch_m_copy.F90:495-547, shifted to 0-based rows).
"""
from __future__ import annotations

import ctypes as ct
import glob
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class orc_mat(ct.Structure):
    _fields_ = [
        ("dim1", ct.c_int),
        ("dim2", ct.c_int),
        ("is_csc", ct.c_int),
        ("nnz", ct.c_int),
        ("val", ct.c_void_p),
        ("colptr", ct.c_void_p),
        ("rowind", ct.c_void_p),
    ]


@dataclass
class CSC:
    """Compressed sparse column matrix (0-based offsets and rows)."""

    dim1: int
    dim2: int
    colptr: np.ndarray  # int32, dim2+1
    rowind: np.ndarray  # int32, nnz
    val: np.ndarray  # float64 or complex128, nnz

    @staticmethod
    def from_dense(a: np.ndarray, threshold: float = 0.0) -> "CSC":
        a = np.asarray(a)
        mask = np.abs(a) > threshold
        cols = [np.nonzero(mask[:, j])[0] for j in range(a.shape[1])]
        colptr = np.zeros(a.shape[1] + 1, dtype=np.int32)
        colptr[1:] = np.cumsum([len(c) for c in cols])
        rowind = np.concatenate(cols).astype(np.int32) if cols else np.zeros(0, np.int32)
        val = np.concatenate([a[c, j] for j, c in enumerate(cols)]) if cols else np.zeros(0, a.dtype)
        return CSC(a.shape[0], a.shape[1], colptr, rowind, np.ascontiguousarray(val))

    @staticmethod
    def from_scipy(sp) -> "CSC":
        sp = sp.tocsc()
        sp.sort_indices()
        return CSC(sp.shape[0], sp.shape[1], sp.indptr.astype(np.int32), sp.indices.astype(np.int32),
                   np.ascontiguousarray(sp.data))

    def to_dense(self) -> np.ndarray:
        out = np.zeros((self.dim1, self.dim2), dtype=self.val.dtype, order="F")
        for j in range(self.dim2):
            s, e = self.colptr[j], self.colptr[j + 1]
            out[self.rowind[s:e], j] = self.val[s:e]
        return out

    @property
    def nnz(self) -> int:
        return int(self.colptr[-1])


def openblas_path() -> str:
    import scipy

    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    libs = sorted(glob.glob(os.path.join(d, "libscipy_openblas-*.so")))
    if not libs:
        raise RuntimeError("SciPy's bundled OpenBLAS was not found in " + d)
    return libs[0]


def build() -> str:
    import subprocess

    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "build", "liboracle.so")


def lib(nthreads: int = 0):
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "build", "liboracle.so")
        src = os.path.join(_HERE, "omm_oracle.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ct.CDLL(path)
        L.orc_last_error.restype = ct.c_char_p
        L.orc_init.argtypes = [ct.c_char_p, ct.c_int]
        L.orc_ctx_new.restype = ct.c_void_p
        L.orc_ctx_free.argtypes = [ct.c_void_p]
        P = ct.POINTER(orc_mat)
        L.orc_omm.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, P, P, ct.c_int, ct.POINTER(ct.c_double),
                              P, ct.c_int, ct.c_double, P, ct.c_int, P, ct.c_double, ct.c_int, ct.c_int, ct.c_int,
                              ct.c_double, ct.c_int, ct.c_void_p, ct.c_int, ct.POINTER(ct.c_int), ct.c_int]
        L.orc_mm_multiply.argtypes = [ct.c_int, P, ct.c_char, P, ct.c_char, P, ct.c_double, ct.c_double,
                                      ct.c_double, ct.c_double, ct.c_int]
        L.orc_calc_coeff.argtypes = [ct.c_int, ct.c_int] + [ct.c_void_p] * 7
        L.orc_mm_trace.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p]
        L.orc_mm_trace.restype = ct.c_double
        L.orc_solve_quartic.argtypes = [ct.c_void_p, ct.POINTER(ct.c_double), ct.POINTER(ct.c_int)]
        L.orc_lcg_init.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p]
        L.orc_calc_G.argtypes = [ct.c_int, ct.c_int, ct.c_int] + [ct.c_void_p] * 5
        rc = L.orc_init(openblas_path().encode(), int(nthreads))
        if rc != 0:
            raise RuntimeError("oracle init failed: " + L.orc_last_error().decode())
        _LIB = L
    elif nthreads:
        _LIB.orc_init(openblas_path().encode(), int(nthreads))
    return _LIB


def _fortran(a: np.ndarray, dtype) -> np.ndarray:
    if not (a.flags.f_contiguous and a.dtype == dtype):
        raise ValueError("expected a Fortran-ordered %s array" % np.dtype(dtype))
    return a


def _mat(a, keep: list) -> orc_mat:
    if isinstance(a, CSC):
        keep.extend([a.colptr, a.rowind, a.val])
        return orc_mat(a.dim1, a.dim2, 1, a.nnz, a.val.ctypes.data, a.colptr.ctypes.data, a.rowind.ctypes.data)
    keep.append(a)
    return orc_mat(a.shape[0], a.shape[1], 0, 0, a.ctypes.data, None, None)


class OmmOracle:
    """Stateful restatement of ``omm`` (libOMM/src/omm.F90:5-672).

    The module-SAVEd per-``ip`` state of the reference lives in this object.
    Arrays passed in are modified in place exactly as the reference modifies
    its ``type(matrix)`` arguments (C_min, D_min, and H/S in the Cholesky
    flavour).
    """

    def __init__(self, nthreads: int = 0):
        self._L = lib(nthreads)
        self._ctx = self._L.orc_ctx_new()
        self.history: list[float] = []
        self.icg = 0

    def __del__(self):
        try:
            self._L.orc_ctx_free(self._ctx)
        except Exception:
            pass

    def omm(self, m, n, H, S, new_S, D_min, calc_ED, eta, C_min, init_C, T=None, scale_T=0.0, flavour=0, np_=1,
            ip=1, cg_tol=-1.0, dealloc=False, hist_cap=100000, max_steps=0):
        is_real = int(np.isrealobj(C_min))
        dt = np.float64 if is_real else np.complex128
        keep: list = []
        for a in (D_min, C_min):
            _fortran(a, dt)
        Hm = _mat(H, keep)
        Sm = _mat(S, keep) if S is not None else None
        Tm = _mat(T, keep) if T is not None else None
        Dm, Cm = _mat(D_min, keep), _mat(C_min, keep)
        e = ct.c_double(0.0)
        hist = np.zeros(hist_cap)
        nh = ct.c_int(0)
        rc = self._L.orc_omm(self._ctx, is_real, m, n, ct.byref(Hm), ct.byref(Sm) if Sm else None, int(new_S),
                             ct.byref(e), ct.byref(Dm), int(calc_ED), float(eta), ct.byref(Cm), int(init_C),
                             ct.byref(Tm) if Tm else None, float(scale_T), int(flavour), int(np_), int(ip),
                             float(cg_tol), int(dealloc), hist.ctypes.data, hist_cap, ct.byref(nh),
                             int(max_steps))
        if rc < 0:
            raise RuntimeError("oracle omm: " + self._L.orc_last_error().decode())
        if not calc_ED:
            self.icg = nh.value
            self.history = list(hist[: min(nh.value, hist_cap)])
        return e.value, rc


def mm_multiply(A, opA, B, opB, C, alpha=1.0, beta=0.0, psp=False):
    """C = alpha*op(A)*op(B) + beta*C (MatrixSwitch mm_multiply / pspBLAS psp_gemspm, psp_gespmm)."""
    L = lib()
    is_real = int(np.isrealobj(C))
    keep: list = []
    a, b, c = _mat(A, keep), _mat(B, keep), _mat(C, keep)
    alpha, beta = complex(alpha), complex(beta)
    rc = L.orc_mm_multiply(is_real, ct.byref(a), opA.encode(), ct.byref(b), opB.encode(), ct.byref(c), alpha.real,
                           alpha.imag, beta.real, beta.imag, int(psp))
    if rc < 0:
        raise RuntimeError(L.orc_last_error().decode())
    return C


def calc_coeff(HW, SW, HWd, SWd, HWdd, SWdd) -> np.ndarray:
    """Quartic line-search coefficients from the six n x n matrices (omm_ops.F90:156-219)."""
    L = lib()
    is_real = int(np.isrealobj(HW))
    mats = [np.asfortranarray(x) for x in (HW, SW, HWd, SWd, HWdd, SWdd)]
    out = np.zeros(5)
    rc = L.orc_calc_coeff(is_real, HW.shape[0], *[x.ctypes.data for x in mats], out.ctypes.data)
    if rc < 0:
        raise RuntimeError(L.orc_last_error().decode())
    return out


def mm_trace(A, B) -> float:
    L = lib()
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    return L.orc_mm_trace(int(np.isrealobj(A)), A.shape[0], A.shape[1], A.ctypes.data, B.ctypes.data)


def solve_quartic(c):
    """omm_solve_quartic (libOMM/src/omm_quartic.F90:60-153) -> (x_min, fail)."""
    L = lib()
    c = np.ascontiguousarray(c, dtype=np.float64)
    x = ct.c_double(0.0)
    f = ct.c_int(0)
    L.orc_solve_quartic(c.ctypes.data, ct.byref(x), ct.byref(f))
    return x.value, bool(f.value)


def lcg_init(n, m, complex_=False) -> np.ndarray:
    """C0 of the reference under NORAND (omm.F90:329-342, omm_rand.F90:19-55)."""
    L = lib()
    C = np.zeros((n, m), dtype=np.complex128 if complex_ else np.float64, order="F")
    L.orc_lcg_init(0 if complex_ else 1, n, m, C.ctypes.data)
    return C


def calc_G(HW, SW, HC, SC) -> np.ndarray:
    """G = 4 HC - 2 SW HC - 2 HW SC (omm_ops.F90:17-39)."""
    L = lib()
    n, m = HC.shape
    G = np.zeros_like(np.asfortranarray(HC))
    mats = [np.asfortranarray(x) for x in (HW, SW)]
    hc, sc = np.asfortranarray(HC), np.asfortranarray(SC)
    rc = L.orc_calc_G(int(np.isrealobj(HC)), n, m, mats[0].ctypes.data, mats[1].ctypes.data, G.ctypes.data,
                      hc.ctypes.data, sc.ctypes.data)
    if rc < 0:
        raise RuntimeError(L.orc_last_error().decode())
    return G


# ----------------------------------------------------------------------------------------------
# tomato_TB (tomato/src/tomato_TB.F90:1-636): tight-binding H and S of a periodic supercell built
# by replicating the element list of a template file.  Pure Python restatement, for small cases.
# Parity unpinned: the reference ships neither templates nor expected matrices, and its Fortran
# cannot be compiled here, so this restatement is checked only by reading it against the source.
# ----------------------------------------------------------------------------------------------
def _tomato_info(basedir, label):
    """<basedir>/<label>_template.info (tomato_TB.F90:124-180)."""
    with open(os.path.join(basedir, label + "_template.info")) as f:
        lines = [ln for ln in f.read().splitlines()]
    it = iter(lines)
    nper = int(next(it).split()[0])
    napc = int(next(it).split()[0])
    nocc = int(next(it).split()[0])
    ncut = int(next(it).split()[0])
    cutoffs = [int(next(it).split()[0]) for _ in range(ncut)]
    nbas = int(next(it).split()[0])
    sizes, refs, index = [], [], []
    for _ in range(nbas):
        tok = next(it).split()
        if len(tok) >= 2:  # "size ref idx(1:size)": a subset of the ref-size basis (:166-174)
            sz, ref = int(tok[0]), int(tok[1])
            idx = [int(t) for t in tok[2:2 + sz]]
            full = list(idx)
            for k in range(2, napc + 1):
                full += [(k - 1) * ref + i for i in idx]
            sizes.append(sz)
            refs.append(ref)
            index.append(full)
        else:
            sizes.append(int(tok[0]))
            refs.append(int(tok[0]))
            index.append(None)
    return nper, napc, nocc, cutoffs, sizes, refs, index


def _tomato_elements(path):
    """An element file (tomato_TB.F90:339-378): num_template, then i1 i2 di dj dk H [S]."""
    with open(path) as f:
        first = f.readline()
        num = int(first[2:12])
        ti, td = [], []
        for _ in range(num):
            tok = f.readline().split()
            ti.append([int(t) for t in tok[:5]])
            td.append([float(t.replace("D", "E")) for t in tok[5:]])
    overlap = len(td[0]) >= 2 if td else False
    return num, ti, td, overlap


def tomato_TB(basedir, label, switch1, frac_occ, num_orbs_per_atom, switch2, num_orbs, num_cells_dir, switch3,
              sparsity, orb_r_cut, gamma_point, k_point, defect, defect_perturbation, build_matrix=True):
    """Returns a dict with the (in/out) scalars and, when build_matrix, dense H and S (numpy, real
    for gamma_point, complex otherwise; S None without overlap).  The sparsity estimate samples
    with the NORAND seed 123456 (omm_rand_seed, tomato_TB.F90:597-611)."""
    nper, napc, nocc, cutoffs, sizes, refs, index = _tomato_info(basedir, label)
    ncd = list(num_cells_dir)
    # basis size (:184-208): strict '<' keeps the first closest
    if switch1:
        dmin, ti_ = 999999.9, 0
        for i, sz in enumerate(sizes):
            d = abs(frac_occ - nocc / sz)
            if d < dmin:
                dmin, num_orbs_per_atom, ti_ = d, sz, i
    else:
        j, ti_ = 999999, 0
        for i, sz in enumerate(sizes):
            k = abs(num_orbs_per_atom - sz)
            if k < j:
                j, num_orbs_per_atom, ti_ = k, sz, i
    nopc = num_orbs_per_atom * napc
    frac_occ = nocc / num_orbs_per_atom
    is_subset = sizes[ti_] != refs[ti_]
    # supercell (:212-245); Fortran nint rounds half away from zero
    nint = lambda x: int(np.floor(x + 0.5)) if x >= 0 else -int(np.floor(-x + 0.5))  # noqa: E731
    if switch2:
        ncd[0] = 1 if nper < 3 else max(nint((num_orbs / nopc) ** (1.0 / 3.0)), 1)
        ncd[1] = 1 if nper < 2 else max(nint(np.sqrt((num_orbs / nopc) / ncd[0])), 1)
        ncd[2] = 1 if nper < 1 else max(nint((num_orbs / nopc) / (ncd[0] * ncd[1])), 1)
    else:
        for i in range(3):
            ncd[i] = 1 if nper < 3 - i else max(ncd[i], 1)
    ncells = ncd[0] * ncd[1] * ncd[2]
    num_orbs = nopc * ncells
    num_occ_states = nocc * napc * ncells

    def elem_path(cut):
        return os.path.join(basedir, "%s_%d_%d.template" % (label, cut, refs[ti_]))

    def num_template_of(cut):
        with open(elem_path(cut)) as f:
            n = int(f.readline()[2:12])
        if is_subset:
            n = n * num_orbs_per_atom ** 2 // refs[ti_] ** 2
        return n

    # orbital cutoff (:249-282)
    if switch3:
        dmin, cut_i = 999999.9, cutoffs[0]
        for c in cutoffs:
            d2 = max(1.0 - num_template_of(c) * ncells / num_orbs ** 2, 0.0)
            d = abs(sparsity - d2)
            if d < dmin:
                dmin, cut_i = d, c
    else:
        j, l_, cut_i = 999999, nint(orb_r_cut * 100.0), cutoffs[0]
        for c in cutoffs:
            k = abs(l_ - c)
            if k < j:
                j, cut_i = k, c
    orb_r_cut = cut_i * 0.01
    kp = list(k_point)
    for d_ in range(3):  # no k points in non-periodic directions (:305-307)
        if nper < 3 - d_:
            kp[d_] = 0.0
    out = dict(num_orbs_per_atom=num_orbs_per_atom, frac_occ=frac_occ, num_orbs=num_orbs, num_cells_dir=ncd,
               orb_r_cut=orb_r_cut, num_occ_states=num_occ_states, k_point=kp, H=None, S=None)
    if not build_matrix:
        out["sparsity"] = max(1.0 - num_template_of(cut_i) * ncells / num_orbs ** 2, 0.0)
        return out
    num, ti, td, overlap = _tomato_elements(elem_path(cut_i))
    dt = np.float64 if gamma_point else np.complex128
    H = np.zeros((num_orbs, num_orbs), dtype=dt)
    S = np.zeros((num_orbs, num_orbs), dtype=dt) if overlap else None
    conv = None
    if is_subset:  # subset_convert (:400-404)
        conv = [0] * (napc * refs[ti_] + 1)
        for i in range(nopc):
            conv[index[ti_][i]] = i + 1
    cell_index = {}
    c = 0
    for i in range(ncd[0]):
        for j in range(ncd[1]):
            for k in range(ncd[2]):
                cell_index[(i, j, k)] = c
                c += nopc
    for l_ in range(num):
        o1, o2, di, dj, dk = ti[l_]
        if is_subset:
            if conv[o1] == 0 or conv[o2] == 0:
                continue
            o1, o2 = conv[o1], conv[o2]
        for i in range(ncd[0]):
            for j in range(ncd[1]):
                for k in range(ncd[2]):
                    i2, j2, k2 = (i + di) % ncd[0], (j + dj) % ncd[1], (k + dk) % ncd[2]
                    a = cell_index[(i, j, k)] + o1 - 1
                    b = cell_index[(i2, j2, k2)] + o2 - 1
                    if gamma_point:
                        ph = 1.0
                    else:  # wrap counts of the image (:486-491), Fortran integer division
                        i3 = int((i + 1 + di - (i2 + 1)) / ncd[0])
                        j3 = int((j + 1 + dj - (j2 + 1)) / ncd[1])
                        k3 = int((k + 1 + dk - (k2 + 1)) / ncd[2])
                        ph = np.exp(1j * 2.0 * np.pi * (kp[0] * i3 + kp[1] * j3 + kp[2] * k3))
                    H[a, b] = td[l_][0] * ph + H[a, b]
                    if overlap:
                        S[a, b] = td[l_][1] * ph + S[a, b]
    if defect:  # the cell-0 block of the first atom, scaled (:425-436)
        for l_ in range(num):
            o1, o2, di, dj, dk = ti[l_]
            if is_subset:
                if conv[o1] == 0 or conv[o2] == 0:
                    continue
                o1, o2 = conv[o1], conv[o2]
            if o1 <= num_orbs_per_atom and o2 <= num_orbs_per_atom and di == 0 and dj == 0 and dk == 0:
                H[o1 - 1, o2 - 1] = defect_perturbation * td[l_][0] + H[o1 - 1, o2 - 1]
    # sparsity estimate: num_orbs LCG-sampled elements, fraction that are zero (:560-580)
    seed, nz, m31 = 123456, 0, 1 << 31
    for _ in range(num_orbs):
        seed = (1103515245 * seed + 12345) % m31
        a = int(np.ceil(num_orbs * (seed / m31)))
        seed = (1103515245 * seed + 12345) % m31
        b = int(np.ceil(num_orbs * (seed / m31)))
        if H[a - 1, b - 1] == 0:
            nz += 1
    out.update(H=H, S=S, sparsity=nz / num_orbs)
    return out
